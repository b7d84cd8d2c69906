"""CPU checker for the B200 engine (test infrastructure, not product).

Holds the numpy restatement of the reference's JDQZ (jdqz_np.py), the C
restatement of the block-bordered LU used as the CPU preconditioner
(c/bbt_oracle.c), and the recipe that builds the reference's own C core from
its sources into oracle/_ref (Makefile).  Only tests/, the smoke() check of
__graft_entry__.py and the CPU-baseline leg of bench.py may import it.
"""
