"""bbjd_b200 -- B200-native JDQZ eigensolver, a drop-in for the reference's
``jdqz`` C and Python API (kyle-augustson/BBJD).

``jdqz`` is re-exported here (reference __init__.py:9-12).  The CUDA library
is loaded on first use; without it every solver call raises (there is no CPU
compute path).
"""
from .bbjd import (DevicePencil, DevicePreconditioner, SparseLU, jdqz, jdqz_batch,  # noqa: F401
                   jdqz_c, jdqz_device)
from .pencils import BBTPencil, make_pencil, start_vector  # noqa: F401

__all__ = ["jdqz", "jdqz_batch", "jdqz_c", "jdqz_device", "DevicePencil", "DevicePreconditioner", "SparseLU", "BBTPencil",
           "make_pencil", "start_vector"]
