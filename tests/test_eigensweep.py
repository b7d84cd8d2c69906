"""The sweep launcher's host side (CPU) and one sweep on the GPU."""
import argparse

import numpy as np
import pytest

from bbjd_b200 import eigensweep, make_pencil


def _ns(**kw):
    base = dict(synthetic=None, pencil=None, sigmas=None, sigma_file=None, sigma_grid=None)
    base.update(kw)
    return argparse.Namespace(**base)


def test_sigma_sources(tmp_path):
    assert eigensweep._sigmas(_ns(sigmas="3+10j, 3-10j,2")) == [3 + 10j, 3 - 10j, 2 + 0j]
    f = tmp_path / "s.txt"
    f.write_text("1+1j\n\n2-2j\n")
    assert eigensweep._sigmas(_ns(sigma_file=str(f))) == [1 + 1j, 2 - 2j]
    g = eigensweep._sigmas(_ns(sigma_grid="3,-40,40,5"))
    assert g == [complex(3, v) for v in np.linspace(-40, 40, 5)]


def test_pencil_file_round_trip(tmp_path):
    P = make_pencil(8, 12, 3, seed=2)
    A, B = P.to_csc("A").tocsr(), P.to_csc("B").tocsr()
    path = tmp_path / "p.npz"
    np.savez(path, A_data=A.data, A_indices=A.indices, A_indptr=A.indptr, A_shape=A.shape,
             B_data=B.data, B_indices=B.indices, B_indptr=B.indptr, B_shape=B.shape)
    Q = eigensweep._load_pencil(_ns(pencil=str(path)))
    for name in ("Ad", "Al", "Au", "E", "F", "Bd"):
        np.testing.assert_array_equal(getattr(Q, name), getattr(P, name))
    S = eigensweep._load_pencil(_ns(synthetic="8,12,3,2"))
    np.testing.assert_array_equal(S.Ad, P.Ad)


@pytest.mark.gpu
def test_sweep_on_one_gpu(tmp_path):
    out = tmp_path / "sweep.npz"
    sig = "3+10j,3-10j,3+0j"
    assert eigensweep.main(["--synthetic", "16,120,16,3", "--sigmas", sig, "--k", "3",
                            "--maxiter", "800", "--maxsub", "40", "--minsub", "16",
                            "--threads", "2", "--vectors", "--out", str(out)]) == 0
    z = np.load(out)
    assert list(z["nconv"]) == [3, 3, 3] and list(z["status"]) == [0, 0, 0]
    P = make_pencil(16, 120, 16, seed=3)
    A, B = P.to_csc("A"), P.to_csc("B")
    for i in range(3):
        assert np.all(z[f"residuals_{i}"] < 1e-10)
        for lam, x in zip(z[f"eigenvalues_{i}"], z[f"eigenvectors_{i}"].T):
            assert np.linalg.norm(A @ x - lam * (B @ x)) / np.linalg.norm(x) < 1e-8
    # every shift found its own nearest eigenvalues: the sets differ
    assert np.min(np.abs(z["eigenvalues_0"][:, None] - z["eigenvalues_1"][None, :])) > 1e-6
