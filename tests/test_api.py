"""Host-side API pieces that need no GPU."""
import numpy as np
import pytest

from bbjd_b200 import jdqz_device
from bbjd_b200.bbjd import _with_oracle


def test_error_vs_oracle_is_the_largest_nearest_distance():
    info = _with_oracle({}, np.array([1.0 + 1e-9j, 2.0]), [2.0 + 1e-7, 1.0, 5.0])
    assert info["error_vs_oracle"] == pytest.approx(1e-7, rel=1e-6)
    assert "error_vs_oracle" not in _with_oracle({}, np.array([1.0]), None)


def test_jdqz_device_takes_only_pencils():
    with pytest.raises(TypeError):
        jdqz_device(np.eye(4), k=1)


def test_device_pencil_arrays_are_size_checked():
    from bbjd_b200 import DevicePencil, make_pencil
    P = make_pencil(8, 4, 2, seed=0)
    d = P.device_arrays()
    bad = dict(d, E=d["E"][:-1])
    with pytest.raises(ValueError, match="'E' must be 64"):
        DevicePencil(arrays=bad, b=8, nblk=4, t=2)
    with pytest.raises(ValueError, match="lacks 'FT'"):
        DevicePencil(arrays={k: v for k, v in d.items() if k != "FT"}, b=8, nblk=4, t=2)
    strided = dict(d, Ad=np.repeat(d["Ad"], 2)[::2])
    with pytest.raises(ValueError, match="not contiguous"):
        DevicePencil(arrays=strided, b=8, nblk=4, t=2)


def test_ritz_estimate_values_checked():
    from bbjd_b200 import jdqz_batch, make_pencil
    P = make_pencil(8, 4, 2, seed=0)
    with pytest.raises(ValueError, match="ritz_estimate must be one of"):
        jdqz_batch([P], [3.0], k=1, ritz_estimate="fp16")
