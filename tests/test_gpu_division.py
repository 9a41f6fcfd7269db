"""The sweep's division arithmetic against CUDA's correctly rounded operations.

The sweep kernels divide by Newton-Raphson refinement of the hardware
reciprocal approximation (sweep.cuh: recip, divide).  This checks, over
operands in the range the sweep meets (denominators sigma_t + geometry terms
between 1e-2 and 1e5, numerators of either sign), that the result is within
one unit in the last place of the correctly rounded 1/b and a/b, in FP64 and
FP32, and that the correctly rounded device results equal the host's IEEE
division.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def ulp_distance(x, y):
    """|x - y| in units in the last place (same-sign finite values)."""
    ix = x.view(np.int64 if x.dtype == np.float64 else np.int32).astype(np.int64)
    iy = y.view(np.int64 if y.dtype == np.float64 else np.int32).astype(np.int64)
    assert np.all(np.sign(x) == np.sign(y))
    return np.abs(ix - iy)


@pytest.mark.parametrize("precision,dtype", [(0, np.float64), (1, np.float32)])
def test_newton_division_within_one_ulp(precision, dtype):
    import sys
    import pathlib
    sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1] / "legion-snap_b200"))
    from snap_b200 import abi
    lib = abi.load()
    rng = np.random.default_rng(7)
    n = 1 << 20
    b = np.exp(rng.uniform(np.log(1e-2), np.log(1e5), n)).astype(dtype)
    a = (rng.uniform(-1.0, 1.0, n) * np.exp(rng.uniform(-20, 20, n))).astype(dtype)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    da = torch.as_tensor(a, device="cuda:0")
    db = torch.as_tensor(b, device="cuda:0")
    out = torch.empty(4 * n, dtype=tdt, device="cuda:0")
    abi.check(lib.snap_selftest_division(precision, da.data_ptr(), db.data_ptr(), n,
                                         out.data_ptr(), None))
    torch.cuda.synchronize()
    o = out.cpu().numpy().reshape(n, 4)
    # the device's correctly rounded operations agree with the host's IEEE ones
    np.testing.assert_array_equal(o[:, 1], (dtype(1) / b).astype(dtype))
    np.testing.assert_array_equal(o[:, 3], (a / b).astype(dtype))
    assert ulp_distance(o[:, 0], o[:, 1]).max() <= 1
    nz = a != 0
    assert ulp_distance(o[nz, 2], o[nz, 3]).max() <= 1
    assert np.all(o[~nz, 2] == 0)
