"""snap_sweep_noalloc: the sweep for callers that cannot allocate device
memory (code where cudaMalloc is unavailable or forbidden, e.g. inside
another library's allocator-free section or a real-time loop, and which
therefore cannot call snap_create).  Its scratch is a static device array;
this checks, through the C ABI, that it gives the same flux as the regular
context-based snap_sweep on two calls in a row (the second call sees the
scratch left over by the first).  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device"),
]

from snap_b200 import abi  # noqa: E402
from snap_b200 import problem as P  # noqa: E402

TOL = 1e-12


def config(d, host):
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    return abi.SnapConfig(d.nx, d.ny, d.nz, d.nang, d.ng, d.nmom, 2, int(d.fixup), abi.SNAP_FP64,
                          2.0 * d.nx / d.lx, 2.0 * d.ny / d.ly, 2.0 * d.nz / d.lz,
                          *(dp(a) for a in host))


@pytest.mark.parametrize("d", [P.deck(1), P.Deck(16, 16, 16, nang=36, ng=3, nmom=4)],
                         ids=["deck1", "A36_cmom16"])
def test_noalloc_sweep_matches_context_sweep(d):
    from snap_b200.solver import Snap
    lib = abi.load()
    host = [np.ascontiguousarray(a) for a in P.quadrature(d.nang, d.nmom)]
    cfg = config(d, host)
    prob = P.make_problem(d)
    snap = Snap(d)
    t_xs = snap.expand_cross_section(torch.as_tensor(prob["sigt"], device="cuda"),
                                     torch.as_tensor(prob["mat"], device="cuda"))
    rng = np.random.default_rng(21)
    stream = torch.cuda.current_stream().cuda_stream
    # set-up call (all arrays NULL): places the static array and the sweep's
    # code on the device, so the sweeps below reserve no device memory
    abi.check(lib.snap_sweep_noalloc(C.byref(cfg), None, None, None, stream))
    for call in range(2):
        q = rng.uniform(0.0, 1.0, size=(d.ng, d.cells, d.cmom))
        if d.cmom > 1:
            q[..., 1:] *= 0.2
        qtot = torch.as_tensor(q, device="cuda")
        want = snap.mini_kba_sweep(qtot, t_xs)
        got = torch.full_like(want, float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.snap_sweep_noalloc(C.byref(cfg), qtot.data_ptr(), t_xs.data_ptr(),
                                    got.data_ptr(), stream)
        abi.check(rc)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before, "the sweep reserved device memory"
        w, g = want.cpu().numpy(), got.cpu().numpy()
        scale = np.abs(w).reshape(-1, d.cmom).max(axis=0)
        err = (np.abs(g - w).reshape(-1, d.cmom).max(axis=0) / scale).max()
        assert err < TOL, (call, err)
    snap.close()


def test_noalloc_rejects_oversized_problem():
    lib = abi.load()
    d = P.deck(2)                      # needs far more than the static scratch
    host = [np.ascontiguousarray(a) for a in P.quadrature(d.nang, d.nmom)]
    cfg = config(d, host)
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.snap_sweep_noalloc(C.byref(cfg), dummy.data_ptr(), dummy.data_ptr(),
                                dummy.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 2   # SNAP_ERR_UNSUPPORTED
    assert b"static limit" in lib.snap_last_error()


def test_noalloc_rejects_partial_null_arrays():
    lib = abi.load()
    d = P.deck(1)
    host = [np.ascontiguousarray(a) for a in P.quadrature(d.nang, d.nmom)]
    cfg = config(d, host)
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.snap_sweep_noalloc(C.byref(cfg), dummy.data_ptr(), None, dummy.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    assert rc == 1   # SNAP_ERR_BAD_ARG
