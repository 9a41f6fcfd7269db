"""The sweep's bounded device-side waits, made to run out on purpose.

snap_inject_stall makes one work item of the next sweep launch withhold its
tile-edge progress counter (nothing else changes), so the tiles downstream of
it wait for faces that are never announced.  With a short wait limit
(SNAP_B200_TIMEOUT_MS, read when the context is created) every wait must give
up, the launch must end, the call must return SNAP_ERR_DEVICE_TIMEOUT, and the
same context must then solve normally.  No GPU fault is involved: the waits
end by their limit and the kernel returns."""
import ctypes as C
import os
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device"),
]

from snap_b200 import abi  # noqa: E402
from snap_b200 import problem as P  # noqa: E402

LIMIT_MS = 50


def make_ctx(d):
    from snap_b200.solver import Snap
    old = os.environ.get("SNAP_B200_TIMEOUT_MS")
    os.environ["SNAP_B200_TIMEOUT_MS"] = str(LIMIT_MS)
    try:
        return Snap(d)
    finally:
        if old is None:
            os.environ.pop("SNAP_B200_TIMEOUT_MS")
        else:
            os.environ["SNAP_B200_TIMEOUT_MS"] = old


@pytest.mark.parametrize("item", [0, 5])
def test_withheld_progress_times_out_and_context_recovers(golden_dir, item):
    d = P.deck(1)
    g = np.load(golden_dir / "deck1_ref.npz")
    snap = make_ctx(d)
    dp = snap.device_problem(P.make_problem(d))
    t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"])
    s_xs = snap.expand_scattering_cross_section(dp["slgg"], dp["mat"])
    flux = torch.zeros(d.ng, d.cells, d.cmom, dtype=torch.float64, device="cuda")
    q2 = snap.calc_outer_source(dp["qi"], dp["slgg"], dp["mat"], flux)
    qtot = torch.empty_like(flux)
    abi.check(snap.lib.snap_inject_stall(snap.handle, item))
    t0 = time.time()
    with pytest.raises(abi.SnapError) as ei:
        snap.inner_iteration(s_xs, q2, t_xs, flux, qtot)
    assert ei.value.status == 4          # SNAP_ERR_DEVICE_TIMEOUT
    assert "waited past its limit" in str(ei.value)
    assert time.time() - t0 < 30.0       # ended by the limit, not by a host timeout
    # the same context, next call: a normal solve, equal to the reference's
    flux2, rec = snap.transport_solve(dp)
    phi = flux2[..., 0].cpu().numpy()
    assert float(np.max(np.abs(phi - g["flux0"]) / np.abs(g["flux0"]))) < 1e-12
    assert rec["inners_per_outer"] == list(g["inners_per_outer"])
    snap.close()


def test_inject_stall_rejects_bad_item():
    d = P.deck(1)
    snap = make_ctx(d)
    assert snap.lib.snap_inject_stall(snap.handle, -1) == 1
    assert snap.lib.snap_inject_stall(snap.handle, 10 ** 6) == 1
    snap.close()
