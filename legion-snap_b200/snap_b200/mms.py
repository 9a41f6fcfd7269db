"""The reference's manufactured-solution check (src_opt = 3 decks such as
input/mms.in) through the C ABI: snap_mms_init builds the reference flux and
the per-angle source on the GPU, the (time-dependent) solve runs with that
source added in the sweep, and snap_mms_compare measures the solved scalar
flux against the reference flux (snap.cc:373-388, 451-466, 542-560)."""
from __future__ import annotations

import ctypes as C
import sys

import torch

from . import abi
from .problem import Deck, make_problem

MAX_LIMIT = 0.1     # snap.cc:551-554
AVG_LIMIT = 1e-3    # snap.cc:555-558


def avg_divisor(d: Deck) -> int:
    """The divisor of the reference's average difference: the global cell
    count times the number of spatial chunks times the groups (snap.cc:547-548
    multiplies the global nx, ny, nz by the chunk counts), so a 2x2x2-chunk
    deck reports an average 8 times smaller than the same deck in one
    chunk."""
    npey, npez, ichunk = d.chunks
    return d.cells * ichunk * npey * npez * d.ng


def mms_solve(d: Deck, device: int = 0):
    """Solves the deck's manufactured problem; returns the flux moments, the
    iteration record and {max, min, sum, avg} of |flux/ref - 1|."""
    from .solver import Snap, _ptr, _stream
    if d.nmom != 1:
        raise ValueError("the manufactured solution has no flux moments (nmom = 1)")
    snap = Snap(d, device=device)
    try:
        dp = snap.device_problem(make_problem(d))
        dev = snap.device
        ref = torch.empty(d.ng, d.cells, dtype=torch.float64, device=dev)
        qim = torch.empty(8, d.ng, d.cells, d.nang, dtype=torch.float64, device=dev)
        qi = torch.zeros(d.ng, d.cells, dtype=torch.float64, device=dev)
        npey, npez, ichunk = d.chunks
        chunk_cells = (C.c_int * 3)(d.nx // ichunk, d.ny // npey, d.nz // npez)
        abi.check(snap.lib.snap_mms_init(
            snap.handle, _ptr(dp["mat"]), _ptr(dp["sigt"]), _ptr(dp["slgg"]), C.c_double(d.lx),
            C.c_double(d.ly), C.c_double(d.lz), chunk_cells, int(d.timedep), C.c_double(d.tf),
            C.c_double(d.dt), _ptr(ref), _ptr(qim), _ptr(qi), _stream()))
        dp["qi"] = qi                  # steady state: no fixed source (snap.cc:351-355)
        dp["qim"] = qim
        flux, rec = snap.transport_solve(dp)
        out = (C.c_double * 3)()
        abi.check(snap.lib.snap_mms_compare(snap.handle, _ptr(flux), _ptr(ref), out, _stream()))
        res = dict(max=out[0], min=out[1], sum=out[2], avg=out[2] / avg_divisor(d))
        return flux, rec, res, ref
    finally:
        snap.close()


def run_mms(d: Deck, device: int = 0, out=None):
    """The MMS deck run with the reference's report lines (snap.cc:546-559)."""
    from .input_deck import convergence_log
    out = sys.stdout if out is None else out
    flux, rec, res, _ = mms_solve(d, device)
    convergence_log(rec["records"], out)
    print(f"MMS Max Diff: {res['max']:.8g}", file=out)
    print(f"MMS Min Diff: {res['min']:.8g}", file=out)
    print(f"MMS Avg Diff: {res['avg']:.8g}", file=out)
    if res["max"] > MAX_LIMIT:
        print("MMS FAILURE! MAX IS LARGER THAN 0.1!", file=out)
    if res["avg"] > AVG_LIMIT:
        print("MMS FAILURE! AVG IS LARGER THAN 0.001!", file=out)
    rec["mms"] = res
    return flux, rec
