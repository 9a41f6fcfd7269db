"""Single-kernel cases for profiling.

Each case runs one small workload through the C ABI and prints the
CUDA-event time of every call, so that a profiler filtering on one kernel
name can capture a launch of it on a few GB of device memory:

    python -m snap_b200.cases sweep --deck 2 --groups 4 [--precision fp32] [--iters 3]
    python -m snap_b200.cases outer-source --deck 2 [--form tcgen05] [--calls 3]
    python -m snap_b200.cases input-deck tests/decks/tiny_4K_1x1x1.in [--inners 3] [--general]
    python -m snap_b200.cases adjoint [--deck 4]

sweep: inner iterations (inner source, sweep of every octant and group,
inner test) of a benchmark deck with its group count overridden, from a
zero flux and the deck's fixed source.  outer-source: the group-to-group
outer source of a benchmark deck from a seeded random flux, in the FP64
tensor-core form or the split-BF16 tcgen05 form.  input-deck: one time step
of a reference input deck, capped at one outer and `--inners` inner
iterations (`--general` pins the general sweep kernel).  adjoint: a
converged forward solve of a benchmark deck, then the adjoint solve of a
detector response on the 4x4x4 far corner (weights 1/g).
"""
from __future__ import annotations

import argparse
import dataclasses
import os

import torch

from . import input_deck as D
from . import problem as P
from .solver import Snap


def _timed(fn):
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    out = fn()
    en.record()
    torch.cuda.synchronize()
    return out, st.elapsed_time(en)


def sweep_case(deck: int, groups: int, precision: str, iters: int) -> None:
    d = P.deck(deck, ng=groups)
    snap = Snap(d, precision=precision)
    dp = snap.device_problem(P.make_problem(d))
    t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"])
    s_xs = snap.expand_scattering_cross_section(dp["slgg"], dp["mat"])
    flux = torch.zeros(d.ng, d.cells, d.cmom, dtype=torch.float64, device="cuda")
    q2 = snap.calc_outer_source(dp["qi"], dp["slgg"], dp["mat"], flux)
    qtot = torch.empty(flux.shape, dtype=snap.sweep_dtype, device="cuda")
    t_xs = t_xs.to(snap.sweep_dtype)
    for it in range(iters):
        _, ms = _timed(lambda: snap.inner_iteration(s_xs, q2, t_xs, flux, qtot))
        print(f"inner iteration {it}: {ms:.3f} ms {snap.timing(reset=True)}")
    snap.close()


def outer_source_case(deck: int, form: str, calls: int) -> None:
    d = P.deck(deck)
    snap = Snap(d, precision="fp32" if form == "tcgen05" else "fp64")
    dp = snap.device_problem(P.make_problem(d))
    g = torch.Generator(device="cuda").manual_seed(1)
    flux = torch.rand(d.ng, d.cells, d.cmom, dtype=torch.float64, device="cuda", generator=g)
    call = snap.calc_outer_source_tc if form == "tcgen05" else snap.calc_outer_source
    for i in range(calls):
        _, ms = _timed(lambda: call(dp["qi"], dp["slgg"], dp["mat"], flux))
        print(f"outer source ({form}) call {i}: {ms:.3f} ms")
    snap.close()


def input_deck_case(path: str, inners: int, general: bool) -> None:
    if general:
        os.environ["SNAP_B200_TD_GENERAL"] = "1"
    d = D.parse_deck(path).deck
    d = dataclasses.replace(d, nsteps=1, tf=d.dt, oitm=1, iitm=inners)
    snap = Snap(d)
    dp = snap.device_problem(P.make_problem(d))
    (flux, rec), ms = _timed(lambda: snap.transport_solve(dp))
    print(f"{path}: {rec['inner_total']} inner iterations, {ms:.3f} ms, "
          f"scalar flux sum {float(flux[..., 0].sum()):.6e}")
    snap.close()


def adjoint_case(deck: int) -> None:
    d = P.deck(deck)
    snap = Snap(d)
    dp = snap.device_problem(P.make_problem(d))
    r = torch.zeros(d.ng, d.nz, d.ny, d.nx, dtype=torch.float64, device="cuda")
    r[:, -4:, -4:, -4:] = (1.0 / torch.arange(1, d.ng + 1, dtype=torch.float64,
                                              device="cuda"))[:, None, None, None]
    r = r.reshape(d.ng, d.cells)
    (flux, rec), ms = _timed(lambda: snap.transport_solve(dp))
    print(f"forward solve: {rec['inner_total']} inner iterations, {ms:.3f} ms")
    t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"])
    if "sigt_scale" in dp:   # the per-cell sigma_t perturbation of the adjoint deck
        t_xs = t_xs * dp["sigt_scale"][None, :]
    g, ms = _timed(lambda: snap.adjoint_solve(dp, t_xs, flux, r))
    print(f"adjoint solve: {g['iterations']} iterations, {ms:.3f} ms")
    snap.close()


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(prog="python -m snap_b200.cases")
    sub = ap.add_subparsers(dest="case", required=True)
    s = sub.add_parser("sweep")
    s.add_argument("--deck", type=int, default=2)
    s.add_argument("--groups", type=int, default=4)
    s.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    s.add_argument("--iters", type=int, default=3)
    o = sub.add_parser("outer-source")
    o.add_argument("--deck", type=int, default=2)
    o.add_argument("--form", choices=["dmma", "tcgen05"], default="dmma")
    o.add_argument("--calls", type=int, default=3)
    i = sub.add_parser("input-deck")
    i.add_argument("path")
    i.add_argument("--inners", type=int, default=3)
    i.add_argument("--general", action="store_true")
    j = sub.add_parser("adjoint")
    j.add_argument("--deck", type=int, default=4)
    a = ap.parse_args(argv)
    if a.case == "sweep":
        sweep_case(a.deck, a.groups, a.precision, a.iters)
    elif a.case == "outer-source":
        outer_source_case(a.deck, a.form, a.calls)
    elif a.case == "input-deck":
        input_deck_case(a.path, a.inners, a.general)
    else:
        adjoint_case(a.deck)


if __name__ == "__main__":
    main()
