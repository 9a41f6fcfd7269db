"""The reference's own input decks (input/*.in, parsed by snap_b200.input_deck)
solved through the C ABI and compared with the reference's CPU task bodies
(oracle/_ref, built from the reference sources) on the same deck: steady-state
decks of several chunk layouts, and time-dependent decks (vdelt, the
time-edge angular flux, its fixup face) of 32 to 1024 angles per octant.
Shapes outside the tiled sweep (6^3 mesh, more than 64 angles) run the
general kernel; time-dependent decks of at most 64 angles the tiled
kernel's time-dependent form.  FP64: scalar flux within 1e-12 relative, iteration records
identical."""
import dataclasses
import os
import pathlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device"),
]

from oracle.bindings import Oracle, RefSnap  # noqa: E402
from snap_b200 import input_deck as D  # noqa: E402
from snap_b200 import problem as P  # noqa: E402

TOL = 1e-12
DECKS = pathlib.Path(__file__).resolve().parent / "decks"
needs_ref = pytest.mark.skipif(not RefSnap.available(), reason="reference build not present")


def rel_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def solve_both(d):
    from snap_b200.solver import Snap
    prob = P.make_problem(d)
    snap = Snap(d)
    flux, rec = snap.transport_solve(snap.device_problem(prob))
    ref, rref = RefSnap(d).solve(prob, nthreads=os.cpu_count() or 1)
    snap.close()
    return flux[..., 0].cpu().numpy(), rec, ref, rref


@needs_ref
@pytest.mark.parametrize("name", ["simple.in", "test.in", "base.in"])
def test_steady_state_deck_matches_reference(name):
    """simple.in (32^3, one group), test.in (32^3, 4 groups, 2x2x2 chunks),
    base.in (6^3, general kernel)."""
    d = D.parse_deck(DECKS / name).deck
    phi, rec, ref, rref = solve_both(d)
    assert rel_err(phi, ref) < TOL
    assert rec["inners_per_outer"] == rref["inners_per_outer"]
    assert rec["converged"] == rref["converged"]


@needs_ref
@pytest.mark.parametrize("name,steps", [("tiny_512_1x1x1.in", None), ("small_512_1x1x1.in", None),
                                        ("medium_512_1x1x1.in", 4), ("huge_512_1x1x1.in", 2)])
def test_time_dependent_deck_matches_reference(name, steps):
    """Time-dependent decks, 32 / 128 / 256 / 1024 angles per octant (the
    larger ones on fewer time steps to bound the CPU reference's time): the
    scalar flux after the last step and the outer/inner record of every
    step."""
    d = D.parse_deck(DECKS / name).deck
    if steps:
        d = dataclasses.replace(d, nsteps=steps, tf=d.dt * steps)
    phi, rec, ref, rref = solve_both(d)
    assert rel_err(phi, ref) < TOL
    assert rec["inners_per_outer"] == rref["inners_per_outer"]
    assert rec["inner_total"] == rref["inner_total"]


@pytest.mark.parametrize("name", ["tiny_512_1x1x1.in", "mms.in"])
def test_time_dependent_tiled_matches_general(name, monkeypatch):
    """Time-dependent decks of at most 64 angles run the tiled kernel's
    time-dependent form (vdelt * psi_t in the numerator and denominator, the
    time face in the fixup, psi_t out, the manufactured source); the general
    kernel (SNAP_B200_TD_GENERAL=1) gives the same flux to 1e-12 and the same
    iteration record."""
    from snap_b200.mms import mms_solve
    from snap_b200.solver import Snap
    d = D.parse_deck(DECKS / name).deck

    def run():
        if name == "mms.in":
            flux, rec, res, _ = mms_solve(d)
            return flux[..., 0].cpu().numpy(), rec
        snap = Snap(d)
        flux, rec = snap.transport_solve(snap.device_problem(P.make_problem(d)))
        snap.close()
        return flux[..., 0].cpu().numpy(), rec

    tiled, rt = run()
    monkeypatch.setenv("SNAP_B200_TD_GENERAL", "1")
    general, rg = run()
    assert rel_err(tiled, general) < TOL
    assert rt["inners_per_outer"] == rg["inners_per_outer"]


@pytest.mark.parametrize("nang", [20, 36, 64])
def test_task_level_time_dependent_sweep_fixups(nang, monkeypatch):
    """snap_sweep_td with vdelt != 0 and time-edge fluxes that drive many
    faces negative (the time face of the fixup): the tiled and the general
    kernel agree on the flux and on the outgoing time-edge flux to 1e-12
    (3, 5 and 8 angle tiles: the tiled kernel's CTA counts differ)."""
    import ctypes as C  # noqa: F401
    from snap_b200 import abi
    from snap_b200.solver import Snap, _ptr, _stream
    d = P.Deck(16, 16, 8, nang=nang, ng=3, nmom=1, epsi=1e-6, iitm=2, oitm=2)
    snap = Snap(d)
    dp = snap.device_problem(P.make_problem(d))
    t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"])
    g = torch.Generator(device="cuda").manual_seed(11)
    qtot = torch.rand(d.ng, d.cells, 1, dtype=torch.float64, device="cuda", generator=g)
    tf_in = 4.0 * torch.rand(8, d.ng, d.cells, d.nang, dtype=torch.float64, device="cuda",
                             generator=g)
    qim = 0.1 * torch.rand(8, d.ng, d.cells, d.nang, dtype=torch.float64, device="cuda",
                           generator=g)
    vd = torch.tensor([0.0, 2.0, 30.0], dtype=torch.float64, device="cuda")   # one steady group

    def sweep():
        flux = torch.empty(d.ng, d.cells, 1, dtype=torch.float64, device="cuda")
        tf_out = torch.zeros_like(tf_in)
        abi.check(snap.lib.snap_sweep_td(snap.handle, _ptr(qtot), _ptr(t_xs), _ptr(vd),
                                         _ptr(tf_in), _ptr(tf_out), _ptr(qim), _ptr(flux),
                                         _stream()))
        return flux.cpu().numpy(), tf_out.cpu().numpy()

    f_tiled, o_tiled = sweep()
    monkeypatch.setenv("SNAP_B200_TD_GENERAL", "1")
    f_gen, o_gen = sweep()
    assert rel_err(f_tiled, f_gen) < TOL
    assert np.max(np.abs(o_tiled - o_gen)) <= TOL * np.max(np.abs(o_gen))
    assert np.all(o_tiled[:, 0] == 0.0)          # vdelt = 0: no time-edge flux written
    assert np.count_nonzero(o_gen[:, 1:] == 0.0) > 0   # some time faces were set to zero
    snap.close()


@pytest.mark.parametrize("case", ["small_512_1x1x1.in", "ragged_nmom3", "ragged_fixup"])
def test_wavefront_general_sweep_matches_cell_by_cell(case, monkeypatch):
    """The general sweep's wavefront form (the cells of a diagonal plane in
    flight at once, one warp per cell; up to 128 angles) against its
    cell-by-cell form (SNAP_B200_WAVE=0) on whole solves: the 128-angle
    time-dependent deck, a ragged mesh with nmom = 3, and a ragged
    fixup-heavy mesh; flux to 1e-12 and identical iteration records."""
    from snap_b200.solver import Snap
    if case.endswith(".in"):
        d = D.parse_deck(DECKS / case).deck
        d = dataclasses.replace(d, nsteps=2, tf=2 * d.dt)
    elif case == "ragged_nmom3":
        d = P.Deck(12, 10, 6, nang=40, ng=3, nmom=3, epsi=1e-6, iitm=3, oitm=3)
    else:
        d = P.Deck(9, 7, 5, nang=96, ng=2, nmom=1, epsi=1e-6, iitm=3, oitm=3, lx=8.0, ly=8.0,
                   lz=8.0)

    def run():
        snap = Snap(d)
        flux, rec = snap.transport_solve(snap.device_problem(P.make_problem(d)))
        snap.close()
        return flux.cpu().numpy(), rec

    wave, rw = run()
    monkeypatch.setenv("SNAP_B200_WAVE", "0")
    cell, rc = run()
    assert rel_err(wave[..., 0], cell[..., 0]) < TOL
    if d.cmom > 1:
        scale = np.abs(cell).reshape(-1, d.cmom).max(axis=0)
        assert float((np.abs(wave - cell).reshape(-1, d.cmom).max(axis=0) / scale).max()) < TOL
    assert rw["inners_per_outer"] == rc["inners_per_outer"]


@needs_ref
def test_time_dependent_2048_angles():
    """The largest angle count the general kernel takes (four angles per
    thread) on a small time-dependent problem."""
    d = P.Deck(4, 4, 4, nang=2048, ng=2, nmom=1, epsi=1e-4, iitm=3, oitm=4, lx=0.6, ly=0.6,
               lz=0.6, timedep=True, tf=1.0, nsteps=2, mat_opt=1, src_opt=1)
    phi, rec, ref, rref = solve_both(d)
    assert rel_err(phi, ref) < TOL
    assert rec["inners_per_outer"] == rref["inners_per_outer"]


def test_general_kernel_multimoment_matches_oracle():
    """A ragged mesh (the tiled kernel needs nx % 8 == 0) with nmom = 3:
    the general kernel's moment expansion and accumulation against the
    oracle."""
    from snap_b200.solver import Snap
    d = P.Deck(12, 10, 6, nang=20, ng=3, nmom=3, epsi=1e-6, iitm=3, oitm=3)
    prob = P.make_problem(d)
    ref, rref = Oracle(d).solve(prob)
    snap = Snap(d)
    flux, rec = snap.transport_solve(snap.device_problem(prob))
    got = flux.cpu().numpy()
    assert rel_err(got[..., 0], ref[..., 0]) < TOL
    scale = np.abs(ref).reshape(-1, d.cmom).max(axis=0)
    assert float((np.abs(got - ref).reshape(-1, d.cmom).max(axis=0) / scale).max()) < TOL
    assert rec["inners_per_outer"] == rref["inners_per_outer"]
    snap.close()


def test_convergence_log_lines():
    """The iteration records of a solve print as the reference's convergence
    log (one line per inner iteration, per outer test, per time step)."""
    import io
    from snap_b200.solver import Snap
    d = D.parse_deck(DECKS / "tiny_512_1x1x1.in").deck
    d = dataclasses.replace(d, nsteps=2, tf=d.dt * 2)
    snap = Snap(d)
    _, rec = snap.transport_solve(snap.device_problem(P.make_problem(d)))
    out = io.StringIO()
    D.convergence_log(rec["records"], out)
    lines = out.getvalue().splitlines()
    assert sum(line.startswith("Inner loop") for line in lines) == rec["inner_total"]
    assert sum(line.startswith("Time step") for line in lines) == 2
    assert "SNAP Execution Summary" in lines
    snap.close()


# ---------------------------------------------------------------- MMS
# The manufactured per-angle source is a sum of streaming, removal and
# scattering terms several times larger than the solution they produce; the
# two compilers' different fused multiply-add choices in those terms (a few
# units in the last place) reach the flux amplified by that cancellation, so
# the flux is compared at 1e-11 here (the reference flux itself at 1e-12).
MMS_TOL = 1e-11

@needs_ref
@pytest.mark.parametrize("case", ["mms.in", "steady", "unequal_spacing"])
def test_mms_deck_matches_reference(case):
    """input/mms.in (16^3, 16 angles, 4 groups, 2 time steps, manufactured
    source, 2x2x2 chunks) against the reference's own MMS tasks and sweep run
    chunk by chunk: the reference flux to 1e-12, the solved flux, the
    iteration record and the comparison (max, min, sum and average of
    |flux/ref - 1|).  The reference's result passes both thresholds on this
    deck; its average (3.2e-4) is the sum over cells times chunks (2.6e-3
    over the cells alone, a discretisation error of the 16^3 mesh, see the
    refinement test).  unequal_spacing: 16 x 8 x 8 cells on 0.6 x 0.5 x 0.4,
    where each chunk's cell edges start at its first cell times that axis's
    spacing and step by dx, as the reference's per-chunk tasks compute
    them."""
    from snap_b200.mms import AVG_LIMIT, MAX_LIMIT, mms_solve
    d = D.parse_deck(DECKS / "mms.in").deck
    if case == "steady":
        d = dataclasses.replace(d, timedep=False, nsteps=1)
    if case == "unequal_spacing":
        d = dataclasses.replace(d, ny=8, nz=8, ly=0.5, lz=0.4)
    flux, rec, res, ref_flux = mms_solve(d)
    rflux, rrec = RefSnap(d).solve(P.make_problem(d), nthreads=os.cpu_count() or 1)
    assert rel_err(ref_flux.cpu().numpy(), rrec["ref_flux"]) < TOL
    assert rel_err(flux[..., 0].cpu().numpy(), rflux) < MMS_TOL
    assert rec["inners_per_outer"] == rrec["inners_per_outer"]
    for key in ("max", "min", "sum", "avg"):
        assert abs(res[key] - rrec["mms"][key]) <= 1e-9 * abs(rrec["mms"][key]), key
    if case == "mms.in":
        assert res["max"] < MAX_LIMIT and res["avg"] < AVG_LIMIT


def test_mms_error_falls_second_order():
    """The manufactured solution's average error shrinks about fourfold per
    halving of the cell size (8^3 -> 16^3 -> 32^3, the mms.in deck
    otherwise), the order of the diamond-difference scheme; at 32^3 it is
    within the reference's 1e-3 threshold even over the cells alone."""
    from snap_b200.mms import AVG_LIMIT, mms_solve
    d0 = D.parse_deck(DECKS / "mms.in").deck
    avg = []
    for n in (8, 16, 32):
        _, _, res, _ = mms_solve(dataclasses.replace(d0, nx=n, ny=n, nz=n))
        avg.append(res["avg"])
    assert avg[0] / avg[1] > 3.0 and avg[1] / avg[2] > 3.0, avg
    assert avg[2] * 8 < AVG_LIMIT      # the deck's 2x2x2 chunks divide the average by 8


def test_task_level_time_dependent_sweep():
    """snap_sweep_td (the time-dependent MiniKBATask body, general kernel):
    with vdelt = 0 it is the steady sweep of the tiled kernel to 1e-12; with
    vdelt != 0 the time term changes the flux and the outgoing time-edge flux
    is written (the time-dependent decks above pin its values against the
    reference)."""
    import ctypes as C
    from snap_b200.solver import Snap, _ptr, _stream
    d = P.Deck(16, 16, 8, nang=12, ng=3, nmom=2, epsi=1e-6, iitm=2, oitm=2)
    prob = P.make_problem(d)
    snap = Snap(d)
    dp = snap.device_problem(prob)
    t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"])
    rng = np.random.default_rng(5)
    q = rng.uniform(0.0, 1.0, size=(d.ng, d.cells, d.cmom))
    q[..., 1:] *= 0.1
    qtot = torch.as_tensor(q, device="cuda")
    want = snap.mini_kba_sweep(qtot, t_xs)
    tf_in = torch.zeros(8, d.ng, d.cells, d.nang, dtype=torch.float64, device="cuda")
    tf_out = torch.zeros_like(tf_in)
    flux = torch.empty_like(want)
    vz = torch.zeros(d.ng, dtype=torch.float64, device="cuda")
    from snap_b200 import abi
    abi.check(snap.lib.snap_sweep_td(snap.handle, _ptr(qtot), _ptr(t_xs), _ptr(vz), _ptr(tf_in),
                                     _ptr(tf_out), None, _ptr(flux), _stream()))
    scale = want.abs().reshape(-1, d.cmom).amax(0)
    assert float(((flux - want).abs().reshape(-1, d.cmom).amax(0) / scale).max()) < TOL
    # vdelt != 0: the time term changes the flux
    vd = torch.full((d.ng,), 0.5, dtype=torch.float64, device="cuda")
    tf_in.uniform_(0.0, 1.0)
    abi.check(snap.lib.snap_sweep_td(snap.handle, _ptr(qtot), _ptr(t_xs), _ptr(vd), _ptr(tf_in),
                                     _ptr(tf_out), None, _ptr(flux), _stream()))
    assert float((flux - want).abs().max()) > 1e-3
    assert torch.isfinite(tf_out).all()
    snap.close()
