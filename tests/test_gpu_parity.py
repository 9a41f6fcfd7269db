"""GPU parity: the CUDA path through the C ABI against the reference's golden
vectors and the CPU oracle.  FP64 tolerance: 1e-12 relative in scalar flux
(higher moments: 1e-12 of the moment's largest magnitude)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device"),
]

from oracle.bindings import Oracle  # noqa: E402
from snap_b200 import problem as P  # noqa: E402

TOL = 1e-12


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def moment_err(a, b):
    """max over moments of max|a-b| / max|b| for that moment."""
    a = np.asarray(a).reshape(-1, a.shape[-1])
    b = np.asarray(b).reshape(-1, b.shape[-1])
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return float((np.abs(a - b).max(axis=0) / scale).max())


def snap_ctx(deck, **env):
    from snap_b200.solver import Snap
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        return Snap(deck)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def dev(a, dtype=None):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def random_qtot(deck, seed):
    rng = np.random.default_rng(seed)
    q = rng.uniform(0.0, 1.0, size=(deck.ng, deck.cells, deck.cmom))
    if deck.cmom > 1:
        q[..., 1:] = rng.uniform(-0.2, 0.2, size=q[..., 1:].shape)
    return q


@pytest.fixture(scope="module")
def golden(golden_dir):
    return {k: np.load(golden_dir / f"{k}_ref.npz") for k in ("deck1", "deck2p")}


# ---------------------------------------------------------------- task level
@pytest.mark.parametrize("d", [P.deck(1), P.Deck(16, 8, 8, nang=12, ng=3, nmom=3)])
def test_expand_cross_sections(d):
    prob = P.make_problem(d)
    snap = snap_ctx(d)
    t_xs = snap.expand_cross_section(dev(prob["sigt"]), dev(prob["mat"])).cpu().numpy()
    s_xs = snap.expand_scattering_cross_section(dev(prob["slgg"]), dev(prob["mat"])).cpu().numpy()
    ot, os_ = Oracle(d).expand(prob)
    assert np.array_equal(t_xs, ot)
    assert np.array_equal(s_xs, os_)


@pytest.mark.parametrize("d", [
    P.deck(1), P.Deck(16, 8, 8, nang=12, ng=5, nmom=4),
    P.Deck(16, 16, 8, nang=12, ng=32, nmom=4),    # deck-2 groups and moments (4 x 8 output tiles)
    P.Deck(8, 8, 8, nang=12, ng=64, nmom=3),      # deck-3/5 groups and moments
    P.Deck(7, 5, 3, nang=4, ng=9, nmom=2),        # ragged cell tile and group tiles
    P.Deck(8, 4, 4, nang=4, ng=70, nmom=1),       # beyond 64 groups: the SIMT form
], ids=lambda d: f"{d.nx}x{d.ny}x{d.nz}_G{d.ng}_M{d.cmom}")
def test_outer_and_inner_source(d):
    prob = P.make_problem(d)
    o = Oracle(d)
    _, s_xs = o.expand(prob)
    flux = random_qtot(d, 7)
    snap = snap_ctx(d)
    q2 = snap.calc_outer_source(dev(prob["qi"]), dev(prob["slgg"]), dev(prob["mat"]), dev(flux))
    q2_ref = o.outer_source(prob, flux)
    assert moment_err(q2.cpu().numpy(), q2_ref) < 1e-14
    qtot = snap.calc_inner_source(dev(s_xs), q2, dev(flux)).cpu().numpy()
    assert moment_err(qtot, o.inner_source(s_xs, q2_ref, flux)) < 1e-14


# ---------------------------------------------------------------- sweep
SWEEP_DECKS = [
    P.deck(1),                                           # A=10 (2 angle tiles), one moment
    P.Deck(16, 16, 16, nang=36, ng=3, nmom=4),           # deck-2 angular shape, 16 moments
    P.Deck(16, 8, 24, nang=24, ng=2, nmom=2),            # adjoint-deck shape, 4 moments
    P.Deck(8, 16, 8, nang=48, ng=2, nmom=3),             # deck-3/5 angles, 9 moments
    P.Deck(8, 8, 5, nang=3, ng=1, nmom=1),               # tiny: one tile, ragged angle tile
    P.Deck(8, 8, 8, nang=32, ng=2, nmom=4),              # 4 angle tiles, 16 moments
    P.Deck(8, 8, 6, nang=56, ng=1, nmom=2),              # 7 angle tiles
    P.Deck(8, 4, 6, nang=64, ng=2, nmom=3),              # 8 angle tiles (the tiled kernel's widest)
]


@pytest.mark.parametrize("d", SWEEP_DECKS, ids=lambda d: f"{d.nx}x{d.ny}x{d.nz}_A{d.nang}_M{d.cmom}")
def test_sweep_matches_oracle(d):
    prob = P.make_problem(d)
    o = Oracle(d)
    t_xs, _ = o.expand(prob)
    qtot = random_qtot(d, 11)
    ref = o.sweep(qtot, t_xs)
    snap = snap_ctx(d)
    got = snap.mini_kba_sweep(dev(qtot), dev(t_xs)).cpu().numpy()
    assert rel_err(got[..., 0], ref[..., 0]) < TOL
    assert moment_err(got, ref) < TOL


@pytest.mark.parametrize("env", [dict(SNAP_B200_OCTANTS_PER_LAUNCH=2),
                                 dict(SNAP_B200_OCTANTS_PER_LAUNCH=1),
                                 dict(SNAP_B200_GRID=1),
                                 dict(SNAP_B200_GRID=3, SNAP_B200_OCTANTS_PER_LAUNCH=4)],
                         ids=["P2", "P1", "grid1", "grid3_P4"])
def test_sweep_launch_plans(env):
    """Fewer octants per launch (slot accumulation) and tiny persistent grids
    (a single CTA walks every item in queue order) give the same flux."""
    d = P.Deck(16, 16, 8, nang=12, ng=2, nmom=2)
    prob = P.make_problem(d)
    o = Oracle(d)
    t_xs, _ = o.expand(prob)
    qtot = random_qtot(d, 3)
    ref = o.sweep(qtot, t_xs)
    got = snap_ctx(d, **env).mini_kba_sweep(dev(qtot), dev(t_xs)).cpu().numpy()
    assert moment_err(got, ref) < TOL


def thick_point_source(d):
    prob = P.make_problem(d)
    prob["sigt"] = prob["sigt"] * 40.0
    prob["slgg"] = prob["slgg"] * 40.0
    prob["qi"][:] = 0.0
    c = (d.nz // 2 * d.ny + d.ny // 2) * d.nx + d.nx // 2
    prob["qi"][:, c] = 100.0
    return prob


@pytest.mark.parametrize("nang,nmom", [(10, 1), (10, 2), (36, 4), (64, 2)],
                         ids=["A10_M1", "A10_M4", "A36_M16", "A64_M4"])
def test_sweep_fixup_heavy(nang, nmom):
    """Optically thick cells around a point source: most cells take the
    negative-flux fixup path (36 angles: the 3-CTA shape whose fixup works on
    faces and fluxes parked in shared memory; 64: the widest tile)."""
    d = P.Deck(16, 16, 8, nang=nang, ng=2, nmom=nmom)
    prob = thick_point_source(d)
    o = Oracle(d)
    t_xs, s_xs = o.expand(prob)
    q2 = o.outer_source(prob, np.zeros((d.ng, d.cells, d.cmom)))
    qtot = o.inner_source(s_xs, q2, np.zeros((d.ng, d.cells, d.cmom)))
    ref = o.sweep(qtot, t_xs)
    nofix = Oracle(P.Deck(**{**d.__dict__, "fixup": False})).sweep(qtot, t_xs)
    assert rel_err(nofix[..., 0], ref[..., 0]) > 1e-3      # the fixup mattered
    got = snap_ctx(d).mini_kba_sweep(dev(qtot), dev(t_xs)).cpu().numpy()
    assert rel_err(got[..., 0], ref[..., 0]) < TOL
    assert moment_err(got, ref) < TOL


def test_convergence_tests():
    d = P.Deck(8, 8, 8, nang=2, ng=2, nmom=2)
    snap = snap_ctx(d)
    rng = np.random.default_rng(5)
    prev = rng.uniform(0.5, 1.0, size=(d.ng, d.cells, d.cmom))
    flux = prev * (1 + 0.5e-4)
    assert snap.test_inner_convergence(dev(flux), dev(prev))
    flux[1, 17, 0] = prev[1, 17, 0] * 1.01
    assert not snap.test_inner_convergence(dev(flux), dev(prev))
    assert snap.test_outer_convergence(dev(flux), dev(prev), True) is False
    flux[1, 17, 0] = prev[1, 17, 0] * (1 + 0.9e-2)   # within 100 eps
    assert snap.test_outer_convergence(dev(flux), dev(prev), True)
    assert snap.test_outer_convergence(dev(flux), dev(prev), False) is False
    prev[0, 3, 0] = 0.0                                # |prev| < 1e-12: tests |flux|
    flux[0, 3, 0] = 5e-5
    assert snap.test_inner_convergence(dev(flux), dev(prev)) is False  # flux[1,17] still off
    flux[1, 17, 0] = prev[1, 17, 0]
    assert snap.test_inner_convergence(dev(flux), dev(prev))


# ---------------------------------------------------------------- full solves
def test_solve_deck1_matches_reference(golden):
    """16^3, A=10, G=4: every cell and group against the reference's own task
    bodies, and the same iteration record."""
    g = golden["deck1"]
    d = P.deck(1)
    snap = snap_ctx(d)
    flux, rec = snap.transport_solve(snap.device_problem(P.make_problem(d)))
    assert rel_err(flux[..., 0].cpu().numpy(), g["flux0"]) < TOL
    assert rec["inner_total"] == int(g["inner_total"])
    assert rec["outer_total"] == int(g["outer_total"])
    assert rec["converged"] == bool(g["converged"])
    assert rec["inners_per_outer"] == list(g["inners_per_outer"])


def test_solve_deck2p_matches_reference(golden):
    """64^3, A=36, G=32, nmom=1 (deck 2 at one moment): the reference's
    converged scalar flux at 4096 seeded samples, per-group sums and maxima,
    and the iteration record."""
    g = golden["deck2p"]
    d = P.deck(2, nmom=1)
    snap = snap_ctx(d)
    flux, rec = snap.transport_solve(snap.device_problem(P.make_problem(d)))
    phi = flux[..., 0].cpu().numpy()
    assert rel_err(phi[g["sample_g"], g["sample_c"]], g["sample_flux0"]) < TOL
    assert rel_err(phi.sum(axis=1), g["group_sum"]) < TOL
    assert rel_err(phi.max(axis=1), g["group_max"]) < TOL
    assert rec["inner_total"] == int(g["inner_total"])
    assert rec["outer_total"] == int(g["outer_total"])
    assert rec["inners_per_outer"] == list(g["inners_per_outer"])


def test_solve_multimoment_matches_oracle():
    d = P.Deck(16, 16, 16, nang=12, ng=4, nmom=4, epsi=1e-6, iitm=3, oitm=4)
    prob = P.make_problem(d)
    ref, rref = Oracle(d).solve(prob)
    snap = snap_ctx(d)
    flux, rec = snap.transport_solve(snap.device_problem(prob))
    got = flux.cpu().numpy()
    assert rel_err(got[..., 0], ref[..., 0]) < TOL
    assert moment_err(got, ref) < TOL
    assert rec["inners_per_outer"] == rref["inners_per_outer"]


@pytest.mark.parametrize("env", [dict(SNAP_B200_GROUP_CHAIN="2"), dict(SNAP_B200_GROUP_CHAIN="3"),
                                 dict(SNAP_B200_GROUP_CHAIN="6"),
                                 dict(SNAP_B200_GROUP_CHAIN="3", SNAP_B200_GRID="1"),
                                 dict(SNAP_B200_GROUP_CHAIN="2", SNAP_B200_OCTANTS_PER_LAUNCH="2")],
                         ids=["chain2", "chain3", "chain6", "chain3_grid1", "chain2_P2"])
def test_solve_group_chains_match_oracle(env, monkeypatch):
    """The inner iteration's sweep with work items of several groups (their z
    columns walked as one chained column; the z face restarts at the vacuum
    boundary of each group): the same solve as the oracle, also with one CTA
    walking every item and with fewer octants per launch."""
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    d = P.Deck(16, 16, 8, nang=12, ng=6, nmom=2, epsi=1e-6, iitm=3, oitm=4)
    prob = P.make_problem(d)
    ref, rref = Oracle(d).solve(prob)
    snap = snap_ctx(d)
    flux, rec = snap.transport_solve(snap.device_problem(prob))
    got = flux.cpu().numpy()
    assert rel_err(got[..., 0], ref[..., 0]) < TOL
    assert moment_err(got, ref) < TOL
    assert rec["inners_per_outer"] == rref["inners_per_outer"]


def test_fp32_solve_group_chains(monkeypatch):
    """FP32 sweep with chained groups: within the FP32 tolerance of the FP64
    oracle, and equal to the unchained FP32 solve up to the atomic order of
    the octant sums."""
    d = P.Deck(16, 16, 8, nang=12, ng=6, nmom=2, epsi=1e-6, iitm=3, oitm=4)
    prob = P.make_problem(d)
    ref, _ = Oracle(d).solve(prob)
    out = []
    for gc in ("1", "3"):
        monkeypatch.setenv("SNAP_B200_GROUP_CHAIN", gc)
        snap = snap_ctx32(d)
        flux, _ = snap.transport_solve(snap.device_problem(prob))
        out.append(flux.cpu().numpy())
    assert rel_err(out[1][..., 0], ref[..., 0]) < FP32_TOL
    assert rel_err(out[1][..., 0], out[0][..., 0]) < 1e-5


def check_oracle_fixture(g, flux, rec, tol):
    """A converged solve against an oracle fixture (tests/golden/*_oracle.npz):
    the scalar flux at the seeded samples, per-group sums and maxima (relative,
    `tol`), every moment at the moment samples (`tol` of that moment's largest
    magnitude), and the iteration record."""
    f = flux.cpu().numpy()
    phi = f[..., 0]
    assert rel_err(phi[g["sample_g"], g["sample_c"]], g["sample_flux0"]) < tol
    assert rel_err(f.sum(axis=1)[:, 0], g["group_sum"][:, 0]) < tol
    assert rel_err(np.abs(f).max(axis=1)[:, 0], g["group_max"][:, 0]) < tol
    scale = g["group_max"].max(axis=0)
    mom = np.abs(f[g["moment_g"], g["moment_c"], :] - g["moment_flux"]).max(axis=0) / scale
    assert float(mom.max()) < tol
    assert rec["converged"] == bool(g["converged"])


def test_solve_deck2_matches_oracle(golden_dir):
    """Deck 2 exactly as benchmarked (64^3, A=36, G=32, nmom=4, 16 moments):
    the oracle's converged solve at seeded samples, per-group sums and maxima,
    all moments at seeded cells, the identical iteration record; and the
    problem's three mirror symmetries to 1e-12."""
    g = np.load(golden_dir / "deck2_oracle.npz")
    d = P.deck(2)
    snap = snap_ctx(d)
    flux, rec = snap.transport_solve(snap.device_problem(P.make_problem(d)))
    check_oracle_fixture(g, flux, rec, TOL)
    assert rec["inner_total"] == int(g["inner_total"])
    assert rec["outer_total"] == int(g["outer_total"])
    assert rec["inners_per_outer"] == list(g["inners_per_outer"])
    phi = flux[..., 0].reshape(d.ng, d.nz, d.ny, d.nx)
    assert torch.isfinite(flux).all()
    assert (phi > 0).all()
    for dim in (1, 2, 3):
        assert rel_err(phi.flip(dim).cpu().numpy(), phi.cpu().numpy()) < TOL


def test_solve_deck4_matches_oracle(golden_dir):
    """The adjoint deck's forward solve (32^3, A=24, G=16, nmom=2, per-cell
    +-10 % sigma_t) against the oracle fixture at 1e-12, iteration record
    identical."""
    g = np.load(golden_dir / "deck4_oracle.npz")
    d = P.deck(4)
    snap = snap_ctx(d)
    flux, rec = snap.transport_solve(snap.device_problem(P.make_problem(d)))
    check_oracle_fixture(g, flux, rec, TOL)
    assert rec["inners_per_outer"] == list(g["inners_per_outer"])


# ---------------------------------------------------------------- FP32 form
FP32_TOL = 1e-5    # scalar-flux error of the FP32 form against the FP64 oracle


def snap_ctx32(deck):
    from snap_b200.solver import Snap
    return Snap(deck, precision="fp32")


def test_fp32_solve_deck2_error_against_oracle(golden_dir):
    """The precision form's whole solve on deck 2 (FP32 sweep, BF16
    tensor-core outer source while far from convergence, FP64 sources and
    tests) against the FP64 oracle fixture: scalar flux within 1e-5 relative
    at the samples and in the per-group sums and maxima, every moment within
    1e-5 of its largest magnitude."""
    g = np.load(golden_dir / "deck2_oracle.npz")
    d = P.deck(2)
    snap = snap_ctx32(d)
    flux, rec = snap.transport_solve(snap.device_problem(P.make_problem(d)))
    check_oracle_fixture(g, flux, rec, FP32_TOL)


@pytest.mark.parametrize("d", [P.deck(1), P.Deck(16, 16, 16, nang=36, ng=3, nmom=4)],
                         ids=["deck1", "A36_cmom16"])
def test_fp32_sweep_error(d):
    prob = P.make_problem(d)
    o = Oracle(d)
    t_xs, _ = o.expand(prob)
    qtot = random_qtot(d, 11)
    ref = o.sweep(qtot, t_xs)
    snap = snap_ctx32(d)
    got = snap.mini_kba_sweep(dev(qtot).float(), dev(t_xs).float()).double().cpu().numpy()
    assert rel_err(got[..., 0], ref[..., 0]) < FP32_TOL
    assert moment_err(got, ref) < FP32_TOL


@pytest.mark.parametrize("nang", [10, 36])
def test_fp32_sweep_fixup_heavy(nang):
    d = P.Deck(16, 16, 8, nang=nang, ng=2, nmom=2)
    prob = thick_point_source(d)
    o = Oracle(d)
    t_xs, s_xs = o.expand(prob)
    q2 = o.outer_source(prob, np.zeros((d.ng, d.cells, d.cmom)))
    qtot = o.inner_source(s_xs, q2, np.zeros((d.ng, d.cells, d.cmom)))
    ref = o.sweep(qtot, t_xs)
    got = snap_ctx32(d).mini_kba_sweep(dev(qtot).float(), dev(t_xs).float()).double().cpu().numpy()
    # thick cells: values span many decades; compare where the flux is not tiny
    phi, rphi = got[..., 0], ref[..., 0]
    big = np.abs(rphi) > 1e-6 * np.abs(rphi).max()
    assert rel_err(phi[big], rphi[big]) < 1e-4


@pytest.mark.parametrize("d", [P.deck(1), P.Deck(16, 16, 16, nang=12, ng=4, nmom=4, epsi=1e-6,
                                                 iitm=3, oitm=4)], ids=["deck1", "cmom16"])
def test_fp32_solve_error(d):
    """The mixed-precision solve (FP32 sweep, FP64 sources, octant sums and
    convergence) stays within 1e-5 of the FP64 oracle in scalar flux."""
    prob = P.make_problem(d)
    ref, _ = Oracle(d).solve(prob)
    snap = snap_ctx32(d)
    flux, rec = snap.transport_solve(snap.device_problem(prob))
    assert rel_err(flux[..., 0].cpu().numpy(), ref[..., 0]) < FP32_TOL


# ------------------------------------- FP32 form, TF32 tensor-core contractions
@pytest.fixture
def tf32_sweep(monkeypatch):
    """Contexts created inside the test sweep with the split-TF32 kernel
    (group pairs on the m16n8k8 TF32 MMA)."""
    monkeypatch.setenv("SNAP_B200_FP32_TC", "1")


@pytest.mark.parametrize("d", [P.deck(1), P.Deck(16, 16, 16, nang=36, ng=3, nmom=4),
                               P.Deck(16, 16, 8, nang=20, ng=4, nmom=3)],
                         ids=["deck1", "A36_cmom16_odd_groups", "cmom9"])
def test_fp32_tf32_sweep_error(d, tf32_sweep):
    prob = P.make_problem(d)
    o = Oracle(d)
    t_xs, _ = o.expand(prob)
    qtot = random_qtot(d, 12)
    ref = o.sweep(qtot, t_xs)
    got = snap_ctx32(d).mini_kba_sweep(dev(qtot).float(), dev(t_xs).float()).double().cpu().numpy()
    assert rel_err(got[..., 0], ref[..., 0]) < FP32_TOL
    assert moment_err(got, ref) < FP32_TOL


def test_fp32_tf32_solve_error(tf32_sweep):
    d = P.Deck(16, 16, 16, nang=12, ng=5, nmom=4, epsi=1e-6, iitm=3, oitm=4)
    prob = P.make_problem(d)
    ref, _ = Oracle(d).solve(prob)
    snap = snap_ctx32(d)
    flux, rec = snap.transport_solve(snap.device_problem(prob))
    assert rel_err(flux[..., 0].cpu().numpy(), ref[..., 0]) < FP32_TOL


# --------------------------- outer source on the tcgen05 tensor cores (BF16)
@pytest.mark.parametrize("d", [P.Deck(16, 16, 16, nang=4, ng=20, nmom=4),
                               P.Deck(16, 16, 8, nang=4, ng=4, nmom=1),
                               P.Deck(16, 16, 8, nang=4, ng=33, nmom=3),
                               P.Deck(16, 16, 8, nang=4, ng=32, nmom=4),
                               P.Deck(16, 8, 8, nang=4, ng=64, nmom=3),
                               P.Deck(7, 5, 3, nang=4, ng=32, nmom=4),
                               P.Deck(7, 5, 3, nang=4, ng=20, nmom=3)],
                         ids=["G20_cmom16", "G4_cmom1", "G33_cmom9", "G32_cmom16", "G64_cmom9",
                              "ragged_cells", "unaligned_runs"])
def test_outer_source_tc_matches_fp64(d):
    """The split-BF16 tensor-core outer source (tcgen05.mma, accumulators in
    tensor memory) against the FP64 one (itself at 1e-12 of the oracle): the
    scattering term within 1e-4 of its largest magnitude per moment, the
    fixed source exact, on batches that mix the two materials, group counts
    that are not multiples of 16, a last batch that is mostly empty, and
    per-group runs that are not 16-byte aligned (no bulk-copy stages)."""
    snap = snap_ctx(d)
    dp = snap.device_problem(P.make_problem(d))
    flux = dev(random_qtot(d, 5))
    ref = snap.calc_outer_source(dp["qi"], dp["slgg"], dp["mat"], flux)
    got = snap.calc_outer_source_tc(dp["qi"], dp["slgg"], dp["mat"], flux)
    scat_ref = ref.clone()
    scat_ref[..., 0] -= dp["qi"]
    scat_got = got.clone()
    scat_got[..., 0] -= dp["qi"]
    err = moment_err(scat_got.cpu().numpy(), scat_ref.cpu().numpy())
    assert err < 1e-4, err
    assert err > 0.0   # it is the low-precision path


def test_fp32_solve_refines_lowp_source():
    """An FP32 solve takes its early outer sources from the tensor cores and
    still lands within 1e-5 of the FP64 oracle: the last outer iterations use
    the FP64 source."""
    d = P.Deck(16, 16, 16, nang=12, ng=6, nmom=2, epsi=1e-6, iitm=3, oitm=30)
    prob = P.make_problem(d)
    ref, _ = Oracle(d).solve(prob)
    from snap_b200.solver import Snap
    snap = Snap(d, precision="fp32")
    flux, rec = snap.transport_solve(snap.device_problem(prob))
    assert rec["converged"]
    assert rec["outers_lowp"] >= 1
    assert rec["outers_lowp"] < rec["outer_total"]
    assert rel_err(flux[..., 0].cpu().numpy(), ref[..., 0]) < FP32_TOL


def test_fp64_finish_of_fp32_solve():
    """One FP64 outer iteration started from the converged FP32-form flux
    removes most of the FP32 rounding error (the refinement used for large
    decks)."""
    from snap_b200.solver import Snap, fp64_finish
    d = P.Deck(16, 16, 16, nang=12, ng=6, nmom=2, epsi=1e-6, iitm=5, oitm=30)
    prob = P.make_problem(d)
    snap64 = Snap(d)
    dp = snap64.device_problem(prob)
    ref, _ = snap64.transport_solve(dp)
    snap64.close()
    snap32 = Snap(d, precision="fp32")
    f32, _ = snap32.transport_solve(dp)
    snap32.close()
    fin, stats = fp64_finish(d, dp, f32)
    e32 = rel_err(f32[..., 0].cpu().numpy(), ref[..., 0].cpu().numpy())
    efin = rel_err(fin[..., 0].cpu().numpy(), ref[..., 0].cpu().numpy())
    assert stats["inner_iterations"] >= 1
    assert efin < max(2e-6, 0.5 * e32), (e32, efin)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_inner_iteration_atomic_octants_match_slots(prec, monkeypatch):
    """Inner iterations add every octant straight into the flux; the
    per-octant slots with a separate reduction (SNAP_B200_OCTANT_SLOTS=1) give
    the same flux up to summation order, and the same inner test result."""
    from snap_b200.solver import Snap
    d = P.Deck(16, 16, 8, nang=12, ng=3, nmom=3)
    prob = P.make_problem(d)
    out = []
    for slots in ("0", "1"):
        monkeypatch.setenv("SNAP_B200_OCTANT_SLOTS", slots)
        snap = Snap(d, precision=prec)
        dp = snap.device_problem(prob)
        t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"]).to(snap.sweep_dtype).contiguous()
        s_xs = snap.expand_scattering_cross_section(dp["slgg"], dp["mat"])
        flux = dev(random_qtot(d, 3))
        q2 = snap.calc_outer_source(dp["qi"], dp["slgg"], dp["mat"], flux)
        qtot = torch.empty(d.ng, d.cells, d.cmom, dtype=snap.sweep_dtype, device="cuda")
        convs = [snap.inner_iteration(s_xs, q2, t_xs, flux, qtot) for _ in range(2)]
        out.append((flux.cpu().numpy(), convs))
        snap.close()
    tol = TOL if prec == "fp64" else 1e-6
    assert moment_err(out[0][0], out[1][0]) < tol
    assert out[0][1] == out[1][1]
