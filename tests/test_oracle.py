"""CPU tests: the oracle pinned against the reference's own outputs, the input
generator against the reference's init tasks, and self-consistency checks
for the moment generalisation (nmom > 1) the reference cannot run."""
import numpy as np
import pytest

from oracle.bindings import Oracle, RefSnap
from snap_b200 import problem as P


def rel_err(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


@pytest.fixture(scope="module")
def deck1_golden(golden_dir):
    return np.load(golden_dir / "deck1_ref.npz")


def test_generator_matches_reference_init(deck1_golden):
    """InitMaterial / InitSource (init.cc:49-191) centre layouts."""
    prob = P.make_problem(P.deck(1))
    assert np.array_equal(prob["mat"], deck1_golden["ref_mat"])
    assert np.array_equal(prob["qi"], deck1_golden["ref_qi"])


def test_quadrature_properties():
    for nang, nmom in [(10, 1), (36, 4), (48, 3), (24, 2)]:
        mu, eta, xi, w, ec = P.quadrature(nang, nmom)
        assert abs(w.sum() - 0.125) < 1e-15
        assert np.allclose(mu ** 2 + eta ** 2 + xi ** 2, 1.0, atol=1e-15)
        assert np.all(ec[:, 0, :] == 1.0)
        assert ec.shape == (8, nmom * nmom, nang)
        o = Oracle(P.Deck(8, 8, 8, nang=nang, ng=1, nmom=nmom))
        assert np.array_equal(o.mu, mu) and np.array_equal(o.eta, eta)
        assert np.array_equal(o.xi, xi) and np.array_equal(o.w, w)
        assert np.allclose(o.ec, ec, rtol=1e-14, atol=1e-300)


def test_oracle_full_solve_matches_reference_deck1(deck1_golden):
    """16^3, A=10, G=4, nmom=1: the restatement against the reference's own
    task bodies, every cell and group, 1e-12 relative."""
    d = P.deck(1)
    prob = P.make_problem(d)
    flux, rec = Oracle(d).solve(prob)
    assert rel_err(flux[:, :, 0], deck1_golden["flux0"]) < 1e-12
    assert rec["inner_total"] == int(deck1_golden["inner_total"])
    assert rec["outer_total"] == int(deck1_golden["outer_total"])
    assert rec["converged"] == bool(deck1_golden["converged"])
    assert rec["inners_per_outer"] == list(deck1_golden["inners_per_outer"])


def test_oracle_first_inner_matches_reference_deck1(deck1_golden):
    d = P.deck(1)
    prob = P.make_problem(d)
    flux, rec = Oracle(d).solve(prob, oitm=1, iitm=1)
    assert rel_err(flux[:, :, 0], deck1_golden["flux0_first_inner"]) < 1e-13


@pytest.mark.skipif(not RefSnap.available(), reason="reference build not present")
def test_oracle_matches_reference_build_fixup_heavy():
    """Optically thick cells with a point source drive the negative-flux
    fixup; oracle and reference must agree there too (fixup on and off)."""
    d = P.Deck(8, 8, 8, nang=8, ng=2, nmom=1, epsi=1e-6, iitm=2, oitm=2)
    prob = P.make_problem(d)
    prob["sigt"] = prob["sigt"] * 40.0
    prob["slgg"] = prob["slgg"] * 40.0
    prob["qi"][:] = 0.0
    prob["qi"][:, 3 * 64 + 3 * 8 + 3] = 100.0
    for fixup in (True, False):
        dd = P.Deck(**{**d.__dict__, "fixup": fixup})
        fo, _ = Oracle(dd).solve(prob)
        fr, _ = RefSnap(dd).solve(prob, variant=0, nthreads=1)
        assert rel_err(fo[:, :, 0], fr) < 1e-12
    # the fixup changed the answer, so it was exercised
    f_on, _ = Oracle(d).solve(prob)
    f_off, _ = Oracle(P.Deck(**{**d.__dict__, "fixup": False})).solve(prob)
    assert rel_err(f_on, f_off) > 1e-6


@pytest.mark.skipif(not RefSnap.available(), reason="reference build not present")
def test_reference_variants_agree():
    """The reference's scalar, SSE and AVX sweep bodies on an A % 4 == 0 deck."""
    d = P.Deck(8, 8, 8, nang=8, ng=3, nmom=1, epsi=1e-5, iitm=3, oitm=3)
    prob = P.make_problem(d)
    ref = RefSnap(d)
    outs = [ref.solve(prob, variant=v, nthreads=2)[0] for v in (0, 1, 2)]
    assert rel_err(outs[1], outs[0]) < 1e-13
    assert rel_err(outs[2], outs[0]) < 1e-13


def test_moment_generalisation_reduces_to_nmom1():
    """With zero higher-order scattering the higher moments never feed back:
    the nmom=3 scalar flux equals the nmom=1 one."""
    d1 = P.Deck(8, 8, 8, nang=6, ng=3, nmom=1, epsi=1e-6, iitm=3, oitm=3)
    d3 = P.Deck(**{**d1.__dict__, "nmom": 3})
    p1 = P.make_problem(d1)
    p3 = P.make_problem(d3)
    p3["slgg"][..., 1:] = 0.0
    f1, r1 = Oracle(d1).solve(p1)
    f3, r3 = Oracle(d3).solve(p3)
    assert rel_err(f3[:, :, 0], f1[:, :, 0]) < 1e-13
    assert r1 == r3


def test_mirror_symmetry_multimoment():
    """The centred problem is symmetric under each mirror x -> nx-1-x (and in
    y, z); the scalar flux must be too, with anisotropic scattering on.  (The
    moment set is not rotation invariant, so no axis swap is tested.)"""
    d = P.Deck(8, 8, 8, nang=6, ng=2, nmom=2, epsi=1e-6, iitm=2, oitm=2)
    f, _ = Oracle(d).solve(P.make_problem(d))
    phi = f[:, :, 0].reshape(d.ng, d.nz, d.ny, d.nx)
    assert rel_err(phi[..., ::-1], phi) < 1e-12
    assert rel_err(phi[:, :, ::-1, :], phi) < 1e-12
    assert rel_err(phi[:, ::-1, :, :], phi) < 1e-12


def test_convergence_test_semantics():
    d = P.Deck(8, 8, 8, nang=2, ng=1, nmom=1)
    o = Oracle(d)
    prev = np.ones((1, d.cells, 1))
    flux = prev.copy()
    assert o.test_convergence(flux, prev, 1e-4)
    flux[0, 5, 0] = 1.001
    assert not o.test_convergence(flux, prev, 1e-4)
    # |prev| < 1e-12 compares |flux| itself (inner.cc:308-312)
    prev[0, 5, 0] = 0.0
    flux[0, 5, 0] = 5e-5
    assert o.test_convergence(flux, prev, 1e-4)
    flux[0, 5, 0] = np.nan      # NaN compares false, counted as converged
    assert o.test_convergence(flux, prev, 1e-4)


def test_oracle_threads_do_not_change_results():
    """Groups spread over host threads: bitwise the same solve as one thread."""
    d = P.Deck(8, 8, 8, nang=6, ng=5, nmom=2, epsi=1e-6, iitm=2, oitm=2)
    prob = P.make_problem(d)
    f1, r1 = Oracle(d, threads=1).solve(prob)
    f4, r4 = Oracle(d, threads=4).solve(prob)
    assert np.array_equal(f1, f4)
    assert r1 == r4


def test_oracle_reproduces_deck4_fixture(golden_dir):
    """The committed adjoint-deck fixture (tests/golden/deck4_oracle.npz)
    is what the oracle computes (the GPU tests compare against it)."""
    import os
    g = np.load(golden_dir / "deck4_oracle.npz")
    d = P.deck(4)
    f, rec = Oracle(d, threads=os.cpu_count() or 1).solve(P.make_problem(d))
    assert np.array_equal(f[g["sample_g"], g["sample_c"], 0], g["sample_flux0"])
    assert np.array_equal(f[g["moment_g"], g["moment_c"], :], g["moment_flux"])
    assert rec["inners_per_outer"] == list(g["inners_per_outer"])


@pytest.mark.parametrize("fixup,thick", [(False, False), (True, True)], ids=["plain", "fixups"])
@pytest.mark.parametrize("nmom", [1, 2])
def test_oracle_adjoint_sweep_is_transpose(fixup, thick, nmom):
    """The CPU adjoint sweep (the check for the GPU adjoint) is the transpose
    of the oracle's forward sweep at the same state: <phi_bar, sweep(q)> =
    <adjoint(phi_bar), q> to rounding (the forward map is linear in q for
    frozen fixup flags), and its t_xs sensitivity matches central
    differences."""
    d = P.Deck(6, 5, 4, nang=6, ng=2, nmom=nmom, fixup=fixup)
    prob = P.make_problem(d)
    if thick:
        prob["sigt"] = prob["sigt"] * 40.0
    o = Oracle(d)
    t_xs, _ = o.expand(prob)
    rng = np.random.default_rng(3)
    q = rng.uniform(0.0, 1.0, size=(d.ng, d.cells, d.cmom))
    if d.cmom > 1:
        q[..., 1:] = rng.uniform(-0.3, 0.3, size=q[..., 1:].shape)
    pb = rng.uniform(-1.0, 1.0, size=(d.ng, d.cells, d.cmom))
    flux = o.sweep(q, t_xs)
    qb, sb = o.adjoint_sweep(q, t_xs, pb)
    lhs, rhs = float((pb * flux).sum()), float((qb * q).sum())
    assert abs(lhs - rhs) <= 1e-13 * max(abs(lhs), 1.0)
    # t_xs sensitivity at a few cells, central differences
    for g, c in ((0, 7), (1, 33), (0, 101)):
        h = 1e-6 * t_xs[g, c]
        tp, tm = t_xs.copy(), t_xs.copy()
        tp[g, c] += h
        tm[g, c] -= h
        fd = (float((pb * o.sweep(q, tp)).sum()) - float((pb * o.sweep(q, tm)).sum())) / (2 * h)
        assert abs(sb[g, c] - fd) <= 1e-6 * max(abs(fd), 1e-6), (g, c, sb[g, c], fd)
