"""Adjoint sweep and sensitivities on the GPU (FP64 unless stated).

- the adjoint sweep is the transpose of the forward sweep (dot-product
  identity, exact up to rounding, fixup flags frozen at the forward state),
  and equals an independent CPU adjoint (the oracle's) to 1e-12;
- the t_xs sensitivity of one sweep against central finite differences;
- the adjoint of the whole solve on the adjoint deck (32^3, 24 angles, 16
  groups, nmom 2, per-cell sigma_t perturbed +-10 %, detector box in the
  corner opposite the source, weights 1/g) against central finite
  differences of converged forward solves (h = 1e-6 relative) on seeded
  cell/group entries of t_xs and of the source;
- the FP32 adjoint against the FP64 adjoint; the autograd wrapper.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device"),
]

from snap_b200 import problem as P  # noqa: E402


def snap_ctx(d, precision="fp64"):
    from snap_b200.solver import Snap
    return Snap(d, precision=precision)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def rand_moments(d, seed, lo=0.0):
    rng = np.random.default_rng(seed)
    q = rng.uniform(lo, 1.0, size=(d.ng, d.cells, d.cmom))
    if d.cmom > 1:
        q[..., 1:] = rng.uniform(-0.2, 0.2, size=q[..., 1:].shape)
    return q


def thick(d):
    prob = P.make_problem(d)
    prob["sigt"] = prob["sigt"] * 40.0
    prob["slgg"] = prob["slgg"] * 40.0
    return prob


@pytest.mark.parametrize("fixup,thick_cells", [(False, False), (True, False), (True, True)])
@pytest.mark.parametrize("nmom", [1, 3])
def test_adjoint_sweep_is_transpose(fixup, thick_cells, nmom):
    d = P.Deck(16, 16, 12, nang=12, ng=2, nmom=nmom, fixup=fixup)
    prob = thick(d) if thick_cells else P.make_problem(d)
    snap = snap_ctx(d)
    t_xs = snap.expand_cross_section(dev(prob["sigt"]), dev(prob["mat"]))
    qtot = dev(rand_moments(d, 1))
    phib = dev(rand_moments(d, 2, lo=-1.0))
    flux = snap.record_forward(qtot, t_xs)
    qbar, _ = snap.adjoint_sweep(phib, t_xs)
    lhs = float((phib * flux).sum())
    rhs = float((qbar * qtot).sum())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


@pytest.mark.parametrize("fixup,thick_cells", [(False, False), (True, True)],
                         ids=["plain", "fixups"])
@pytest.mark.parametrize("nmom", [1, 3])
def test_adjoint_sweep_matches_cpu_adjoint(fixup, thick_cells, nmom):
    """The GPU adjoint sweep against an independent CPU adjoint (the oracle's
    transpose of its own forward sweep, fixup flags frozen at the forward
    state): qtot_bar within 1e-12 of each moment's largest magnitude and the
    t_xs sensitivity within 1e-11 relative to its largest magnitude."""
    from oracle.bindings import Oracle
    d = P.Deck(16, 16, 8, nang=12, ng=2, nmom=nmom, fixup=fixup)
    prob = thick(d) if thick_cells else P.make_problem(d)
    snap = snap_ctx(d)
    t_xs = snap.expand_cross_section(dev(prob["sigt"]), dev(prob["mat"]))
    q = rand_moments(d, 4)
    pb = rand_moments(d, 5, lo=-1.0)
    snap.record_forward(dev(q), t_xs)
    qbar, sbar = snap.adjoint_sweep(dev(pb), t_xs, with_sigma=True)
    o = Oracle(d)
    qref, sref = o.adjoint_sweep(q, t_xs.cpu().numpy(), pb)
    got = qbar.cpu().numpy()
    scale = np.abs(qref).reshape(-1, d.cmom).max(axis=0)
    assert float((np.abs(got - qref).reshape(-1, d.cmom).max(axis=0) / scale).max()) < 1e-12
    sg = sbar.cpu().numpy()
    assert float(np.abs(sg - sref).max() / np.abs(sref).max()) < 1e-11
    snap.close()


@pytest.mark.parametrize("fixup", [False, True])
def test_adjoint_sweep_sigma_sensitivity(fixup):
    """d<phib, sweep(qtot; t_xs)>/dt_xs against central differences."""
    d = P.Deck(16, 16, 8, nang=10, ng=2, nmom=2, fixup=fixup)
    prob = P.make_problem(d)
    snap = snap_ctx(d)
    t_xs = snap.expand_cross_section(dev(prob["sigt"]), dev(prob["mat"]))
    qtot = dev(rand_moments(d, 3))
    phib = dev(rand_moments(d, 4, lo=-1.0))
    snap.record_forward(qtot, t_xs)
    _, sbar = snap.adjoint_sweep(phib, t_xs, with_sigma=True)
    rng = np.random.default_rng(9)
    h = 1e-6
    for _ in range(12):
        g, c = int(rng.integers(d.ng)), int(rng.integers(d.cells))
        tp, tm = t_xs.clone(), t_xs.clone()
        dt = h * float(t_xs[g, c])
        tp[g, c] += dt
        tm[g, c] -= dt
        jp = float((phib * snap.mini_kba_sweep(qtot, tp)).sum())
        jm = float((phib * snap.mini_kba_sweep(qtot, tm)).sum())
        fd = (jp - jm) / (2 * dt)
        assert abs(float(sbar[g, c]) - fd) <= 1e-5 * abs(fd) + 1e-9 * float(sbar.abs().max())


def detector_response(d):
    """Group weights 1/g on the 4^3 box in the corner opposite the source."""
    r = np.zeros((d.ng, d.nz, d.ny, d.nx))
    w = 1.0 / np.arange(1, d.ng + 1)
    r[:, -4:, -4:, -4:] = w[:, None, None, None]
    return r.reshape(d.ng, d.cells)


def expanded_txs(snap, dp):
    return snap.expand_cross_section(dp["sigt"], dp["mat"]) * dp["sigt_scale"][None, :]


def fd_check(d, n_entries, tol, epsi=1e-14, adjoint_precision="fp64", min_resolved=0.5):
    """The adjoint gradient against central differences (h = 1e-6 relative)
    of converged FP64 solves on n_entries seeded (group, cell) entries, half
    of t_xs and half of the source; one entry in four anywhere in the mesh,
    the others within 8 cells of the detector corner (further away most
    sensitivities of a single cell and group are below what central
    differences resolve).  Central differences resolve a sensitivity only
    above their noise floor epsi*|J|/step (the converged solves agree with the
    exact fixed point to about epsi in J): resolved entries must agree to
    `tol` relative, every entry within 10 noise floors, and at least
    `min_resolved` of the entries must be resolved."""
    snap = snap_ctx(d)
    dp = snap.device_problem(P.make_problem(d))
    t_xs = expanded_txs(snap, dp)
    qi = dp["qi"].clone()
    r = dev(detector_response(d))
    flux, rec = snap.solve_with_txs(dp, t_xs, qi, epsi=epsi, iitm=5, oitm=2000)
    assert rec["converged"]
    if adjoint_precision == "fp64":
        g = snap.adjoint_solve(dp, t_xs, flux, r, epsi=epsi)
    else:
        # the precision form's adjoint (FP32 sweeps) at the FP64 forward solution
        snap32 = snap_ctx(d, adjoint_precision)
        g = snap32.adjoint_solve(dp, t_xs, flux, r, epsi=1e-6)
        snap32.close()
    assert g["converged"]
    J = lambda f: float((r * f[..., 0]).sum())   # noqa: E731
    J0 = J(flux)
    rng = np.random.default_rng(2024)
    h = 1e-6
    resolved = []
    for k in range(n_entries):
        gi = int(rng.integers(d.ng))
        if k % 4 == 0:   # one in four anywhere, the rest near the detector corner
            ci = int(rng.integers(d.cells))
        else:
            z, y, x = (int(v) for v in rng.integers(d.nx - 8, d.nx, size=3))
            ci = (z * d.ny + y) * d.nx + x
        which = "sigt" if k % 2 == 0 else "qi"
        base = t_xs if which == "sigt" else qi
        val = float(base[gi, ci])
        step = h * val if val != 0.0 else h
        plus, minus = base.clone(), base.clone()
        plus[gi, ci] += step
        minus[gi, ci] -= step
        args = ((plus, qi), (minus, qi)) if which == "sigt" else ((t_xs, plus), (t_xs, minus))
        fp, _ = snap.solve_with_txs(dp, *args[0], epsi=epsi, iitm=5, oitm=2000)
        fm, _ = snap.solve_with_txs(dp, *args[1], epsi=epsi, iitm=5, oitm=2000)
        fd = (J(fp) - J(fm)) / (2 * step)
        adj = float(g["grad_sigt" if which == "sigt" else "grad_qi"][gi, ci])
        noise = epsi * abs(J0) / step
        assert abs(adj - fd) <= tol * abs(fd) + 10 * noise, (which, gi, ci, adj, fd, noise)
        if abs(fd) > 100 * noise:
            resolved.append(abs(adj - fd) / abs(fd))
    assert len(resolved) >= min_resolved * n_entries, (len(resolved), n_entries)
    assert max(resolved) <= tol
    return g, max(resolved)


def test_adjoint_solve_matches_finite_differences_no_fixup():
    """Adjoint deck with the fixup off (a linear operator): 64 seeded entries
    (32 of t_xs, 32 of the source) against central differences."""
    fd_check(P.deck(4, fixup=False), 64, 1e-4)


def test_adjoint_solve_matches_finite_differences_fixup_on():
    """Same deck with the fixup on: the adjoint differentiates the solve with
    the fixup flags frozen, the derivative wherever no flag flips under the
    +-1e-6 perturbation; 64 entries."""
    fd_check(P.deck(4, fixup=True), 64, 1e-3)


def test_fp32_adjoint_matches_finite_differences():
    """The precision form's adjoint (FP32 sweeps, FP64 iteration) against the
    same central differences of FP64 solves, 64 entries, fixup on."""
    fd_check(P.deck(4, fixup=True), 64, 1e-3, adjoint_precision="fp32")


def test_fp32_adjoint_matches_fp64_adjoint():
    d = P.deck(4, fixup=False)
    prob = P.make_problem(d)
    out = {}
    for prec in ("fp64", "fp32"):
        snap = snap_ctx(d, prec)
        dp = snap.device_problem(prob)
        t_xs = expanded_txs(snap, dp)
        flux, _ = snap.solve_with_txs(dp, t_xs, dp["qi"], epsi=1e-6, iitm=5, oitm=200)
        out[prec] = snap.adjoint_solve(dp, t_xs, flux, dev(detector_response(d)), epsi=1e-6)
    for key in ("grad_sigt", "grad_qi"):
        a, b = out["fp32"][key], out["fp64"][key]
        assert float((a - b).abs().max() / b.abs().max()) < 1e-4


def test_autograd_wrapper():
    from snap_b200.autograd import SnapSolve
    d = P.Deck(16, 16, 8, nang=8, ng=3, nmom=2, fixup=False)
    snap = snap_ctx(d)
    dp = snap.device_problem(P.make_problem(d))
    t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"]).requires_grad_(True)
    qi = dp["qi"].clone().requires_grad_(True)
    w = dev(detector_response(d))
    J = (w * SnapSolve.apply(t_xs, qi, snap, dp, 1e-12)).sum()
    J.backward()
    flux, _ = snap.solve_with_txs(dp, t_xs.detach(), qi.detach(), epsi=1e-12)
    direct = snap.adjoint_solve(dp, t_xs.detach(), flux, w, epsi=1e-12)
    assert torch.allclose(t_xs.grad, direct["grad_sigt"], rtol=1e-9, atol=1e-15)
    assert torch.allclose(qi.grad, direct["grad_qi"], rtol=1e-9, atol=1e-15)
    # one directional finite difference through the wrapper
    v = torch.randn(qi.shape, dtype=torch.float64, device="cuda",
                    generator=torch.Generator("cuda").manual_seed(3)) * 1e-6
    with torch.no_grad():
        jp = (w * SnapSolve.apply(t_xs.detach(), qi.detach() + v, snap, dp, 1e-12)).sum()
        jm = (w * SnapSolve.apply(t_xs.detach(), qi.detach() - v, snap, dp, 1e-12)).sum()
    fd = float(jp - jm) / 2
    assert abs(float((qi.grad * v).sum()) - fd) <= 1e-5 * abs(fd)


def test_adjoint_group_batches_match_whole_state():
    """The adjoint solve with the forward state held for 3 groups at a time
    (re-recorded from the converged flux moments for every batch of every
    adjoint iteration, as large decks need) gives the same gradients as with
    the state of all 16 groups recorded once."""
    import os
    d = P.deck(4, fixup=True)
    out = {}
    for key, groups in (("whole", None), ("batched", "3")):
        old = os.environ.get("SNAP_B200_ADJOINT_GROUPS")
        if groups:
            os.environ["SNAP_B200_ADJOINT_GROUPS"] = groups
        try:
            snap = snap_ctx(d)
            dp = snap.device_problem(P.make_problem(d))
            t_xs = expanded_txs(snap, dp)
            flux, _ = snap.solve_with_txs(dp, t_xs, dp["qi"], epsi=1e-8, iitm=5, oitm=200)
            out[key] = snap.adjoint_solve(dp, t_xs, flux, dev(detector_response(d)), epsi=1e-8)
            snap.close()
        finally:
            if groups:
                if old is None:
                    os.environ.pop("SNAP_B200_ADJOINT_GROUPS")
                else:
                    os.environ["SNAP_B200_ADJOINT_GROUPS"] = old
    assert out["whole"]["iterations"] == out["batched"]["iterations"]
    for key in ("grad_sigt", "grad_qi", "grad_sxs"):
        a, b = out["batched"][key], out["whole"][key]
        assert float((a - b).abs().max() / b.abs().max()) < 1e-13, key
