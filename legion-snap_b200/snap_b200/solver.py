"""Host-side mirror of the reference's task-level interface on the solve path.

Each method of :class:`Snap` corresponds to one of the reference's logical
tasks and calls the matching C ABI entry point (include/snap_b200.h) on CUDA
tensors owned by the caller.  Names follow the reference's task classes:

=============================  ==============================================
reference task                 method
=============================  ==============================================
ExpandCrossSection             ``expand_cross_section`` (expxs.cc:25-160)
ExpandScatteringCrossSection   ``expand_scattering_cross_section``
                               (expxs.cc:163-290)
CalcOuterSource                ``calc_outer_source`` (outer.cc:26-284)
CalcInnerSource                ``calc_inner_source`` (inner.cc:27-215)
MiniKBATask (8 octants x G)    ``mini_kba_sweep`` (sweep.cc:28-129,
                               snap.cc:849-887)
TestInnerConvergence           ``test_inner_convergence`` (inner.cc:218-367)
TestOuterConvergence           ``test_outer_convergence`` (outer.cc:287-451)
Snap::transport_solve          ``transport_solve`` (snap.cc:225-568)
=============================  ==============================================

Torch is used for device memory and the current stream only.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi
from .problem import Deck, quadrature


def _ptr(t: torch.Tensor) -> int:
    assert t.is_cuda and t.is_contiguous()
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class Snap:
    """One context (quadrature tables + sweep scratch) for a deck on one GPU."""

    def __init__(self, deck: Deck, precision: str = "fp64", device: int = 0):
        self.lib = abi.load()
        self.deck = deck
        self.device = torch.device("cuda", device)
        self.precision = precision
        self.sweep_dtype = torch.float64 if precision == "fp64" else torch.float32
        mu, eta, xi, w, ec = quadrature(deck.nang, deck.nmom)
        self._host = [np.ascontiguousarray(a, dtype=np.float64) for a in (mu, eta, xi, w, ec)]
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        cfg = abi.SnapConfig(
            deck.nx, deck.ny, deck.nz, deck.nang, deck.ng, deck.nmom, deck.nmat, int(deck.fixup),
            abi.SNAP_FP64 if precision == "fp64" else abi.SNAP_FP32,
            *deck.h, *(dp(a) for a in self._host))
        handle = C.c_void_p()
        with torch.cuda.device(self.device):
            abi.check(self.lib.snap_create(C.byref(cfg), device, C.byref(handle)))
        self.handle = handle

    def close(self):
        if self.handle:
            self.lib.snap_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def scratch_bytes(self) -> int:
        return int(self.lib.snap_scratch_bytes(self.handle))

    # ---- allocation helpers -------------------------------------------------
    def _empty(self, *shape, dtype=torch.float64):
        return torch.empty(*shape, dtype=dtype, device=self.device)

    @property
    def C(self) -> int:
        return self.deck.cells

    # ---- task-level operations ----------------------------------------------
    def expand_cross_section(self, sig: torch.Tensor, mat: torch.Tensor) -> torch.Tensor:
        xs = self._empty(self.deck.ng, self.C)
        abi.check(self.lib.snap_expand_xs(self.handle, _ptr(sig), _ptr(mat), _ptr(xs), _stream()))
        return xs

    def expand_scattering_cross_section(self, slgg, mat) -> torch.Tensor:
        s_xs = self._empty(self.deck.ng, self.C, self.deck.nmom)
        abi.check(self.lib.snap_expand_scattering_xs(self.handle, _ptr(slgg), _ptr(mat),
                                                     _ptr(s_xs), _stream()))
        return s_xs

    def calc_outer_source(self, qi, slgg, mat, flux) -> torch.Tensor:
        q2 = self._empty(self.deck.ng, self.C, self.deck.cmom)
        abi.check(self.lib.snap_calc_outer_source(self.handle, _ptr(qi), _ptr(slgg), _ptr(mat),
                                                  _ptr(flux), _ptr(q2), _stream()))
        return q2

    def calc_outer_source_tc(self, qi, slgg, mat, flux) -> torch.Tensor:
        """The outer source with the group-to-group contraction on the
        tcgen05 tensor cores (split BF16 operands, FP32 accumulation in tensor
        memory)."""
        q2 = self._empty(self.deck.ng, self.C, self.deck.cmom)
        abi.check(self.lib.snap_calc_outer_source_tc(self.handle, _ptr(qi), _ptr(slgg), _ptr(mat),
                                                     _ptr(flux), _ptr(q2), _stream()))
        return q2

    def calc_inner_source(self, s_xs, q2grp, flux) -> torch.Tensor:
        qtot = self._empty(self.deck.ng, self.C, self.deck.cmom, dtype=self.sweep_dtype)
        abi.check(self.lib.snap_calc_inner_source(self.handle, _ptr(s_xs), _ptr(q2grp),
                                                  _ptr(flux), _ptr(qtot), _stream()))
        return qtot

    def mini_kba_sweep(self, qtot, t_xs) -> torch.Tensor:
        flux = self._empty(self.deck.ng, self.C, self.deck.cmom, dtype=self.sweep_dtype)
        abi.check(self.lib.snap_sweep(self.handle, _ptr(qtot), _ptr(t_xs), _ptr(flux), _stream()))
        return flux

    def _test(self, kind, flux, prev, epsi) -> bool:
        conv = C.c_int(0)
        abi.check(self.lib.snap_test_convergence(self.handle, kind, _ptr(flux), _ptr(prev),
                                                 C.c_double(epsi), C.byref(conv), _stream()))
        return bool(conv.value)

    def test_inner_convergence(self, flux, flux_pi) -> bool:
        return self._test(0, flux, flux_pi, self.deck.epsi)

    def test_outer_convergence(self, flux, flux_po, inner_converged: bool) -> bool:
        if not inner_converged:       # outer.cc:361-365
            return False
        return self._test(1, flux, flux_po, 100.0 * self.deck.epsi)

    def inner_iteration(self, s_xs, q2grp, t_xs, flux, qtot, epsi=None) -> bool:
        """One inner iteration on resident data (snap.cc:487-503); flux is
        updated in place, qtot is scratch.  Returns the inner test result."""
        conv = C.c_int(0)
        abi.check(self.lib.snap_inner_iteration(
            self.handle, _ptr(s_xs), _ptr(q2grp), _ptr(t_xs), _ptr(flux), _ptr(qtot),
            C.c_double(self.deck.epsi if epsi is None else epsi), C.byref(conv), _stream()))
        return bool(conv.value)

    def timing(self, reset: bool = False) -> dict:
        t = abi.SnapTiming()
        abi.check(self.lib.snap_get_timing(self.handle, C.byref(t), int(reset)))
        return dict(sweep_ms=t.sweep_ms, sweep_calls=t.sweep_calls,
                    kernel_launches=t.kernel_launches)

    # ---- sensitivities ------------------------------------------------------
    def record_forward(self, qtot, t_xs) -> torch.Tensor:
        """Forward sweep that also records the state the adjoint needs."""
        flux = self._empty(self.deck.ng, self.C, self.deck.cmom, dtype=self.sweep_dtype)
        abi.check(self.lib.snap_record_forward(self.handle, _ptr(qtot), _ptr(t_xs), _ptr(flux),
                                               _stream()))
        return flux

    def adjoint_sweep(self, phi_bar, t_xs, with_sigma: bool = False):
        """qtot_bar = M^T L^-T D^T phi_bar (and the t_xs sensitivity)."""
        d = self.deck
        qbar = self._empty(d.ng, self.C, d.cmom)
        sbar = self._empty(d.ng, self.C) if with_sigma else None
        abi.check(self.lib.snap_adjoint_sweep(self.handle, _ptr(phi_bar), _ptr(t_xs), _ptr(qbar),
                                              _ptr(sbar) if sbar is not None else None,
                                              _stream()))
        return qbar, sbar

    def adjoint_solve(self, dprob: dict, t_xs: torch.Tensor, flux: torch.Tensor,
                      response: torch.Tensor, epsi=None, maxit=None, with_sxs: bool = True) -> dict:
        """dJ/dt_xs, dJ/dqi and (with_sxs) dJ/ds_xs of J = sum response *
        scalar flux at the converged forward flux (discrete adjoint, fixup
        flags frozen)."""
        d = self.deck
        gs = self._empty(d.ng, self.C)
        gq = self._empty(d.ng, self.C)
        gx = self._empty(d.ng, self.C, d.nmom) if with_sxs else None
        info = abi.SnapSolveInfo()
        info.epsi = d.epsi if epsi is None else epsi
        info.iitm = 1
        info.oitm = 2000 if maxit is None else maxit
        abi.check(self.lib.snap_adjoint_solve(
            self.handle, _ptr(dprob["mat"]), _ptr(dprob["qi"]), _ptr(t_xs.contiguous()),
            _ptr(dprob["slgg"]), _ptr(flux), _ptr(response.contiguous()), _ptr(gs), _ptr(gq),
            _ptr(gx) if gx is not None else None, C.byref(info), _stream()))
        return dict(grad_sigt=gs, grad_qi=gq, grad_sxs=gx, iterations=info.inner_total,
                    converged=bool(info.converged), total_ms=info.total_ms,
                    sweep_ms=info.sweep_ms)

    def solve_with_txs(self, dprob: dict, t_xs: torch.Tensor, qi: torch.Tensor,
                       epsi=None, iitm=None, oitm=None):
        """The solve loop of snap.cc:472-540 driven from the host through the
        task-level ABI, with an arbitrary per-cell, per-group t_xs (the
        reference expands t_xs from material tables; sensitivities need it
        free).  Returns the flux moments (float64) and the iteration record."""
        d = self.deck
        epsi = d.epsi if epsi is None else epsi
        iitm = d.iitm if iitm is None else iitm
        oitm = d.oitm if oitm is None else oitm
        s_xs = self.expand_scattering_cross_section(dprob["slgg"], dprob["mat"])
        t_sw = t_xs.to(self.sweep_dtype).contiguous()
        flux = torch.zeros(d.ng, self.C, d.cmom, dtype=torch.float64, device=self.device)
        qtot = self._empty(d.ng, self.C, d.cmom, dtype=self.sweep_dtype)
        rec = dict(inner_total=0, outer_total=0, converged=False, inners_per_outer=[])
        for o in range(oitm):
            q2 = self.calc_outer_source(qi.contiguous(), dprob["slgg"], dprob["mat"], flux)
            fpo = flux.clone()
            conv, inners = False, 0
            for _ in range(iitm):
                conv = self.inner_iteration(s_xs, q2, t_sw, flux, qtot, epsi)
                inners += 1
                if conv:
                    break
            rec["inner_total"] += inners
            rec["outer_total"] += 1
            rec["inners_per_outer"].append(inners)
            if o == 0:
                continue
            if conv and self._test(1, flux, fpo, 100.0 * epsi):
                rec["converged"] = True
                break
        return flux, rec

    # ---- the solve loop ----------------------------------------------------
    def device_problem(self, prob: dict) -> dict:
        dev = self.device
        out = dict(
            mat=torch.as_tensor(prob["mat"], device=dev),
            qi=torch.as_tensor(np.ascontiguousarray(prob["qi"]), device=dev),
            sigt=torch.as_tensor(np.ascontiguousarray(prob["sigt"]), device=dev),
            slgg=torch.as_tensor(np.ascontiguousarray(prob["slgg"]), device=dev),
        )
        if "sigt_scale" in prob:
            out["sigt_scale"] = torch.as_tensor(prob["sigt_scale"], device=dev)
        return out

    def transport_solve(self, dprob: dict, flux: torch.Tensor | None = None,
                        epsi=None, iitm=None, oitm=None):
        """Runs the whole steady-state solve on the device.  Returns the flux
        moments [G, C, cmom] (float64) and the iteration record."""
        d = self.deck
        if flux is None:
            flux = self._empty(d.ng, self.C, d.cmom)
        info = abi.SnapSolveInfo()
        info.epsi = d.epsi if epsi is None else epsi
        info.iitm = d.iitm if iitm is None else iitm
        info.oitm = d.oitm if oitm is None else oitm
        scale = dprob.get("sigt_scale")
        cap = 4096
        recs = (abi.SnapIterRecord * cap)()
        info.records = C.cast(recs, C.POINTER(abi.SnapIterRecord))
        info.records_cap = cap
        args = (self.handle, _ptr(dprob["mat"]), _ptr(dprob["qi"]), _ptr(dprob["sigt"]),
                _ptr(dprob["slgg"]), _ptr(scale) if scale is not None else None)
        if d.timedep or "qim" in dprob:
            # time stepping, or a manufactured per-angle source (a steady
            # MMS deck runs one step with vdelt = 0)
            tc = abi.SnapTimeConfig()
            tc.nsteps = d.nsteps if d.timedep else 1
            tc.dt = d.dt
            if not d.timedep:
                vzero = torch.zeros(d.ng, dtype=torch.float64, device=self.device)
                tc.vdelt = _ptr(vzero)
            tc.qim = _ptr(dprob["qim"]) if "qim" in dprob else None
            tc.qim_time_scaled = 1 if "qim" in dprob else 0
            if "psi_t" in dprob:
                tc.psi_t = _ptr(dprob["psi_t"])
                tc.psi_t_initialised = 1
            abi.check(self.lib.snap_transport_solve_td(*args, C.byref(tc), _ptr(flux),
                                                       C.byref(info), _stream()))
        else:
            abi.check(self.lib.snap_transport_solve(*args, _ptr(flux), C.byref(info), _stream()))
        n_rec = min(info.outer_total, 1024)
        rec = dict(inner_total=info.inner_total, outer_total=info.outer_total,
                   converged=bool(info.converged),
                   inners_per_outer=list(info.inners_per_outer[:n_rec]),
                   total_ms=info.total_ms, sweep_ms=info.sweep_ms, outers_lowp=info.outers_lowp,
                   records=_records(info))
        return flux, rec


def _records(info) -> list:
    return [dict(kind="inner" if r.kind == 0 else "outer", time_step=r.time_step, outer=r.outer,
                 inner=r.inner, converged=bool(r.converged), us=r.us)
            for r in info.records[:info.records_len]]


def fp64_finish(deck: Deck, dprob: dict, flux: torch.Tensor, outers: int = 1, device: int = 0,
                max_inners: int | None = None):
    """FP64 refinement of a mixed-precision solution: `outers` outer
    iterations of the FP64 path (FP64 outer source, FP64 sweeps until the
    inner test passes, iitm or `max_inners`) started from `flux` (the
    converged FP32-form flux moments, float64), through the task-level C ABI
    of an FP64 context.  Each FP64 iteration contracts the FP32 rounding
    error like any other error, so one outer removes most of it and a single
    sweep a large part.  The FP32 context should be destroyed first when
    memory is tight.  Returns the refined flux (a new tensor) and the device
    time and iteration counts."""
    snap = Snap(deck, precision="fp64", device=device)
    try:
        flux = flux.clone()
        t_xs = snap.expand_cross_section(dprob["sigt"], dprob["mat"])
        if "sigt_scale" in dprob:
            t_xs *= dprob["sigt_scale"][None, :]
        s_xs = snap.expand_scattering_cross_section(dprob["slgg"], dprob["mat"])
        qtot = torch.empty_like(flux)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        inners = 0
        for _ in range(outers):
            q2 = snap.calc_outer_source(dprob["qi"], dprob["slgg"], dprob["mat"], flux)
            for _ in range(deck.iitm if max_inners is None else min(deck.iitm, max_inners)):
                inners += 1
                if snap.inner_iteration(s_xs, q2, t_xs, flux, qtot):
                    break
        e1.record()
        torch.cuda.synchronize()
        return flux, dict(ms=e0.elapsed_time(e1), outers=outers, inner_iterations=inners)
    finally:
        snap.close()
