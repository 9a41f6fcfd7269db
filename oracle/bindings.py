"""ctypes bindings for the CPU oracles (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product path never does.

- ``Oracle``: our C restatement (oracle/snap_oracle.c -> liboracle.so).
- ``RefSnap``: the reference's own CPU task bodies compiled through the shim
  (oracle/refshim -> oracle/_ref/libsnapref.so), nmom = 1 only.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


class _Geom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nang", C.c_int),
                ("ng", C.c_int), ("nmom", C.c_int), ("cmom", C.c_int), ("nmat", C.c_int),
                ("fixup", C.c_int), ("hi", C.c_double), ("hj", C.c_double),
                ("hk", C.c_double), ("mu", _dp), ("eta", _dp), ("xi", _dp), ("w", _dp),
                ("ec", _dp)]


class _Info(C.Structure):
    _fields_ = [("epsi", C.c_double), ("iitm", C.c_int), ("oitm", C.c_int),
                ("inner_total", C.c_int), ("outer_total", C.c_int), ("converged", C.c_int),
                ("inners_per_outer", C.c_int * 1024)]


def build():
    """Compiles both oracles (make in oracle/); the reference build is skipped
    when the reference sources are absent."""
    import subprocess
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


class Oracle:
    """Our FP64 restatement of the reference's CPU task bodies."""

    def __init__(self, deck, prob=None, threads: int = 1):
        lib_path = HERE / "liboracle.so"
        if not lib_path.exists():
            build()
        self.lib = C.CDLL(str(lib_path))
        # groups are independent sweeps: spread them over host threads (the
        # result does not depend on the thread count)
        self.lib.oracle_set_threads(int(threads))
        self.deck = deck
        d = deck
        self.mu = np.zeros(d.nang)
        self.eta = np.zeros(d.nang)
        self.xi = np.zeros(d.nang)
        self.w = np.zeros(d.nang)
        self.ec = np.zeros((8, d.cmom, d.nang))
        self.lib.oracle_quadrature(d.nang, d.nmom, _d(self.mu), _d(self.eta), _d(self.xi),
                                   _d(self.w), _d(self.ec))
        self.geom = _Geom(d.nx, d.ny, d.nz, d.nang, d.ng, d.nmom, d.cmom, d.nmat, int(d.fixup),
                          *d.h, _d(self.mu), _d(self.eta), _d(self.xi), _d(self.w), _d(self.ec))
        self.prob = prob

    @property
    def C(self):
        return self.deck.cells

    def expand(self, prob):
        d = self.deck
        t_xs = np.zeros((d.ng, self.C))
        s_xs = np.zeros((d.ng, self.C, d.nmom))
        self.lib.oracle_expand_xs(C.byref(self.geom), _d(np.ascontiguousarray(prob["sigt"])),
                                  _i(prob["mat"]), _d(t_xs))
        if "sigt_scale" in prob:
            t_xs *= prob["sigt_scale"][None, :]
        self.lib.oracle_expand_scattering(C.byref(self.geom), _d(np.ascontiguousarray(prob["slgg"])),
                                          _i(prob["mat"]), _d(s_xs))
        return t_xs, s_xs

    def outer_source(self, prob, flux):
        d = self.deck
        q2 = np.zeros((d.ng, self.C, d.cmom))
        self.lib.oracle_outer_source(C.byref(self.geom), _d(prob["qi"]),
                                     _d(np.ascontiguousarray(prob["slgg"])), _i(prob["mat"]),
                                     _d(flux), _d(q2))
        return q2

    def inner_source(self, s_xs, q2grp, flux):
        d = self.deck
        qtot = np.zeros((d.ng, self.C, d.cmom))
        self.lib.oracle_inner_source(C.byref(self.geom), _d(s_xs), _d(q2grp), _d(flux), _d(qtot))
        return qtot

    def sweep(self, qtot, t_xs):
        d = self.deck
        flux = np.zeros((d.ng, self.C, d.cmom))
        self.lib.oracle_sweep(C.byref(self.geom), _d(qtot), _d(t_xs), _d(flux))
        return flux

    def adjoint_sweep(self, qtot, t_xs, phi_bar):
        """The transpose of sweep() at the forward state of qtot (fixup flags
        frozen): (qtot_bar [G][C][cmom], sigt_bar [G][C])."""
        d = self.deck
        qb = np.zeros((d.ng, self.C, d.cmom))
        sb = np.zeros((d.ng, self.C))
        self.lib.oracle_adjoint_sweep(C.byref(self.geom), _d(qtot), _d(t_xs), _d(phi_bar), _d(qb),
                                      _d(sb))
        return qb, sb

    def test_convergence(self, flux, prev, epsi):
        self.lib.oracle_test_convergence.restype = C.c_int
        return bool(self.lib.oracle_test_convergence(C.byref(self.geom), _d(flux), _d(prev),
                                                     C.c_double(epsi)))

    def solve(self, prob, epsi=None, iitm=None, oitm=None):
        d = self.deck
        t_xs, s_xs = self.expand(prob)
        flux = np.zeros((d.ng, self.C, d.cmom))
        info = _Info()
        info.epsi = d.epsi if epsi is None else epsi
        info.iitm = d.iitm if iitm is None else iitm
        info.oitm = d.oitm if oitm is None else oitm
        self.lib.oracle_transport_solve(C.byref(self.geom), _d(prob["qi"]),
                                        _d(np.ascontiguousarray(prob["slgg"])), _i(prob["mat"]),
                                        _d(t_xs), _d(s_xs), _d(flux), C.byref(info))
        rec = dict(inner_total=info.inner_total, outer_total=info.outer_total,
                   converged=bool(info.converged),
                   inners_per_outer=list(info.inners_per_outer[:info.outer_total]))
        return flux, rec


class RefSnap:
    """The reference's CPU task bodies (sweep.cc, outer.cc, inner.cc,
    expxs.cc, init.cc) run by oracle/refshim/ref_driver.cc."""

    PATH = HERE / "_ref" / "libsnapref.so"

    @classmethod
    def available(cls) -> bool:
        return cls.PATH.exists()

    def __init__(self, deck):
        if deck.nmom != 1:
            raise ValueError("the reference CPU path supports nmom = 1 only")
        self.lib = C.CDLL(str(self.PATH))
        self.lib.snapref_solve.restype = C.c_double
        self.deck = deck
        if deck.mat_opt is None and not deck.timedep:
            rc = self.lib.snapref_configure(deck.nx, deck.ny, deck.nz, deck.nang, deck.ng,
                                            deck.nmom, 1, C.c_double(deck.epsi), deck.iitm,
                                            deck.oitm, int(deck.fixup))
        else:
            # a reference deck: its layouts, lengths and time stepping
            mat_opt = 1 if deck.mat_opt is None else deck.mat_opt
            src_opt = 1 if deck.src_opt is None else deck.src_opt
            # the deck's spatial chunks (npey, npez, ichunk): the reference's
            # sweep runs one task per chunk, faces passed between them
            npey, npez, ichunk = deck.chunks
            rc = self.lib.snapref_configure_deck(
                deck.nx, deck.ny, deck.nz, C.c_double(deck.lx), C.c_double(deck.ly),
                C.c_double(deck.lz), deck.nang, deck.ng, deck.nmom, C.c_double(deck.epsi),
                deck.iitm, deck.oitm, int(deck.fixup), int(deck.timedep), C.c_double(deck.tf),
                deck.nsteps, mat_opt, src_opt, ichunk, npey, npez)
        if rc != 0:
            raise RuntimeError(f"reference configuration failed: {rc}")

    def quadrature(self):
        n = self.deck.nang
        mu, eta, xi, w = (np.zeros(n) for _ in range(4))
        self.lib.snapref_quadrature(_d(mu), _d(eta), _d(xi), _d(w))
        return mu, eta, xi, w

    def init_layout(self):
        d = self.deck
        mat = np.zeros(d.cells, dtype=np.int32)
        qi = np.zeros((d.ng, d.cells))
        self.lib.snapref_init_layout(_i(mat), _d(qi))
        return mat, qi

    @staticmethod
    def default_variant(nang: int) -> int:
        """AVX body when A % 4 == 0 (sweep.cc:1064), else SSE when A is even
        (sweep.cc:646), else the scalar body."""
        return 2 if nang % 4 == 0 else (1 if nang % 2 == 0 else 0)

    def time_inner(self, prob, steps: int, variant=None, nthreads=None):
        """Seconds of `steps` inner iterations (inner source, sweep, inner
        test; group-parallel on nthreads host threads) after one outer source:
        the GPU benchmark's step, run by the reference's task bodies."""
        d = self.deck
        if variant is None:
            variant = self.default_variant(d.nang)
        if nthreads is None:
            nthreads = os.cpu_count() or 1
        self.lib.snapref_time_inner.restype = C.c_double
        sweep_s = C.c_double(0.0)
        secs = self.lib.snapref_time_inner(_i(prob["mat"]), _d(prob["qi"]),
                                           _d(np.ascontiguousarray(prob["sigt"])),
                                           _d(np.ascontiguousarray(prob["slgg"])),
                                           int(prob.get("nmat", 2)), variant, nthreads, steps,
                                           C.byref(sweep_s))
        if secs < 0:
            raise RuntimeError(f"snapref_time_inner failed: {secs}")
        return dict(seconds=secs, sweep_seconds=sweep_s.value, variant=variant,
                    nthreads=nthreads, steps=steps)

    def solve(self, prob, variant=None, nthreads=None, max_inners=0):
        d = self.deck
        if variant is None:
            variant = self.default_variant(d.nang)
        if nthreads is None:
            nthreads = os.cpu_count() or 1
        flux = np.zeros((d.ng, d.cells))
        mms = np.zeros(3)                       # MMS compare: max, min, sum of |flux/ref - 1|
        ref_flux = np.zeros((d.ng, d.cells))    # MMS reference flux (scaled as compared)
        steps = d.nsteps if d.timedep else 1
        info = np.zeros(3 + d.oitm * steps, dtype=np.int32)
        sweep_s = C.c_double(0.0)
        secs = self.lib.snapref_solve(_i(prob["mat"]), _d(prob["qi"]),
                                      _d(np.ascontiguousarray(prob["sigt"])),
                                      _d(np.ascontiguousarray(prob["slgg"])),
                                      int(prob.get("nmat", 2)), variant, nthreads,
                                      max_inners, _d(flux), info.ctypes.data_as(_ip),
                                      C.byref(sweep_s), _d(mms), _d(ref_flux))
        if secs < 0:
            raise RuntimeError(f"snapref_solve failed: {secs}")
        rec = dict(inner_total=int(info[0]), outer_total=int(info[1]), converged=bool(info[2]),
                   inners_per_outer=[int(x) for x in info[3:3 + info[1]]],
                   seconds=secs, sweep_seconds=sweep_s.value, variant=variant,
                   nthreads=nthreads)
        if d.src_opt == 3:
            rec["mms"] = dict(max=float(mms[0]), min=float(mms[1]), sum=float(mms[2]),
                              avg=float(mms[2]) / (d.cells * int(np.prod(d.chunks)) * d.ng))
            rec["ref_flux"] = ref_flux
        return flux, rec
