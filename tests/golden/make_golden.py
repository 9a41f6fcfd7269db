"""Generates the golden fixtures in this directory from the reference itself.

The reference's own CPU task bodies (sweep.cc, outer.cc, inner.cc, expxs.cc,
init.cc; compiled from the reference sources through oracle/refshim into
oracle/_ref/libsnapref.so) are run on the benchmark decks and their outputs are
saved as small .npz fixtures:

  deck1_ref.npz   16^3, A=10, G=4, nmom=1: full solve (scalar flux of every
                  cell and group, iteration record), the flux after the first
                  inner iteration, and the reference's own material/source
                  layout from InitMaterial/InitSource.
  deck2p_ref.npz  64^3, A=36, G=32, nmom=1 ("deck 2 prime", deck 2 at nmom=1,
                  the largest case the reference's CPU path can run): the
                  iteration record, per-group sums and maxima and 4096 seeded
                  sample entries of the converged scalar flux.

The reference's CPU path cannot run nmom > 1 (its non-MMS sweep dereferences
an unbound flux-moment accessor, sweep.cc:312-317 against :575-590), so the
multi-moment benchmark decks are pinned by the oracle's C restatement
(oracle/snap_oracle.c, itself checked against the reference build at nmom = 1
and against deck1_ref/deck2p_ref above), run on all host threads:

  deck2_oracle.npz  64^3, A=36, G=32, nmom=4 (deck 2 exactly, the benchmark
                    configuration): iteration record, per-group sums and
                    maxima of every moment, 4096 seeded samples of the
                    converged scalar flux and 512 seeded samples of all 16
                    moments.
  deck4_oracle.npz  32^3, A=24, G=16, nmom=2 with the per-cell +-10 % sigma_t
                    field (the adjoint deck's forward solve): the same items.

Usage: python tests/golden/make_golden.py [deck1] [deck2p] [deck2] [deck4]
"""
from __future__ import annotations

import pathlib
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "legion-snap_b200"))

from oracle.bindings import Oracle, RefSnap, build  # noqa: E402
from snap_b200 import problem as P  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent


def deck1():
    d = P.deck(1)
    prob = P.make_problem(d)
    ref = RefSnap(d)
    mat, qi = ref.init_layout()
    flux, rec = ref.solve(prob)
    flux1, rec1 = ref.solve(prob, max_inners=1)
    np.savez_compressed(
        OUT / "deck1_ref.npz", flux0=flux, flux0_first_inner=flux1, ref_mat=mat, ref_qi=qi,
        inner_total=rec["inner_total"], outer_total=rec["outer_total"],
        converged=rec["converged"], inners_per_outer=np.array(rec["inners_per_outer"]),
        variant=rec["variant"])
    print("deck1", rec)


def deck2p():
    d = P.deck(2, nmom=1)
    prob = P.make_problem(d)
    ref = RefSnap(d)
    t = time.time()
    flux, rec = ref.solve(prob)
    print("deck2p solve", time.time() - t, "s", rec)
    rng = np.random.default_rng(2024)
    gs = rng.integers(0, d.ng, 4096)
    cs = rng.integers(0, d.cells, 4096)
    np.savez_compressed(
        OUT / "deck2p_ref.npz", sample_g=gs, sample_c=cs, sample_flux0=flux[gs, cs],
        group_sum=flux.sum(axis=1), group_max=flux.max(axis=1),
        inner_total=rec["inner_total"], outer_total=rec["outer_total"],
        converged=rec["converged"], inners_per_outer=np.array(rec["inners_per_outer"]),
        variant=rec["variant"], seconds=rec["seconds"], nthreads=rec["nthreads"])


def oracle_fixture(name, d):
    import os
    prob = P.make_problem(d)
    threads = os.cpu_count() or 1
    t = time.time()
    flux, rec = Oracle(d, threads=threads).solve(prob)
    secs = time.time() - t
    print(name, "oracle solve", secs, "s", rec)
    rng = np.random.default_rng(2025)
    gs = rng.integers(0, d.ng, 4096)
    cs = rng.integers(0, d.cells, 4096)
    mg = rng.integers(0, d.ng, 512)
    mc = rng.integers(0, d.cells, 512)
    np.savez_compressed(
        OUT / f"{name}_oracle.npz", sample_g=gs, sample_c=cs, sample_flux0=flux[gs, cs, 0],
        moment_g=mg, moment_c=mc, moment_flux=flux[mg, mc, :],
        group_sum=flux.sum(axis=1), group_max=np.abs(flux).max(axis=1),
        inner_total=rec["inner_total"], outer_total=rec["outer_total"],
        converged=rec["converged"], inners_per_outer=np.array(rec["inners_per_outer"]),
        seconds=secs, nthreads=threads)


def deck2():
    oracle_fixture("deck2", P.deck(2))


def deck4():
    oracle_fixture("deck4", P.deck(4))


if __name__ == "__main__":
    build()
    which = sys.argv[1:] or ["deck1", "deck2p"]
    for w in which:
        globals()[w]()
