#!/usr/bin/env python
"""Grind-time benchmark of the steady-state solve path on deck 2.

Workload (deck 2): 64^3 cells on the unit cube, 36 angles per octant (288),
32 groups, nmom = 4 (16 flux moments), FP64, centre material-2 block with a
unit source, fixup on.  Inputs are generated on the host with the deck's
cross-section rule (synthetic, seeded; there is no external data set).

A step is one inner iteration on device-resident data (inner source, the
8-octant x 32-group sweep, octant sum and inner convergence test).  The metric
is grind time = step time / (cells x 8 x angles x groups), in ns; lower is
better.  qtot alone is 1.07 GB per step, far larger than the 126 MB L2, so no
L2 flush is needed between steps.

  value   device-resident grind time (CUDA events, max over ranks)
  e2e     grind time of whole solves through the public C ABI
          (snap_transport_solve) from pinned host buffers, host->device copies
          of the deck and the device->host copy of the flux inside the timed
          region, per inner iteration executed
  roofline  the sweep kernel: algorithmic bytes (3*cmom+1)*8/angles per unit
          x units per launch / CUDA-event duration, against the measured HBM
          copy bandwidth
  cpu_baseline  the reference's own CPU task bodies (oracle/_ref) on the host
          cores, bounded sample

  same_config  deck 2' (deck 2 at nmom = 1) on the GPU against the reference's
          own task bodies running the same step (the reference's CPU path
          cannot run nmom > 1)
  reference_decks  the reference's own time-dependent performance decks
          (input/*_4K_1x1x1.in) solved on the GPU, beside a bounded sample of
          the reference's task bodies on the same decks

--impl reference times the reference's CPU path alone (rank 0 only) on deck
2', the same step.
Multi-GPU (torchrun): each rank owns a 32-group shard of a 32*N-group deck
(weak scaling); every step ANDs the inner tests over the ranks and every
iitm-th step carries the per-outer exchange (NCCL all-gather of the flux
moments, then each rank's outer source from all groups).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "legion-snap_b200"))

METRIC = "grind time ns/(cell*angle*group), FP64 inner iteration"
UNIT = "ns"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["snap", "reference"], default="snap")
    ap.add_argument("--e2e-solves", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-inners", type=int, default=2)
    ap.add_argument("--no-mixed", action="store_true", help="skip the FP32 leg")
    ap.add_argument("--no-mixed-large", action="store_true",
                    help="skip the mixed-precision leg on the 128^3, 64-group deck")
    ap.add_argument("--no-memory-deck", action="store_true",
                    help="skip the FP32 forward solve on the 192^3, 64-group, nmom 3 deck")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint leg")
    ap.add_argument("--no-decks", action="store_true",
                    help="skip the reference's own time-dependent decks")
    ap.add_argument("--decks", default="tiny_4K_1x1x1.in,small_4K_1x1x1.in,medium_4K_1x1x1.in,"
                                       "large_4K_1x1x1.in,huge_4K_1x1x1.in")
    ap.add_argument("--groups", type=int, default=None,
                    help="override deck 2's 32 groups (small cases for profiling only)")
    return ap.parse_args()


GROUPS = None


def deck2():
    from snap_b200 import problem as P
    return P.deck(2) if GROUPS is None else P.deck(2, ng=GROUPS)


def workload_config(d, precision="fp64"):
    name = "deck 2" if d.nmom == 4 else f"deck 2' (deck 2 at nmom={d.nmom})"
    return {
        "workload": f"{name}: {d.nx}^3 cells, {d.nang} angles/octant, {d.ng} groups, "
                    f"nmom={d.nmom} ({d.cmom} moments), steady-state fixed source, fixup on",
        "cells": d.cells, "angles_per_octant": d.nang, "groups": d.ng, "nmom": d.nmom,
        "cmom": d.cmom, "precision": precision,
        "step": "one inner iteration: inner source + sweep of 8 octants x all groups + "
                "octant sum + inner convergence test",
        "units_per_step": d.units_per_sweep,
        "l2": "inputs larger than L2 (qtot 1.07 GB per step), no flush",
        "parallelism": "group shards per rank (weak)",
    }


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        j = json.loads(p.read_text())
        return float(j["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(name: str):
    """dram bytes per launch recorded in profiles/<name>.md (line
    'traffic_bytes_per_launch: N'), or None."""
    p = ROOT / "profiles" / f"{name}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in open(self.file.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], pcap=parts[8]))
            except ValueError:
                continue
        os.unlink(self.file.name)
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("pcap", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows),
                "sm_max_mhz": max(r["smax"] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


def deck2_prime():
    """Deck 2 at one moment (nmom = 1): the largest configuration of the
    benchmark deck the reference's CPU path can run (its nmom > 1 sweep
    dereferences an unbound flux-moment accessor, sweep.cc:312-317 against
    :575-590)."""
    from snap_b200 import problem as P
    return P.deck(2, nmom=1) if GROUPS is None else P.deck(2, nmom=1, ng=GROUPS)


def cpu_reference_sample(steps: int, warmup: int = 0):
    """The reference's own CPU task bodies (oracle/_ref) on deck 2' running
    exactly the GPU step: `steps` inner iterations (inner source, sweep,
    inner test; group-parallel on every host thread, as the reference's
    index launches run), after `warmup` untimed ones and one outer source."""
    from oracle.bindings import RefSnap
    from snap_b200 import problem as P
    if not RefSnap.available():
        return None
    d = deck2_prime()
    prob = P.make_problem(d)
    ref = RefSnap(d)
    threads = os.cpu_count() or 1
    if warmup:
        ref.time_inner(prob, warmup, nthreads=threads)
    r = ref.time_inner(prob, steps, nthreads=threads)
    grind = r["seconds"] * 1e9 / (d.units_per_sweep * steps)
    return {"value": grind, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"reference CPU task bodies (variant {r['variant']}: "
                      f"{['scalar', 'SSE', 'AVX'][r['variant']]}), deck 2' (deck 2 at nmom=1), "
                      f"{steps} inner iterations (inner source + sweep + inner test, "
                      f"group-parallel), {threads} threads",
            "sweep_only_ns": r["sweep_seconds"] * 1e9 / (d.units_per_sweep * steps),
            "ms_per_step": r["seconds"] * 1e3 / steps}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    d = deck2_prime()
    s = cpu_reference_sample(args.steps, args.warmup)
    if s is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU build oracle/_ref/libsnapref.so not present"}))
        return 0
    value = s["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": s["ms_per_step"], "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(d, "fp64"),
        "note": "the reference's CPU path runs nmom = 1 only, so this arm times deck 2' (deck 2 "
                "at nmom = 1, same mesh, angles and groups); the GPU arm's headline is deck 2 at "
                "nmom = 4 and its same_config block times deck 2' on the GPU",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": s["cores"],
                         "kind": "reference", "sample": s["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def gpu_inner_grind(d, steps, warmup, local, precision="fp64"):
    """Device-resident inner iterations of deck d on one GPU: ms per step and
    grind time."""
    import torch

    from snap_b200 import problem as P
    from snap_b200.solver import Snap
    snap = Snap(d, precision=precision, device=local)
    prob = P.make_problem(d)
    dp = snap.device_problem(prob)
    t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"])
    if precision != "fp64":
        t_xs = t_xs.float()
    s_xs = snap.expand_scattering_cross_section(dp["slgg"], dp["mat"])
    flux = torch.zeros(d.ng, d.cells, d.cmom, dtype=torch.float64, device="cuda")
    q2 = snap.calc_outer_source(dp["qi"], dp["slgg"], dp["mat"], flux)
    qtot = torch.empty(d.ng, d.cells, d.cmom, dtype=snap.sweep_dtype, device="cuda")
    for _ in range(warmup):
        snap.inner_iteration(s_xs, q2, t_xs, flux, qtot)
    torch.cuda.synchronize()
    snap.timing(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        snap.inner_iteration(s_xs, q2, t_xs, flux, qtot)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    tm = snap.timing()
    snap.close()
    return {"ms_per_step": ms, "value": ms * 1e6 / d.units_per_sweep,
            "sweep_ms": tm["sweep_ms"] / max(tm["sweep_calls"], 1)}


MIXED_PRECISION = ("fp32 sweep (moment contractions on FP64 tensor cores); group-to-group "
                   "outer source on the tcgen05 tensor cores (split BF16 operands, fp32 "
                   "accumulation in tensor memory) while some scalar flux changes by more than "
                   "1000*epsi per outer, fp64 tensor-core source for the final outers; fp64 "
                   "octant sums, inner sources and convergence")


def outer_source_times(snap, snap32, dp, flux, reps=5):
    """Device time of one outer source: the FP64 tensor-core (DMMA) kernel
    against the split-BF16 tcgen05 kernel, on the same flux."""
    import torch
    out = {}
    for name, fn in (("fp64_dmma_ms", snap.calc_outer_source),
                     ("bf16_tcgen05_ms", snap32.calc_outer_source_tc)):
        fn(dp["qi"], dp["slgg"], dp["mat"], flux)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn(dp["qi"], dp["slgg"], dp["mat"], flux)
        e1.record()
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    out["speedup"] = out["fp64_dmma_ms"] / out["bf16_tcgen05_ms"]
    return out


def mixed_large_deck(local):
    """The mixed-precision configuration at 128^3 cells, 48 angles, 64 groups,
    nmom 4: FP32 inner-iteration grind time against FP64, whole-solve times
    and the scalar-flux error of the FP32 solve against the FP64 solve."""
    import torch

    from snap_b200 import problem as P
    from snap_b200.solver import Snap, fp64_finish
    d = P.deck(3)
    prob = P.make_problem(d)
    res = {"deck": "128^3 cells, 48 angles/octant, 64 groups, nmom=4 (16 moments), fixup on",
           "units_per_sweep": d.units_per_sweep}
    try:
        phi = {}
        for prec in ("fp64", "fp32"):
            snap = Snap(d, precision=prec, device=local)
            dp = snap.device_problem(prob)
            flux, rec = snap.transport_solve(dp)
            phi[prec] = flux[..., 0].clone()
            if prec == "fp32":
                phi["fp32_flux"] = flux
                snap_dp = dp
            res[prec] = {"solve_ms": rec["total_ms"], "inner_iterations": rec["inner_total"],
                         "outer_iterations": rec["outer_total"], "converged": rec["converged"],
                         "sweep_ms": rec["sweep_ms"] / max(rec["inner_total"], 1),
                         "grind_ns": rec["sweep_ms"] / max(rec["inner_total"], 1) * 1e6
                                     / d.units_per_sweep,
                         "sweep_scratch_gb": snap.scratch_bytes / 1e9}
            if prec == "fp32":
                res[prec]["outers_lowp_source"] = rec["outers_lowp"]
            del flux
            snap.close()
            del snap
            torch.cuda.empty_cache()
        diff = (phi["fp32"] - phi["fp64"]).abs() / phi["fp64"].abs().clamp_min(1e-300)
        if "fp32_flux" in phi:
            # FP64 refinement from the FP32 solution: one FP64 outer iteration
            # (inner sweeps until the inner test passes), and a single FP64
            # inner iteration
            dp = snap_dp
            f32 = phi.pop("fp32_flux")
            for key, kw in (("fp64_finish", {}), ("fp64_one_sweep", {"max_inners": 1})):
                fin, st = fp64_finish(d, dp, f32, outers=1, device=local, **kw)
                dfin = (fin[..., 0] - phi["fp64"]).abs() / phi["fp64"].abs().clamp_min(1e-300)
                res[key] = {"ms": st["ms"], "inner_iterations": st["inner_iterations"],
                            "max_rel_err_scalar_flux": float(dfin.max()),
                            "rms_rel_err_scalar_flux": float(dfin.pow(2).mean().sqrt()),
                            "solve_plus_finish_speedup_vs_fp64":
                                res["fp64"]["solve_ms"] / (res["fp32"]["solve_ms"] + st["ms"])}
                del fin
                torch.cuda.empty_cache()
            del f32, dp, snap_dp
        res["max_rel_err_scalar_flux"] = float(diff.max())
        res["rms_rel_err_scalar_flux"] = float(diff.pow(2).mean().sqrt())
        res["frac_values_above_1e-5"] = float((diff > 1e-5).double().mean())
        res["sweep_speedup_fp32_vs_fp64"] = res["fp64"]["sweep_ms"] / res["fp32"]["sweep_ms"]
        res["solve_speedup_fp32_vs_fp64"] = res["fp64"]["solve_ms"] / res["fp32"]["solve_ms"]
    except Exception as e:   # report, do not lose the main bench line
        res["error"] = f"{type(e).__name__}: {e}"
    # the library allocates with cudaMalloc: hand torch's cached blocks back
    phi = None
    torch.cuda.empty_cache()
    return res


def memory_pressure_deck(local):
    """FP32 forward solve of the 192^3 cells, 48 angles, 64 groups, nmom 3
    deck with a seeded random 50 % material mix in the central 96^3 block,
    one octant per sweep launch (the device holds about 140 GB for it).  The
    FP64 solve of this deck does not fit beside it, so the error is not
    measured here; the 128^3 deck carries the error comparison."""
    import torch

    from snap_b200 import problem as P
    from snap_b200.solver import Snap
    d = P.deck(5)
    res = {"deck": "192^3 cells, 48 angles/octant, 64 groups, nmom=3 (9 moments), random 50% "
                   "material mix in the central 96^3 block, fixup on, FP32 sweep; adjoint of a "
                   "4^3 far-corner detector (weights 1/g), forward state recorded in group "
                   "batches from the converged moments",
           "units_per_sweep": d.units_per_sweep}
    old = os.environ.get("SNAP_B200_OCTANTS_PER_LAUNCH")
    os.environ["SNAP_B200_OCTANTS_PER_LAUNCH"] = "1"
    torch.cuda.empty_cache()   # the library's own cudaMalloc needs the memory torch caches
    try:
        snap = Snap(d, precision="fp32", device=local)
        dp = snap.device_problem(P.make_problem(d))
        flux, rec = snap.transport_solve(dp)
        free, total = torch.cuda.mem_get_info()
        res.update({"solve_ms": rec["total_ms"], "inner_iterations": rec["inner_total"],
                    "outer_iterations": rec["outer_total"], "converged": rec["converged"],
                    "outers_lowp_source": rec["outers_lowp"],
                    "sweep_ms": rec["sweep_ms"] / max(rec["inner_total"], 1),
                    "grind_ns": rec["sweep_ms"] / max(rec["inner_total"], 1) * 1e6 / d.units_per_sweep,
                    "scalar_flux_positive_finite": bool(torch.isfinite(flux).all()
                                                        and (flux[..., 0] > 0).all()),
                    "device_gb_in_use_after_solve": (total - free) / 1e9})
        # the adjoint of the same deck on the same context (FP32 adjoint
        # vectors in the context's solve arrays, state in group batches)
        try:
            r = torch.zeros(d.ng, d.nz, d.ny, d.nx, dtype=torch.float64, device="cuda")
            r[:, -4:, -4:, -4:] = (1.0 / torch.arange(1, d.ng + 1, dtype=torch.float64,
                                                      device="cuda"))[:, None, None, None]
            r = r.reshape(d.ng, d.cells)
            t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"])
            torch.cuda.empty_cache()
            g = snap.adjoint_solve(dp, t_xs, flux, r, epsi=1e-5, with_sxs=False)
            free, total = torch.cuda.mem_get_info()
            res["adjoint"] = {"ms": g["total_ms"], "iterations": g["iterations"],
                              "converged": g["converged"],
                              "adjoint_over_forward": g["total_ms"] / rec["total_ms"],
                              "grad_sigt_finite": bool(torch.isfinite(g["grad_sigt"]).all()),
                              "grad_qi_finite": bool(torch.isfinite(g["grad_qi"]).all()),
                              "device_gb_in_use": (total - free) / 1e9,
                              "scratch_gb": snap.scratch_bytes / 1e9}
            del g, r, t_xs
        except Exception as e:   # report, do not lose the main bench line
            res["adjoint"] = {"error": f"{type(e).__name__}: {e}"}
        del flux, dp
        snap.close()
        del snap
        torch.cuda.empty_cache()
    except Exception as e:   # report, do not lose the main bench line
        res["error"] = f"{type(e).__name__}: {e}"
    finally:
        if old is None:
            os.environ.pop("SNAP_B200_OCTANTS_PER_LAUNCH", None)
        else:
            os.environ["SNAP_B200_OCTANTS_PER_LAUNCH"] = old
    return res


def reference_decks(names, local, cpu: bool):
    """The reference's own performance decks (input/*_1x1x1.in: time
    dependent, 10 steps, 16 x 16 x 16 cells, 32 to 1024 angles, 16 to 96
    groups), solved whole on the GPU (second of two solves timed) and, when
    `cpu`, a bounded sample of the reference's task bodies on the same deck
    (2 inner iterations incl. one outer source, all host threads): time per
    inner iteration on both sides."""
    import torch

    from snap_b200 import input_deck as D
    from snap_b200 import problem as P
    from snap_b200.solver import Snap
    out = {}
    for name in names:
        try:
            d = D.parse_deck(ROOT / "tests" / "decks" / name).deck
            prob = P.make_problem(d)
            snap = Snap(d, device=local)
            dp = snap.device_problem(prob)
            snap.transport_solve(dp)
            flux, rec = snap.transport_solve(dp)
            snap.close()
            del snap, flux, dp
            torch.cuda.empty_cache()
            r = {"angles": d.nang, "groups": d.ng, "cells": d.cells, "steps": d.nsteps,
                 "gpu_solve_ms": rec["total_ms"], "inner_iterations": rec["inner_total"],
                 "gpu_ms_per_inner": rec["total_ms"] / rec["inner_total"],
                 "gpu_sweep_ps_per_unit": rec["sweep_ms"] / rec["inner_total"] * 1e9
                                          / d.units_per_sweep}
            if cpu:
                from oracle.bindings import RefSnap
                if RefSnap.available():
                    _, rr = RefSnap(d).solve(prob, nthreads=os.cpu_count() or 1, max_inners=2)
                    r["reference_cpu_ms_per_inner"] = rr["seconds"] * 1e3 / rr["inner_total"]
                    r["reference_cpu_threads"] = os.cpu_count() or 1
                    r["reference_over_gpu_per_inner"] = (r["reference_cpu_ms_per_inner"]
                                                         / r["gpu_ms_per_inner"])
            out[name] = r
        except Exception as e:   # report, do not lose the main bench line
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    return out


def run_snap(args):
    import torch
    import torch.distributed as dist

    from snap_b200 import problem as P
    from snap_b200.solver import Snap

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        # NCCL's communicator set-up log (stderr) shows the ranks and the
        # transport it chose (NVLink / NVLS), unless the caller set otherwise
        os.environ.setdefault("NCCL_DEBUG", "INFO")
        os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    d = deck2()
    snap = Snap(d, device=local)
    prob = P.make_problem(d)
    dp = snap.device_problem(prob)
    t_xs = snap.expand_cross_section(dp["sigt"], dp["mat"])
    s_xs = snap.expand_scattering_cross_section(dp["slgg"], dp["mat"])
    flux = torch.zeros(d.ng, d.cells, d.cmom, dtype=torch.float64, device="cuda")
    q2grp = snap.calc_outer_source(dp["qi"], dp["slgg"], dp["mat"], flux)
    qtot = torch.empty(d.ng, d.cells, d.cmom, dtype=torch.float64, device="cuda")

    step_no = [0]
    if world > 1:
        # weak scaling: rank r owns groups 32r .. 32r+31 of a 32*world-group
        # deck; every iitm-th step carries the per-outer exchange (all-gather
        # of every group's flux moments over NCCL, then the outer source of
        # this rank's groups from all of them), every step the AND of the
        # inner tests
        import dataclasses

        from snap_b200.parallel import GpuShard, TorchComm
        d_total = dataclasses.replace(d, ng=d.ng * world)
        shard = GpuShard(d_total, P.make_problem(d_total), rank * d.ng, d.ng, device=local)
        comm = TorchComm(dist)
        counts = [d.ng] * world
        snap.close()
        snap = shard.snap
        flux = shard.zero_flux()
        q2_box = [shard.outer_source(comm.all_gather_groups(flux, counts))]

        def step():
            if step_no[0] % d.iitm == 0:
                q2_box[0] = shard.outer_source(comm.all_gather_groups(flux, counts))
            step_no[0] += 1
            return comm.all_true(shard.inner_iteration(q2_box[0], flux), shard.device)
    else:
        def step():
            step_no[0] += 1
            return snap.inner_iteration(s_xs, q2grp, t_xs, flux, qtot)

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    snap.timing(reset=True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    tm = snap.timing()
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    ms_per_step = ms / args.steps
    units_step = d.units_per_sweep * world
    value = ms_per_step * 1e6 / units_step

    # roofline of the sweep kernel
    sweep_ms = tm["sweep_ms"] / max(tm["sweep_calls"], 1)
    bytes_unit = (3 * d.cmom + 1) * 8 / d.nang
    algo = bytes_unit * d.units_per_sweep
    achieved = algo / (sweep_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic("sweep_fp64_deck2")

    # end to end: whole solves through the C ABI from pinned host memory
    host = {k: torch.as_tensor(v).pin_memory() for k, v in
            (("mat", prob["mat"]), ("qi", prob["qi"]), ("sigt", prob["sigt"]),
             ("slgg", prob["slgg"]))}
    flux_host = torch.empty(d.ng, d.cells, d.cmom, dtype=torch.float64).pin_memory()
    h2d = sum(t.numel() * t.element_size() for t in host.values())
    d2h = flux_host.numel() * flux_host.element_size()
    e2e_vals = []
    for _ in range(args.e2e_solves):
        dev = {k: torch.empty_like(v, device="cuda") for k, v in host.items()}
        out = torch.empty(d.ng, d.cells, d.cmom, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in dev:
            dev[k].copy_(host[k], non_blocking=True)
        _, rec = snap.transport_solve(dev, flux=out)
        flux_host.copy_(out, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        e2e_vals.append(e0.elapsed_time(e1) * 1e6 / (d.units_per_sweep * rec["inner_total"]))
    e2e_t = torch.tensor([statistics.mean(e2e_vals) if e2e_vals else float("nan")],
                         dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e = float(e2e_t.item()) / world

    # mixed-precision form on the same deck: FP32 sweep (FP64 octant sums,
    # sources and convergence); grind time and scalar-flux error against the
    # FP64 solve above
    mixed = None
    if not args.no_mixed:
        snap32 = Snap(d, precision="fp32", device=local)
        t_xs32 = t_xs.float()
        flux32 = torch.zeros(d.ng, d.cells, d.cmom, dtype=torch.float64, device="cuda")
        q2grp32 = snap32.calc_outer_source(dp["qi"], dp["slgg"], dp["mat"], flux32)
        qtot32 = torch.empty(d.ng, d.cells, d.cmom, dtype=torch.float32, device="cuda")
        for _ in range(args.warmup):
            snap32.inner_iteration(s_xs, q2grp32, t_xs32, flux32, qtot32)
        torch.cuda.synchronize()
        snap32.timing(reset=True)
        ev0.record()
        for _ in range(args.steps):
            snap32.inner_iteration(s_xs, q2grp32, t_xs32, flux32, qtot32)
        ev1.record()
        torch.cuda.synchronize()
        ms32 = ev0.elapsed_time(ev1) / args.steps
        tm32 = snap32.timing()
        sweep32 = tm32["sweep_ms"] / max(tm32["sweep_calls"], 1)
        mixed = {"precision": MIXED_PRECISION,
                 "value": ms32 * 1e6 / d.units_per_sweep, "unit": UNIT, "ms_per_step": ms32,
                 "speedup_vs_fp64": ms_per_step / ms32, "sweep_ms": sweep32,
                 "roofline": {"bound": "hbm", "bytes_per_unit": (3 * d.cmom + 1) * 4 / d.nang,
                              "achieved": (3 * d.cmom + 1) * 4 / d.nang * d.units_per_sweep
                                          / (sweep32 * 1e-3) / 1e9, "peak": peak}}
        mixed["roofline"]["frac"] = mixed["roofline"]["achieved"] / peak
        if e2e_vals:   # whole mixed solve against the FP64 solve of the e2e leg
            f32, rec32 = snap32.transport_solve(dp)
            ref = out[..., 0]
            diff = (f32[..., 0] - ref).abs() / ref.abs().clamp_min(1e-300)
            mixed["max_rel_err_scalar_flux"] = float(diff.max())
            mixed["rms_rel_err_scalar_flux"] = float(diff.pow(2).mean().sqrt())
            mixed["inner_iterations"] = rec32["inner_total"]
            mixed["fp64_inner_iterations"] = rec["inner_total"]
            mixed["outers_lowp_source"] = rec32["outers_lowp"]
            mixed["outer_iterations"] = rec32["outer_total"]
            mixed["solve_ms"] = rec32["total_ms"]
            mixed["fp64_solve_ms"] = rec["total_ms"]
            mixed["solve_speedup_vs_fp64"] = rec["total_ms"] / rec32["total_ms"]
        mixed["outer_source"] = outer_source_times(snap, snap32, dp, flux)
        snap32.close()
        del snap32, qtot32, flux32, q2grp32
        if not args.no_mixed_large:
            mixed["large_deck"] = mixed_large_deck(local)

    # adjoint cost on the adjoint deck (32^3, 24 angles, 16 groups, nmom 2,
    # per-cell sigma_t +-10 %): one converged forward solve and one converged
    # adjoint solve (detector response) to the same tolerance, device time
    adjoint = None
    if not args.no_adjoint:
        d4 = P.deck(4)
        snap4 = Snap(d4, device=local)
        dp4 = snap4.device_problem(P.make_problem(d4))
        r = torch.zeros(d4.ng, d4.nz, d4.ny, d4.nx, dtype=torch.float64, device="cuda")
        r[:, -4:, -4:, -4:] = (1.0 / torch.arange(1, d4.ng + 1, dtype=torch.float64,
                                                  device="cuda"))[:, None, None, None]
        r = r.reshape(d4.ng, d4.cells)
        eps4 = 1e-6
        fwd_ms, adj_ms = [], []
        for _ in range(2):
            f4, rec4 = snap4.transport_solve(dp4, epsi=eps4, iitm=5, oitm=100)
            t4 = snap4.expand_cross_section(dp4["sigt"], dp4["mat"]) * dp4["sigt_scale"][None, :]
            g4 = snap4.adjoint_solve(dp4, t4, f4, r, epsi=eps4)
            fwd_ms.append(rec4["total_ms"])
            adj_ms.append(g4["total_ms"])
        adjoint = {"deck": "32^3 cells, 24 angles/octant, 16 groups, nmom=2, fixup on, "
                           "detector 4^3 corner box, weights 1/g",
                   "epsi": eps4, "forward_ms": min(fwd_ms), "adjoint_ms": min(adj_ms),
                   "adjoint_over_forward": min(adj_ms) / min(fwd_ms),
                   "forward_inner_iterations": rec4["inner_total"],
                   "adjoint_iterations": g4["iterations"], "adjoint_converged": g4["converged"],
                   "note": "forward: per-cell relative test of snap.cc; adjoint: max-norm "
                           "relative change (the importance spans many decades)"}
        # per sweep: the adjoint solve runs its iterations plus one recording
        # forward sweep and one gradient sweep
        adjoint["adjoint_ms_per_sweep_over_forward_ms_per_inner"] = (
            (adjoint["adjoint_ms"] / (g4["iterations"] + 2))
            / (adjoint["forward_ms"] / rec4["inner_total"]))
        snap4.close()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (deck-2 rule, generated on the host)",
        "config": workload_config(d),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "step": "one whole solve (snap_transport_solve), per inner iteration executed",
                "inner_iterations": rec["inner_total"] if e2e_vals else 0},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "sweep_fp64_kernel", "peak_source": f"{peak_kind} hbm_gbs",
                     "bytes_per_unit": bytes_unit, "sweep_ms": sweep_ms},
        "gpu_launches": tm["kernel_launches"],
        "clocks": clk,
    }
    if mixed is not None:
        line["mixed_precision"] = mixed
    if adjoint is not None:
        line["adjoint"] = adjoint
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_reference_sample(args.cpu_inners)
        if cb is not None:
            line["cpu_baseline"] = cb
            # the same configuration on both sides: deck 2' on the GPU, the
            # same step as the reference's task bodies above
            d1 = deck2_prime()
            g1 = gpu_inner_grind(d1, args.steps, args.warmup, local)
            line["same_config"] = {
                "workload": workload_config(d1)["workload"],
                "step": "one inner iteration (inner source + sweep + inner test), both sides",
                "gpu_ns": g1["value"], "gpu_ms_per_step": g1["ms_per_step"],
                "reference_ns": cb["value"], "reference_ms_per_step": cb["ms_per_step"],
                "reference_over_gpu": cb["value"] / g1["value"],
                "note": "the driver's reference arm times deck 2' (the reference cannot run "
                        "nmom > 1); this block is the like-for-like ratio"}
    if rank == 0 and world == 1 and not args.no_decks:
        line["reference_decks"] = reference_decks(
            [x for x in args.decks.split(",") if x], local, not args.no_cpu_baseline)
    # the 192^3 deck needs nearly all of the device: run it last, after the
    # other legs' contexts and tensors are released
    snap.close()
    if mixed is not None and not args.no_memory_deck:
        del flux, qtot, q2grp, t_xs, s_xs, dp
        if args.e2e_solves > 0:
            del out, dev
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        mixed["memory_pressure_deck"] = memory_pressure_deck(local)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    global GROUPS
    args = parse()
    GROUPS = args.groups
    if args.impl == "reference":
        return run_reference(args)
    return run_snap(args)


if __name__ == "__main__":
    sys.exit(main())
