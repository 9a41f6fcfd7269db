"""Group-sharded solve over several processes (one per GPU).

The energy groups are independent within every inner iteration (inner
source, sweep and inner test are per group); only the outer source couples
them (outer.cc:107-217 reads every group's flux).  A rank therefore owns a
contiguous block of groups and the solve loop of snap.cc:472-540 needs two
exchanges:

- once per outer iteration, an all-gather of the flux moments, so that each
  rank can form the outer source of its own groups from every group's flux;
- after every inner iteration and outer test, an AND of the convergence
  flags (the reference ANDs per-group-chunk futures, snap.cc:890-936).

``sharded_transport_solve`` is written against two small interfaces, so the
same loop runs on GPUs (``GpuShard`` over the C ABI, NCCL) and in the CPU
tests (an oracle-backed shard, gloo).
"""
from __future__ import annotations

import numpy as np


def shard_groups(ng: int, world: int, rank: int) -> tuple[int, int]:
    """(first group, group count) of `rank`: contiguous, sizes differ by <= 1."""
    base, extra = divmod(ng, world)
    lo = rank * base + min(rank, extra)
    return lo, base + (1 if rank < extra else 0)


class TorchComm:
    """The two exchanges over torch.distributed (NCCL on GPUs, gloo on CPUs).
    Group shards may differ in size by one group, so the gather pads."""

    def __init__(self, dist, group=None):
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)

    def all_gather_groups(self, local, counts):
        import torch
        width = max(counts)
        pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
        pad[: local.shape[0]] = local
        out = torch.empty((self.world * width,) + tuple(local.shape[1:]), dtype=local.dtype,
                          device=local.device)
        self.dist.all_gather_into_tensor(out, pad, group=self.group)
        parts = [out[r * width: r * width + counts[r]] for r in range(self.world)]
        return torch.cat(parts, 0).contiguous()

    def all_true(self, flag: bool, device) -> bool:
        import torch
        t = torch.tensor([0 if flag else 1], dtype=torch.int32, device=device)
        self.dist.all_reduce(t, group=self.group)
        return int(t.item()) == 0


def sharded_transport_solve(shard, comm, ng_total: int, world: int, epsi: float, iitm: int,
                            oitm: int):
    """snap.cc:472-540 with the groups split over ranks.

    shard: this rank's operations on its groups --
      zero_flux() -> local flux; outer_source(flux_all) -> q2;
      inner_iteration(q2, flux) -> bool (flux updated in place);
      outer_test(flux, flux_po) -> bool; copy(flux) -> copy; device
    comm: all_gather_groups(local, counts) and all_true(flag, device).
    Returns the local flux and the iteration record (identical on every rank).
    """
    counts = [shard_groups(ng_total, world, r)[1] for r in range(world)]
    flux = shard.zero_flux()
    rec = dict(inner_total=0, outer_total=0, converged=False, inners_per_outer=[])
    for o in range(oitm):
        flux_all = comm.all_gather_groups(flux, counts)
        q2 = shard.outer_source(flux_all)
        fpo = shard.copy(flux)
        conv, inners = False, 0
        for _ in range(iitm):
            conv = comm.all_true(shard.inner_iteration(q2, flux), shard.device)
            inners += 1
            if conv:
                break
        rec["inner_total"] += inners
        rec["outer_total"] += 1
        rec["inners_per_outer"].append(inners)
        if o == 0:
            continue
        if conv and comm.all_true(shard.outer_test(flux, fpo), shard.device):
            rec["converged"] = True
            break
    return flux, rec


def shard_problem(prob: dict, g_lo: int, g_n: int) -> dict:
    """The host-side deck arrays a shard needs: its groups' fixed source and
    total cross sections, the in-shard block of the scattering table (for the
    in-group expansion) and the full table (for the outer source)."""
    sl = slice(g_lo, g_lo + g_n)
    out = dict(mat=prob["mat"], qi=np.ascontiguousarray(prob["qi"][sl]),
               sigt=np.ascontiguousarray(prob["sigt"][sl]),
               slgg_block=np.ascontiguousarray(prob["slgg"][sl, :, sl, :]),
               slgg_full=np.ascontiguousarray(prob["slgg"]), nmat=prob.get("nmat", 2))
    if "sigt_scale" in prob:
        out["sigt_scale"] = prob["sigt_scale"]
    return out


class GpuShard:
    """Shard operations on one GPU through the C ABI (a context holding the
    shard's g_n groups)."""

    def __init__(self, deck, prob: dict, g_lo: int, g_n: int, device: int = 0,
                 precision: str = "fp64"):
        import dataclasses

        import torch

        from .solver import Snap
        self.torch = torch
        self.g_lo, self.g_n, self.ng_total = g_lo, g_n, deck.ng
        self.deck = dataclasses.replace(deck, ng=g_n)
        self.snap = Snap(self.deck, precision=precision, device=device)
        self.device = self.snap.device
        sp = shard_problem(prob, g_lo, g_n)
        dev = lambda a: torch.as_tensor(a, device=self.device)   # noqa: E731
        self.mat, self.qi = dev(sp["mat"]), dev(sp["qi"])
        self.slgg_full = dev(sp["slgg_full"])
        t_xs = self.snap.expand_cross_section(dev(sp["sigt"]), self.mat)
        if "sigt_scale" in sp:
            t_xs *= dev(sp["sigt_scale"])[None, :]
        self.t_xs = t_xs.to(self.snap.sweep_dtype).contiguous()
        self.s_xs = self.snap.expand_scattering_cross_section(dev(sp["slgg_block"]), self.mat)
        d = self.deck
        self.qtot = torch.empty(g_n, d.cells, d.cmom, dtype=self.snap.sweep_dtype,
                                device=self.device)
        self.epsi = deck.epsi

    def zero_flux(self):
        d = self.deck
        return self.torch.zeros(self.g_n, d.cells, d.cmom, dtype=self.torch.float64,
                                device=self.device)

    def copy(self, flux):
        return flux.clone()

    def outer_source(self, flux_all):
        from . import abi
        from .solver import _ptr, _stream
        q2 = self.torch.empty_like(self.zero_flux())
        abi.check(self.snap.lib.snap_calc_outer_source_groups(
            self.snap.handle, self.g_lo, self.ng_total, _ptr(self.qi), _ptr(self.slgg_full),
            _ptr(self.mat), _ptr(flux_all), _ptr(q2), _stream()))
        return q2

    def inner_iteration(self, q2, flux):
        return self.snap.inner_iteration(self.s_xs, q2, self.t_xs, flux, self.qtot, self.epsi)

    def outer_test(self, flux, fpo):
        return self.snap._test(1, flux, fpo, 100.0 * self.epsi)
