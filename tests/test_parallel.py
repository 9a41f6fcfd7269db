"""Group-sharded solve: the multi-rank loop on CPU with gloo (world size 2),
oracle-backed shards; it must reproduce the single-process solve."""
import os
import socket

import numpy as np
import pytest

from snap_b200 import parallel as par
from snap_b200 import problem as P

DECK = P.Deck(8, 8, 8, nang=4, ng=5, nmom=2, epsi=1e-6, iitm=3, oitm=6)


def test_shard_groups_partition():
    for ng in (1, 5, 32, 33):
        for world in (1, 2, 3, 8):
            if world > ng:
                continue
            spans = [par.shard_groups(ng, world, r) for r in range(world)]
            assert spans[0][0] == 0
            for (lo, n), (lo2, _) in zip(spans, spans[1:]):
                assert lo + n == lo2
            assert sum(n for _, n in spans) == ng
            assert max(n for _, n in spans) - min(n for _, n in spans) <= 1


class OracleShard:
    """Shard operations on the CPU oracle (test infrastructure)."""

    def __init__(self, deck, prob, g_lo, g_n):
        import dataclasses

        import torch

        from oracle.bindings import Oracle
        self.torch = torch
        self.device = torch.device("cpu")
        self.g_lo, self.g_n = g_lo, g_n
        self.full = Oracle(deck)
        self.prob = prob
        self.local = Oracle(dataclasses.replace(deck, ng=g_n))
        sp = par.shard_problem(prob, g_lo, g_n)
        local_prob = dict(mat=sp["mat"], sigt=sp["sigt"], slgg=sp["slgg_block"], qi=sp["qi"])
        self.t_xs, self.s_xs = self.local.expand(local_prob)
        self.deck = deck

    def zero_flux(self):
        d = self.deck
        return self.torch.zeros(self.g_n, d.cells, d.cmom, dtype=self.torch.float64)

    def copy(self, flux):
        return flux.clone()

    def outer_source(self, flux_all):
        q2 = self.full.outer_source(self.prob, np.ascontiguousarray(flux_all.numpy()))
        return q2[self.g_lo:self.g_lo + self.g_n].copy()

    def inner_iteration(self, q2, flux):
        f = flux.numpy()
        qtot = self.local.inner_source(self.s_xs, q2, np.ascontiguousarray(f))
        new = self.local.sweep(qtot, self.t_xs)
        conv = self.local.test_convergence(new, f, self.deck.epsi)
        f[...] = new
        return conv

    def outer_test(self, flux, fpo):
        return self.local.test_convergence(flux.numpy(), fpo.numpy(), 100.0 * self.deck.epsi)


def _rank_main(rank, world, port, out_dir):
    import sys
    import pathlib
    root = pathlib.Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "legion-snap_b200")]
    import datetime

    import torch.distributed as dist

    from snap_b200 import parallel as p2
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    prob = P.make_problem(DECK)
    g_lo, g_n = p2.shard_groups(DECK.ng, world, rank)
    shard = OracleShard(DECK, prob, g_lo, g_n)
    flux, rec = p2.sharded_transport_solve(shard, p2.TorchComm(dist), DECK.ng, world, DECK.epsi,
                                           DECK.iitm, DECK.oitm)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), flux=flux.numpy(), g_lo=g_lo,
             inners=np.array(rec["inners_per_outer"]), converged=rec["converged"])
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_rank_gloo_solve_matches_single_process(tmp_path):
    import torch.multiprocessing as mp

    from oracle.bindings import Oracle
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    ref, rec = Oracle(DECK).solve(P.make_problem(DECK))
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    flux = np.concatenate([p["flux"] for p in parts], axis=0)
    assert np.max(np.abs(flux - ref)) <= 1e-13 * np.max(np.abs(ref))
    for p in parts:
        assert list(p["inners"]) == rec["inners_per_outer"]
        assert bool(p["converged"]) == rec["converged"]
