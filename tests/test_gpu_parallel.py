"""The group-sharded solve's GPU operations: two C-ABI shards on one GPU,
driven from two host threads through an in-process exchange (the shards'
kernels never wait on each other; each shard's work is stream-ordered), must
reproduce the single-context solve."""
import threading

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not torch.cuda.is_available(), reason="needs a CUDA device"),
]

from snap_b200 import parallel as par  # noqa: E402
from snap_b200 import problem as P  # noqa: E402


class ThreadComm:
    def __init__(self, world, rank, shared):
        self.world, self.rank, self.s = world, rank, shared

    def _exchange(self, value):
        s = self.s
        s["slots"][self.rank] = value
        s["barrier"].wait()
        vals = list(s["slots"])
        s["barrier"].wait()
        return vals

    def all_gather_groups(self, local, counts):
        torch.cuda.synchronize()
        return torch.cat(self._exchange(local), 0).contiguous()

    def all_true(self, flag, device):
        return all(self._exchange(bool(flag)))


def test_two_gpu_shards_match_single_context():
    from snap_b200.solver import Snap
    d = P.Deck(16, 16, 16, nang=12, ng=5, nmom=2, epsi=1e-6, iitm=3, oitm=8)
    prob = P.make_problem(d)
    world = 2
    shards = [par.GpuShard(d, prob, *par.shard_groups(d.ng, world, r)) for r in range(world)]
    shared = dict(slots=[None] * world, barrier=threading.Barrier(world))
    out = [None] * world

    def run(r):
        out[r] = par.sharded_transport_solve(shards[r], ThreadComm(world, r, shared), d.ng, world,
                                             d.epsi, d.iitm, d.oitm)

    threads = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    snap = Snap(d)
    ref, rec = snap.transport_solve(snap.device_problem(prob))
    flux = torch.cat([o[0] for o in out], 0)
    assert float((flux - ref).abs().max() / ref.abs().max()) < 1e-12
    for o in out:
        assert o[1]["inners_per_outer"] == rec["inners_per_outer"]
