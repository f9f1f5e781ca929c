"""The host logic of sharded HYBRID (mercuda_b200/shards.py
sharded_hybrid_step) on CPU: two gloo ranks against one process, with a
stand-in backend whose deterministic "physics" makes every member's end state
depend on the global pair list (its number of pairs over all ranks), so the
all-gather, the union of pairs and members, and the application of Big and
own members to each shard are all exercised. The GPU test
(test_shards_hybrid_gpu.py) runs the real kernels."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
NSTEPS, H = 6, 2.0


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class StandInBackend:
    """hybrid_begin / encounter_subsystem / hybrid_members / hybrid_finish /
    download with a made-up deterministic step; pairs form between a Big body
    and any later body closer than R before the 'drift'."""

    R = 0.35

    def __init__(self, sys_):
        self.x = sys_.x.copy()
        self.v = sys_.v.copy()
        self.nbig = sys_.nbig
        self.members = None

    def hybrid_begin(self, h, rcrit, flag, x, v):
        n = len(self.x)
        self.pre = self.x + 0.5 * h * self.v
        ce = np.zeros(n, dtype=np.int32)
        pi, pj = [], []
        for i in range(1, self.nbig):
            for j in range(i + 1, n):
                if np.linalg.norm(self.pre[i] - self.pre[j]) < self.R:
                    pi.append(i + 1)
                    pj.append(j + 1)
                    ce[i] = ce[j] = 2
        mem = np.nonzero(ce)[0]
        x[mem] = self.pre[mem]
        v[mem] = self.v[mem]
        self.members = mem
        return ce, np.array(pi, dtype=np.int64), np.array(pj, dtype=np.int64)

    def encounter_subsystem(self, sub, nbig, m, x, v, rcrit, rce, rphys, pi, pj, time, h, tol, state, rcen,
                            fused=True):
        from mercuda_b200.backend import EVENT_DTYPE
        sub = np.asarray(sub)
        counts = np.zeros(len(sub))
        for a in np.concatenate([pi, pj]):
            counts[np.searchsorted(sub, a - 1)] += 1
        xe = np.array(x) + h * np.array(v)
        xe[:, 0] += 1e-3 * counts
        ve = np.array(v) * (1.0 + 1e-4 * counts[:, None])
        records = []
        for a, b in zip(pi, pj):
            e = np.zeros(1, dtype=EVENT_DTYPE)[0]
            e["i"], e["j"], e["kind"] = a, b, 1
            ka, kb = np.searchsorted(sub, a - 1), np.searchsorted(sub, b - 1)
            e["time"] = time + h
            e["distance"] = np.linalg.norm(xe[ka] - xe[kb])
            records.append(e)
        state["hrec"] = state.get("hrec", h) * 0.5
        return xe, ve, records

    def hybrid_members(self, ids):
        self.members = np.asarray(ids)

    def hybrid_finish(self, h, m, x, v):
        post = self.pre + 0.5 * h * self.v
        mem = self.members
        post[mem] = x[mem]
        vv = self.v.copy()
        vv[mem] = v[mem]
        self.x, self.v = post, vv

    def download(self):
        return self.x.copy(), self.v.copy()


def system():
    from mercuda_b200.system import make_system
    return make_system(seed=9, n_particles=60, nplanets=4, near_fraction=0.5, h=8.0)


def run(ranks, sys_, ids):
    from mercuda_b200.shards import sharded_hybrid_step
    be = StandInBackend(sys_)
    state, out = {"dtflag": 0}, []
    for k in range(NSTEPS):
        ev, npair = sharded_hybrid_step(be, ranks, sys_, ids, k * H, H, 1e-12, state)
        out.append((ev, npair))
    return be.download(), out, state["hrec"]


def worker(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    import torch.distributed as dist
    from datetime import timedelta
    from mercuda_b200.shards import Ranks, particle_shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        s = system()
        shard, ids = particle_shard(s, rank, world)
        (x, v), out, hrec = run(Ranks(dist), shard, ids)
        ev = np.concatenate([o[0] for o in out])
        np.savez(Path(out_dir) / f"rank{rank}.npz", x=x, v=v, ids=ids, ev=ev,
                 pairs=np.array([o[1] for o in out]), hrec=hrec)
    finally:
        dist.destroy_process_group()


def test_sharded_hybrid_host_logic_equals_one_process(tmp_path):
    from mercuda_b200.shards import Ranks
    s = system()
    (x, v), out, hrec = run(Ranks(), s, np.arange(s.n))
    pairs = [o[1] for o in out]
    ev = np.concatenate([o[0] for o in out])
    assert sum(pairs) > 10
    world = 2
    mp.start_processes(worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npz")
        ids = got["ids"]
        assert np.array_equal(got["x"], x[ids]) and np.array_equal(got["v"], v[ids])
        assert list(got["pairs"]) == pairs and float(got["hrec"]) == hrec
        assert got["ev"].tobytes() == ev.tobytes()
