"""One HYBRID system with its massless particles split across two processes
on the GPU (mercuda_b200/shards.py sharded_hybrid_step): each step the ranks
all-gather mce_snif's pairs and the members' pre-drift states over gloo and
integrate the one global encounter subsystem a single process would, so each
shard's final states, the encounter records and the pair counts equal the
single-process run's bit for bit. The processes exchange host values between
calls only; no kernel waits on another process."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
H, NSTEPS, TOL, RCEN = 8.0, 14, 1e-12, 0.005

pytestmark = pytest.mark.gpu


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def case():
    from mercuda_b200.system import make_system
    return make_system(seed=12, n_particles=900, nplanets=8, near_fraction=0.08, h=H)


def worker(rank, world, port, out_dir):
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    import torch.distributed as dist
    from datetime import timedelta
    from mercuda_b200.backend import Backend
    from mercuda_b200.shards import Ranks, particle_shard, sharded_hybrid_step

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        ranks = Ranks(dist, device="cpu")
        s = case()
        shard, ids = particle_shard(s, rank, world)
        be = Backend("HYBRID")
        be.configure()
        be.upload(shard)
        state, t, pairs, records = {"dtflag": 0}, 0.0, [], []
        try:
            for _ in range(NSTEPS):
                ev, npair = sharded_hybrid_step(be, ranks, shard, ids, t, H, TOL, state, RCEN)
                t += H
                pairs.append(npair)
                records.append(ev)
            x, v = be.download()
        finally:
            be.free()
        ev = np.concatenate(records)
        np.savez(Path(out_dir) / f"rank{rank}.npz", x=x, v=v, ids=ids, pairs=np.array(pairs), ev=ev)
    finally:
        dist.destroy_process_group()


def canonical(ev):
    return sorted(e.tobytes() for e in ev)


def test_sharded_hybrid_run_equals_unsharded(cuda_lib, tmp_path):
    from mercuda_b200.backend import Backend
    s = case()
    be = Backend("HYBRID", cuda_lib)
    be.configure()
    be.upload(s.copy())
    state, t, pairs, records = {"dtflag": 0}, 0.0, [], []
    for _ in range(NSTEPS):
        ev, npair = be.hybrid_step(s, t, H, TOL, state, RCEN)
        t += H
        pairs.append(npair)
        records.append(ev)
    x, v = be.download()
    be.free()
    assert sum(pairs) > 20
    world = 2
    mp.start_processes(worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    ranks = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    want_ev = canonical(np.concatenate(records))
    for r in ranks:
        ids = r["ids"]
        assert np.array_equal(r["x"], x[ids]) and np.array_equal(r["v"], v[ids])
        assert list(r["pairs"]) == pairs
        assert canonical(r["ev"]) == want_ev
