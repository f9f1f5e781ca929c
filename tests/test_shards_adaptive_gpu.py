"""One adaptive system (RADAU, BS, BS2) with its massless particles split
across two processes on the GPU, the step control's maxima all-reduced (MAX)
over gloo through the library's step-reduce hook (mercuda_b200/shards.py
step_reduce): every process takes the whole system's steps, so each shard's
final states equal the single-process run's bit for bit, and the event
records of all shards (Big-body records once) equal the single-process list.
The processes exchange only host values between steps; no kernel waits on
another process."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
TSTOP, H0, TOL, RCEN = 400.0, 2.0, 1e-12, 0.005

pytestmark = pytest.mark.gpu


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def case():
    from adaptive_cases import hvar_system
    return hvar_system(massive=False, pn=1, count=120)


def worker(rank, world, port, out_dir, algorithm):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    import torch.distributed as dist
    from datetime import timedelta
    from mercuda_b200.backend import Backend
    from mercuda_b200.shards import Ranks, particle_shard, step_reduce

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        ranks = Ranks(dist, device="cpu")
        s = case()
        shard, ids = particle_shard(s, rank, world)
        be = Backend(algorithm)
        be.configure()
        be.upload(shard)
        cb = step_reduce(ranks)
        be.set_step_reduce(cb)
        try:
            ev, where, h, steps = be.hvar_run(0.0, TSTOP, H0, TOL, RCEN)
            x, v = be.download()
        finally:
            be.set_step_reduce(None)
            be.free()
        ev = ev.copy()
        for f in ("i", "j"):
            ev[f] = ids[ev[f] - 1] + 1
        if rank != 0:   # records among the central and Big bodies: rank 0's
            keep = np.maximum(ev["i"], ev["j"]) > s.nbig
            ev, where = ev[keep], where[keep]
        np.savez(Path(out_dir) / f"rank{rank}.npz", x=x, v=v, ids=ids, h=h, steps=steps, ev=ev, where=where)
    finally:
        dist.destroy_process_group()


def key(ev, where):
    return sorted((int(w), min(int(e["i"]), int(e["j"])), max(int(e["i"]), int(e["j"])), int(e["kind"]),
                   e.tobytes()) for e, w in zip(ev, where))


@pytest.mark.parametrize("algorithm", ["RADAU", "BS", "BS2"])
def test_sharded_adaptive_run_equals_unsharded(cuda_lib, tmp_path, algorithm):
    from mercuda_b200.backend import Backend
    s = case()
    be = Backend(algorithm, cuda_lib)
    be.configure()
    be.upload(s.copy())
    ev, where, h, steps = be.hvar_run(0.0, TSTOP, H0, TOL, RCEN)
    x, v = be.download()
    be.free()
    assert steps > 15
    world = 2
    mp.start_processes(worker, args=(world, free_port(), str(tmp_path), algorithm), nprocs=world, join=True,
                       start_method="spawn")
    ranks = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    for r in ranks:
        assert int(r["steps"]) == steps and float(r["h"]) == h
        ids = r["ids"]
        assert np.array_equal(r["x"], x[ids]) and np.array_equal(r["v"], v[ids])
    got_ev = np.concatenate([r["ev"] for r in ranks])
    got_where = np.concatenate([r["where"] for r in ranks])
    assert key(got_ev, got_where) == key(ev, where)
