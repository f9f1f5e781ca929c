"""The N > 1 path on CPU: two gloo ranks, each integrating its share of the
test particles (mercuda_b200/shards.py). The oracle stands in for the device
backend behind the same host code, so the sharding, id mapping, de-duplication
of Big-body records and gathering are exercised without a GPU: the gathered
states and event records must equal an unsharded run bit for bit (massless
particles act on nothing)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
H, NSTEPS, RCEN = 8.0, 30, 0.005


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def canonical(ev, st):
    order = sorted(range(len(ev)), key=lambda q: (int(st[q]), ev[q].tobytes()))
    order = np.asarray(order, dtype=np.int64)
    return ev[order], st[order]


class OracleBackend:
    """The upload / mvs_advance / download surface of backend.Backend, on the
    CPU oracle (test infrastructure)."""

    def __init__(self, oracle):
        self.oracle = oracle
        self.s = None

    def upload(self, s, ngflag=None):
        self.s = s.copy()

    def mvs_advance(self, time, h, nsteps, rcen, steps_per_launch=0):
        return self.oracle.mvs_run(self.s, time, h, nsteps, rcen, central=True, threads=1)

    def download(self):
        return self.s.x.copy(), self.s.v.copy()

    def mvs_run(self, s, time, h, nsteps, rcen, steps_per_launch=0, ngflag=None, out=None):
        self.upload(s, ngflag)
        ev, st = self.mvs_advance(time, h, nsteps, rcen, steps_per_launch)
        x, v = self.download()
        if out is not None:
            out[0][...] = x
            out[1][...] = v
            x, v = out
        return ev, st, x, v


def system():
    from mercuda_b200.system import make_system
    return make_system(seed=5, n_particles=401, near_fraction=0.3, h=H)


def worker(rank, world, port, out_dir, case):
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    import torch.distributed as dist
    from datetime import timedelta
    from mercuda_b200.shards import Ranks, ShardedRun, particle_shard
    from oracle import oracle as O

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        ranks = Ranks(dist)
        assert ranks.rank == rank and ranks.world == world and ranks.device == "cpu"
        if case == "run":
            s = system()
            shard, ids = particle_shard(s, rank, world)
            run = ShardedRun(ranks, OracleBackend(O))
            run.upload(shard, ids, s.n)
            ranks.barrier()
            got = run.advance(0.0, H, NSTEPS, RCEN)
            states = run.download()
            own = run.download(gather=False)
            t = ranks.max(1.0 + rank)
            if rank == 0:
                ev, st = got
                np.savez(Path(out_dir) / "rank0.npz", ev=ev, st=st, x=states[0], v=states[1], t=t,
                         value=ranks.whole_job(100.0, t), own_n=len(own[0]))
            else:
                assert got is None and states is None
                np.savez(Path(out_dir) / f"rank{rank}.npz", own_n=len(own[0]), t=t)
        elif case == "onecall":
            # upload + advance + own states back in one call per rank
            s = system()
            shard, ids = particle_shard(s, rank, world)
            run = ShardedRun(ranks, OracleBackend(O))
            out = (np.zeros((shard.n, 3)), np.zeros((shard.n, 3)))
            got, (x, v) = run.run(shard, ids, s.n, 0.0, H, NSTEPS, RCEN, out=out)
            assert x is out[0] and v is out[1]
            if rank == 0:
                ev, st = got
                np.savez(Path(out_dir) / "rank0.npz", ev=ev, st=st, x=x, v=v, ids=ids)
            else:
                assert got is None
                np.savez(Path(out_dir) / f"rank{rank}.npz", x=x, v=v, ids=ids)
        elif case == "reduce":
            # the adaptive step control's maxima, all-reduced through the
            # library's callback type (called here as the library calls it)
            import ctypes
            from mercuda_b200.shards import step_reduce
            cb = step_reduce(ranks)
            vals = (ctypes.c_double * 4)(float(rank), -float(rank), float("inf") if rank == 1 else 0.0, 5.0)
            cb(vals, 4, None)
            np.savez(Path(out_dir) / f"rank{rank}.npz", vals=np.array(list(vals)))
        elif case == "mismatch":
            s = system()
            shard, ids = particle_shard(s, rank, world)
            run = ShardedRun(ranks, OracleBackend(O))
            try:
                run.upload(shard, ids, s.n + rank)   # rank 1 claims another body count
                raised = False
            except ValueError:
                raised = True
            np.savez(Path(out_dir) / f"rank{rank}.npz", raised=raised)
    finally:
        dist.destroy_process_group()


def launch(tmp_path, case, world=2):
    port = free_port()
    mp.start_processes(worker, args=(world, port, str(tmp_path), case), nprocs=world, join=True,
                       start_method="spawn")
    return [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]


def test_sharded_run_equals_unsharded(tmp_path, oracle):
    r0, r1 = launch(tmp_path, "run")
    s = system()
    ref = s.copy()
    rev, rst = oracle.mvs_run(ref, 0.0, H, NSTEPS, RCEN, central=True, threads=1)
    assert len(rev) > 0 and np.any(np.maximum(rev["i"], rev["j"]) > s.nbig)
    assert np.array_equal(r0["x"], ref.x) and np.array_equal(r0["v"], ref.v)
    a, ast = canonical(r0["ev"], r0["st"])
    b, bst = canonical(rev, rst)
    assert np.array_equal(ast, bst)
    assert a.tobytes() == b.tobytes()
    # rank order of the records: by step, then by pair
    lo = np.minimum(r0["ev"]["i"], r0["ev"]["j"])
    key = r0["st"].astype(np.int64) * (1 << 40) + lo
    assert np.all(np.diff(key) >= 0)
    # slowest rank's time, whole-job throughput, each rank's own shard
    assert float(r0["t"]) == 2.0 and float(r1["t"]) == 2.0
    assert float(r0["value"]) == 100.0
    npart = s.n - s.nbig
    assert int(r0["own_n"]) == s.nbig + (npart + 1) // 2 and int(r1["own_n"]) == s.nbig + npart // 2


def test_sharded_one_call_run_equals_unsharded(tmp_path, oracle):
    """ShardedRun.run (one upload + run + download call per rank, as the
    bench's end-to-end leg makes it): rank 0's records are the whole
    system's, every rank's own states are its shard's rows of an unsharded
    run."""
    r0, r1 = launch(tmp_path, "onecall")
    s = system()
    ref = s.copy()
    rev, rst = oracle.mvs_run(ref, 0.0, H, NSTEPS, RCEN, central=True, threads=1)
    a, ast = canonical(r0["ev"], r0["st"])
    b, bst = canonical(rev, rst)
    assert np.array_equal(ast, bst) and a.tobytes() == b.tobytes()
    for r in (r0, r1):
        ids = r["ids"]
        assert np.array_equal(r["x"], ref.x[ids]) and np.array_equal(r["v"], ref.v[ids])


def test_step_reduce_takes_the_maximum_over_ranks(tmp_path):
    r0, r1 = launch(tmp_path, "reduce")
    want = [1.0, 0.0, float("inf"), 5.0]
    assert list(r0["vals"]) == want and list(r1["vals"]) == want


def test_ranks_that_disagree_fail_together(tmp_path):
    r0, r1 = launch(tmp_path, "mismatch")
    assert bool(r0["raised"]) and bool(r1["raised"])


def test_particle_shards_partition_the_system():
    from mercuda_b200.shards import particle_shard
    s = system()
    world = 3
    seen = []
    for r in range(world):
        shard, ids = particle_shard(s, r, world)
        assert shard.nbig == s.nbig and np.array_equal(ids[:s.nbig], np.arange(s.nbig))
        assert np.array_equal(shard.x, s.x[ids]) and np.array_equal(shard.rce, s.rce[ids])
        seen.append(ids[s.nbig:])
    allp = np.sort(np.concatenate(seen))
    assert np.array_equal(allp, np.arange(s.nbig, s.n))
    with pytest.raises(ValueError):
        particle_shard(s, world, world)


def test_rank_workloads_share_their_planets():
    """Per-rank particle draws keep the planets of the job's seed."""
    from mercuda_b200.system import make_system
    a = make_system(seed=1, n_particles=50, particle_seed=(1, 1))
    b = make_system(seed=1, n_particles=50, particle_seed=(1, 2))
    c = make_system(seed=1, n_particles=50)
    assert np.array_equal(a.x[:a.nbig], b.x[:b.nbig]) and np.array_equal(a.x[:a.nbig], c.x[:c.nbig])
    assert not np.array_equal(a.x[a.nbig:], b.x[b.nbig:])
