"""Test particles split across ranks (one process per GPU).

Massless test particles act on nothing, so the MVS integration of one system
shards by particle with no data-path exchange: every rank holds the central
body and all Big bodies (integrated redundantly, the same way on every rank)
and its own subset of the particles. The only collective steps are the
barriers around a timed region, the maximum of the ranks' times, and the
gathering of event records and final states at the output boundary — the
host-side equivalent of the reference's per-step event list and download
(mercury_cuda.cu:466-493, the records of mercury_gpu.f90:206-247), now with
global body ids.

The adaptive integrators (RADAU, BS, BS2) shard the same way with one real
exchange: their step control takes the maximum of an error measure over every
body, so each attempt's maxima are all-reduced (MAX) across ranks through the
library's step-reduce hook (`step_reduce`); every rank then takes the same
decisions and its particles follow the whole system's steps bit for bit.

Every rank takes the same collective steps in the same order. The classes are
backend-agnostic: `ShardedRun` drives any object with the `upload`,
`mvs_advance`, `download` methods of `backend.Backend`, and `Ranks` works over
NCCL (CUDA tensors) or gloo (CPU tensors).
"""
from __future__ import annotations

import numpy as np

from .system import System


class Ranks:
    """Rank plumbing over a torch.distributed process group (or one process)."""

    def __init__(self, dist=None, device=None):
        self.dist = dist if dist is not None and dist.is_initialized() else None
        self.world = self.dist.get_world_size() if self.dist else 1
        self.rank = self.dist.get_rank() if self.dist else 0
        if device is None:
            device = "cuda" if self.dist and self.dist.get_backend() == "nccl" else "cpu"
        self.device = device

    def _sync(self):
        if str(self.device).startswith("cuda"):
            import torch
            torch.cuda.synchronize()

    def barrier(self) -> None:
        """Device idle, then all ranks, then device idle again."""
        self._sync()
        if self.dist:
            self.dist.barrier()
        self._sync()

    def max(self, value: float) -> float:
        """The maximum of a per-rank number (a time) over all ranks."""
        if not self.dist:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def gather(self, obj, everywhere: bool = False):
        """Every rank's object in rank order: on rank 0 (None elsewhere), or on
        every rank."""
        if not self.dist:
            return [obj]
        out = [None] * self.world
        if everywhere:
            self.dist.all_gather_object(out, obj)
            return out
        self.dist.gather_object(obj, out if self.rank == 0 else None, dst=0)
        return out if self.rank == 0 else None

    def whole_job(self, units_per_rank: float, seconds: float) -> float:
        """Throughput of the job: all ranks' units over the slowest rank's time."""
        return self.world * units_per_rank / seconds


def particle_shard(sys: System, rank: int, world: int) -> tuple[System, np.ndarray]:
    """The system with all Big bodies and every world-th particle starting at
    `rank`, and the 0-based body indices in `sys` of the shard's bodies."""
    if not 0 <= rank < world:
        raise ValueError("rank outside the world")
    idx = np.concatenate([np.arange(sys.nbig), np.arange(sys.nbig + rank, sys.n, world)])
    take = lambda a: np.ascontiguousarray(a[idx])
    shard = System(m=take(sys.m), x=take(sys.x), v=take(sys.v), nbig=sys.nbig, ngf=take(sys.ngf),
                   jcen=sys.jcen.copy(), rce=take(sys.rce), rphys=take(sys.rphys), rcrit=take(sys.rcrit),
                   rceh=take(sys.rceh), rho=take(sys.rho), pn=sys.pn)
    return shard, idx


def order_events(events: np.ndarray, steps: np.ndarray):
    """Records ordered by step, then by the pair (min(i, j), max(i, j)) as the
    reference sorts one step's list (mercury_cuda.cu:487-490); stable."""
    lo = np.minimum(events["i"], events["j"])
    hi = np.maximum(events["i"], events["j"])
    order = np.lexsort((hi, lo, steps))
    return events[order], steps[order]


class ShardedRun:
    """One rank's share of an MVS integration whose particles are split
    across ranks. `advance` returns the whole system's event records (global
    1-based ids) on rank 0 and None elsewhere; `download` the whole system's
    states on rank 0 (or each rank's own shard with gather=False)."""

    def __init__(self, ranks: Ranks, backend):
        self.ranks = ranks
        self.backend = backend
        self.ids = None
        self.nbig = 0
        self.n = 0
        self.local_events = 0

    def _adopt(self, shard: System, ids: np.ndarray, n_total: int) -> None:
        ids = np.asarray(ids, dtype=np.int64)
        if len(ids) != shard.n or np.any(ids[:shard.nbig] != np.arange(shard.nbig)):
            raise ValueError("a shard holds every Big body first, then its particles")
        self.ids = ids
        self.nbig = shard.nbig
        self.n = int(n_total)
        # every rank must agree on the Big bodies and the total
        seen = self.ranks.gather((self.nbig, self.n), everywhere=True)
        if any(s != seen[0] for s in seen):
            raise ValueError("ranks disagree on the Big bodies or the body count")

    def upload(self, shard: System, ids: np.ndarray, n_total: int, ngflag: int | None = None) -> None:
        """This rank's shard and the global 0-based index of each of its bodies
        (Big bodies first, the same on every rank); n_total bodies in all.
        ngflag: the input's force-law flag (None: derived from shard.ngf)."""
        self._adopt(shard, ids, n_total)
        self.backend.upload(shard, ngflag)

    def run(self, shard: System, ids: np.ndarray, n_total: int, time: float, h: float, nsteps: int, rcen: float,
            steps_per_launch: int = 0, ngflag: int | None = None, out=None):
        """upload + advance + this rank's own states back in one library call
        per rank (Backend.mvs_run: the copies overlap the steps). Returns
        (records as advance returns them, (x, v) of this rank's shard)."""
        self._adopt(shard, ids, n_total)
        events, steps, x, v = self.backend.mvs_run(shard, time, h, nsteps, rcen, steps_per_launch, ngflag, out)
        return self._collect(events, steps), (x, v)

    def _to_global(self, events: np.ndarray) -> np.ndarray:
        """The records with global ids, in place (the array is the backend's
        fresh copy)."""
        for f in ("i", "j"):
            events[f] = self.ids[events[f] - 1] + 1
        return events

    def advance(self, time: float, h: float, nsteps: int, rcen: float, steps_per_launch: int = 0):
        events, steps = self.backend.mvs_advance(time, h, nsteps, rcen, steps_per_launch)
        return self._collect(events, steps)

    def _collect(self, events: np.ndarray, steps: np.ndarray):
        """This rank's records of a run as the whole system's, on rank 0."""
        self.local_events = len(events)   # records read back from this rank's device
        events = self._to_global(events)
        if self.ranks.rank != 0:
            # records among the central and Big bodies are the same on every
            # rank: rank 0 reports them
            particle = np.maximum(events["i"], events["j"]) > self.nbig
            events, steps = events[particle], steps[particle]
        parts = self.ranks.gather((events, steps))
        if parts is None:
            return None
        if len(parts) == 1:
            # the backend's order, which the monotone id map keeps
            return parts[0]
        ev = np.concatenate([p[0] for p in parts])
        st = np.concatenate([p[1] for p in parts])
        return order_events(ev, st)

    def download(self, gather: bool = True, out=None):
        x, v = self.backend.download(out=out) if out is not None else self.backend.download()
        if not gather:
            return x, v
        parts = self.ranks.gather((self.ids, x, v))
        if parts is None:
            return None
        X = np.zeros((self.n, 3))
        V = np.zeros((self.n, 3))
        for ids, xs, vs in parts:
            X[ids] = xs
            V[ids] = vs
        return X, V


def step_reduce(ranks: Ranks):
    """A callback for Backend.set_step_reduce: replaces the library's
    step-control maxima by their maximum over all ranks (all-reduce MAX, on
    the ranks' device). Keep the returned object alive while it is installed."""
    import ctypes

    from .backend import REDUCE_FN

    def reduce(ptr, count, user):
        if ranks.dist is None:
            return
        vals = np.ctypeslib.as_array(ptr, shape=(count,))
        try:
            import torch
            t = torch.tensor(vals, dtype=torch.float64, device=ranks.device)
            ranks.dist.all_reduce(t, op=ranks.dist.ReduceOp.MAX)
            vals[:] = t.cpu().numpy()
        except Exception:  # noqa: BLE001 - an exception cannot cross the C callback
            # a failed exchange must not let this rank decide alone: +inf makes
            # the library fail the step loudly
            vals[:] = np.inf

    return REDUCE_FN(reduce)


def sharded_hybrid_step(backend, ranks: Ranks, shard: System, ids: np.ndarray, time: float, h: float, tol: float,
                        state: dict, rcen: float = 0.005, fused: bool = True):
    """One HYBRID step (mdt_hy, mercury6_2.for:3618-3782) of this rank's shard
    of one system: every Big body and this rank's particles, `ids` the global
    0-based index of each shard body (sorted, Big bodies first).

    mce_snif's pairs of every rank are all-gathered with the members'
    pre-drift states, and every rank integrates the one global encounter
    subsystem that a single process would (the same members, pair list and
    BS2 substeps, so the same results); each rank then takes the end states
    of every Big member and of its own particle members. Returns the
    subsystem's records (global 1-based ids, the same on every rank) and the
    global number of encounter pairs."""
    from .backend import EVENT_DTYPE

    ids = np.asarray(ids, dtype=np.int64)
    n, nbig = shard.n, shard.nbig
    if state.get("dtflag", 0) == 0:
        state["hrec"] = h
    rows = getattr(backend, "_shard_rows", None)
    if rows is None or rows[0].shape[0] != n:
        rows = (np.zeros((n, 3)), np.zeros((n, 3)))
        backend._shard_rows = rows
    x, v = rows
    ce, pi, pj = backend.hybrid_begin(h, shard.rcrit, state.get("dtflag", 0), x, v)
    state["dtflag"] = 2
    local = np.nonzero(ce[1:])[0] + 1 if len(pi) else np.zeros(0, dtype=np.int64)
    mine = (ids[pi - 1] + 1, ids[pj - 1] + 1, ids[local],
            np.column_stack([shard.m[local], x[local], v[local], shard.rcrit[local], shard.rce[local],
                             shard.rphys[local]]) if len(local) else np.zeros((0, 10)))
    parts = ranks.gather(mine, everywhere=True)
    gpi = np.concatenate([p[0] for p in parts]).astype(np.int64)
    gpj = np.concatenate([p[1] for p in parts]).astype(np.int64)
    events = np.zeros(0, dtype=EVENT_DTYPE)
    if len(gpi):
        # the pair list a single process would find: unique, sorted by (i, j)
        pairs = np.unique(np.stack([gpi, gpj], axis=1), axis=0)
        gpi, gpj = pairs[:, 0], pairs[:, 1]
        members, first = np.unique(np.concatenate([p[2] for p in parts]), return_index=True)
        data = np.concatenate([p[3] for p in parts])[first]
        sub = np.concatenate([[0], members])
        central = np.zeros((1, 10))
        central[0, 0] = shard.m[0]
        d = np.concatenate([central, data])
        xbs, vbs, events = backend.encounter_subsystem(sub, nbig, d[:, 0], d[:, 1:4], d[:, 4:7], d[:, 7], d[:, 8],
                                                        d[:, 9], gpi, gpj, time, h, tol, state, rcen, fused)
        # the members this shard holds: every Big member and its own particles
        pos = np.searchsorted(ids, members)
        held = (pos < n) & (ids[np.minimum(pos, n - 1)] == members)
        apply = pos[held]
        x[apply] = xbs[1:][held]
        v[apply] = vbs[1:][held]
        backend.hybrid_members(apply)
    backend.hybrid_finish(h, shard.m, x, v)
    return events, len(gpi)
