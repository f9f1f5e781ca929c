"""Batched MVS systems (mercury_b200_batch_*, an extension with no reference
counterpart): every system of a batch must come out exactly as the drop-in
single-system path integrates it alone (same states and event records, bit
for bit), whatever the launch shape, and close to the oracle."""
import numpy as np
import pytest

from mercuda_b200.backend import Backend, Batch
from mercuda_b200.system import make_batch

pytestmark = pytest.mark.gpu

RCEN = 0.005


def single_runs(cuda_lib, systems, h, nsteps):
    out = []
    for sys, hs in zip(systems, h):
        be = Backend("MVS", cuda_lib)
        be.configure()
        be.upload(sys.copy())
        ev, st = be.mvs_advance(0.0, float(hs), nsteps, RCEN)
        x, v = be.download()
        be.free()
        out.append((x, v, ev, st))
    return out


def canonical(ev, st):
    """Records in a canonical order: by step, then by the record's bytes. Records
    of one step are a set (parallel kernels append them in any order), so two
    logs hold the same events exactly when their canonical forms are equal."""
    order = sorted(range(len(ev)), key=lambda q: (int(st[q]), ev[q].tobytes()))
    order = np.asarray(order, dtype=np.int64)
    return ev[order], st[order]


def first_difference(a, b):
    """The first differing record and the fields it differs in (for messages)."""
    for q in range(min(len(a), len(b))):
        if a[q].tobytes() != b[q].tobytes():
            fields = [f for f in a.dtype.names if np.asarray(a[q][f]).tobytes() != np.asarray(b[q][f]).tobytes()]
            return q, fields, a[q], b[q]
    return None


def check_against(batch_out, events, sy, st, singles):
    for k, ((x, v), (xs, vs, ev, est)) in enumerate(zip(batch_out, singles)):
        assert np.array_equal(x, xs) and np.array_equal(v, vs), (k, np.max(np.abs(x - xs)))
        mine, mst = canonical(events[sy == k], st[sy == k])
        ref, rst = canonical(ev, est)
        assert np.array_equal(mst, rst), k
        assert mine.tobytes() == ref.tobytes(), (k, first_difference(mine, ref))


@pytest.mark.parametrize("shape", [dict(), dict(steps_per_launch=7, graph=0, threads=64)])
def test_batch_matches_single_system_path(cuda_lib, shape):
    systems, h = make_batch(seed=7, nsys=24, nmin=10, nmax=400, near_fraction=0.05)
    nsteps = 40
    b = Batch(systems, h, cuda_lib)
    if shape:
        b.set(threads=shape["threads"], steps_per_launch=shape["steps_per_launch"], graph=shape["graph"])
    ev, sy, st = b.advance(0.0, nsteps, RCEN)
    out = b.download()
    b.set(threads=0, steps_per_launch=0, graph=1)
    b.free()
    assert len(ev) > 0
    check_against(out, ev, sy, st, single_runs(cuda_lib, systems, h, nsteps))


def test_batch_two_advances_and_event_growth(cuda_lib):
    """Two advances in a row (the second replays the captured graph) and
    more event records than the initial buffer holds."""
    systems, h = make_batch(seed=3, nsys=48, nmin=300, nmax=800, near_fraction=0.9)
    b = Batch(systems, h, cuda_lib)
    ev1, sy1, st1 = b.advance(0.0, 40, RCEN)
    ev2, sy2, st2 = b.advance(0.0, 40, RCEN)
    out = b.download()
    b.free()
    assert len(ev1) > 4096
    singles = single_runs(cuda_lib, systems, h, 80)
    for k, ((x, v), (xs, vs, ev, est)) in enumerate(zip(out, singles)):
        assert np.array_equal(x, xs) and np.array_equal(v, vs), k
        first = est < 40
        a, ast = canonical(ev1[sy1 == k], st1[sy1 == k])
        b_, bst = canonical(ev[first], est[first])
        assert np.array_equal(ast, bst), (k, len(a), len(b_))
        assert a.tobytes() == b_.tobytes(), (k, first_difference(a, b_))
        # the second advance restarts the clock at its own time argument
        c, cst = canonical(ev2[sy2 == k], st2[sy2 == k] + 40)
        d, dst = canonical(ev[~first], est[~first])
        assert np.array_equal(cst, dst), k
        assert np.array_equal(c[["i", "j", "kind", "now"]], d[["i", "j", "kind", "now"]]), k


def test_batch_against_oracle(cuda_lib, oracle):
    systems, h = make_batch(seed=11, nsys=6, nmin=50, nmax=300, near_fraction=0.05)
    b = Batch(systems, h, cuda_lib)
    ev, sy, st = b.advance(0.0, 25, RCEN)
    out = b.download()
    b.free()
    for k, (sys, hs) in enumerate(zip(systems, h)):
        ref = sys.copy()
        oev, ost = oracle.mvs_run(ref, 0.0, float(hs), 25, RCEN)
        x, v = out[k]
        scale = np.maximum(np.abs(ref.x), 1e-3)
        assert np.max(np.abs(x - ref.x) / scale) < 1e-11
        mine = ev[sy == k]
        key = lambda e: (min(e["i"], e["j"]), max(e["i"], e["j"]), int(e["kind"]))
        assert sorted(map(key, mine)) == sorted(map(key, oev))
