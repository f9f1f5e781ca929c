"""HYBRID (mdt_hy) through the drop-in C ABI on the GPU against the oracle:
mercury_cuda_hybrid_begin / _finish for the resident system and, for the
encounter members, mercury_cuda_encounter_enter / _step / _download / _events
/ _exit driven as mdt_hkce drives them (mercury6_2.for:3798-3940). Restates the
reference's tests/test_gpu_algorithms.py:34-41 (HYBRID with and without
semi-active bodies, both directions, a close Big pair that forces the BS2
path, no Big bodies at all). Only the Kepler solver's cos/sin differ from the
host's libm, so states are compared at the reference's 1e-10 parity bar with
most coordinates bit-identical, and encounter records by ids and kinds."""
import math

import numpy as np
import pytest

from adaptive_cases import hvar_system, planar_body
from mercuda_b200.backend import Backend
from mercuda_b200.system import K2, System, make_system, mce_init

pytestmark = pytest.mark.gpu


def run_device(cuda_lib, sys, h, nsteps, tol=1e-12, rcen=0.005, fused=True):
    be = Backend("HYBRID", cuda_lib)
    be.configure()
    be.upload(sys)
    state = {"dtflag": 0}
    events, pairs, t = [], 0, 0.0
    for _ in range(nsteps):
        ev, npair = be.hybrid_step(sys, t, h, tol, state, rcen, fused=fused)
        pairs += npair
        t = t + h
        events.append(ev)
        events.append(be.events(t, h, rcen))
    x, v = be.download()
    xp, vp = be.export(h, physical=True)
    forces = be.forces
    be.free()
    ev = np.concatenate(events) if events else np.zeros(0)
    return x, v, xp, vp, ev, pairs, forces


def compare(sys, got, ref_sys, want, bound=1e-10):
    x, v, xp, vp, ev, pairs, forces = got
    want_ev, _, want_forces, want_pairs = want
    assert pairs == want_pairs
    assert forces == want_forces
    dx = np.max(np.abs(x - ref_sys.x))
    dv = np.max(np.abs(v - ref_sys.v))
    assert dx < bound and dv < bound, (dx, dv)
    same = np.mean(np.all(x == ref_sys.x, axis=1) & np.all(v == ref_sys.v, axis=1))
    assert same > 0.5, same
    key = lambda e: (min(e["i"], e["j"]), max(e["i"], e["j"]), int(e["kind"]))
    assert sorted(map(key, ev)) == sorted(map(key, want_ev))


def hybrid_case(massive, count=33):
    sys = hvar_system(massive=massive, pn=0, count=count)
    return mce_init(sys, 0.5, 3.0)


@pytest.mark.parametrize("massive", [False, True])
@pytest.mark.parametrize("direction", [-1, 1])
def test_hybrid_semi_active(cuda_lib, oracle, massive, direction):
    sys = hybrid_case(massive)
    ref = sys.copy()
    h = 0.5 * direction
    got = run_device(cuda_lib, sys, h, 60)
    want = oracle.hy_run(ref, 0.0, h, 60)
    compare(sys, got, ref, want)


def test_hybrid_close_big_pair(cuda_lib, oracle):
    """Overlapping Hill spheres: the two planets are encounter members every step."""
    bodies = [(K2, [0.0] * 3, [0.0] * 3), planar_body(1e-5, 1.0, 0.0, 0.0), planar_body(1e-5, 1.02, 0.0, 0.02)]
    bodies += [planar_body(0.0, 1.6 + j * 0.012, 0.12, j * 0.37) for j in range(3)]
    sys = System(m=np.array([b[0] for b in bodies]), x=np.array([b[1] for b in bodies]),
                 v=np.array([b[2] for b in bodies]), nbig=3, rce=np.full(6, 0.01), rphys=np.full(6, 1e-5))
    sys = mce_init(sys, 0.5, 3.0)
    ref = sys.copy()
    got = run_device(cuda_lib, sys, 0.5, 16)
    want = oracle.hy_run(ref, 0.0, 0.5, 16)
    assert want[3] > 0
    compare(sys, got, ref, want)


@pytest.mark.parametrize("count", [0, 1, 257])
def test_hybrid_without_big_bodies(cuda_lib, oracle, count):
    bodies = [(K2, [0.0] * 3, [0.0] * 3)] + [planar_body(0.0, 1.6 + j * 0.012, 0.12, j * 0.37) for j in range(count)]
    sys = System(m=np.array([b[0] for b in bodies]), x=np.array([b[1] for b in bodies]).reshape(-1, 3),
                 v=np.array([b[2] for b in bodies]).reshape(-1, 3), nbig=1)
    sys = mce_init(sys, 0.5, 3.0)
    ref = sys.copy()
    got = run_device(cuda_lib, sys, 0.5, 32)
    want = oracle.hy_run(ref, 0.0, 0.5, 32)
    compare(sys, got, ref, want)


def test_hybrid_particles_and_encounters(cuda_lib, oracle):
    """Thousands of massless particles, 5% near the planets: many encounter
    pairs per step go through the BS2 subsystem."""
    sys = make_system(seed=3, n_particles=2000, nplanets=8, near_fraction=0.05, h=8.0)
    ref = sys.copy()
    got = run_device(cuda_lib, sys, 8.0, 12)
    want = oracle.hy_run(ref, 0.0, 8.0, 12)
    assert want[3] > 20
    compare(sys, got, ref, want, bound=1e-9)
    x, v, xp, vp = got[:4]
    vh = np.zeros_like(v)
    mv = (sys.m[1:, None] * v[1:]).sum(axis=0) / sys.m[0]
    vh[1:] = v[1:] + mv
    assert np.allclose(xp, x) and np.max(np.abs(vp - vh)) < 1e-15


def test_encounter_loop_in_library_matches_drop_in_calls(cuda_lib):
    """mercury_b200_encounter_run makes the drop-in calls of mdt_hkce's host
    loop inside the library: the same states, records, pairs and force calls
    as driving them one at a time."""
    sys0 = make_system(seed=4, n_particles=1500, nplanets=8, near_fraction=0.05, h=8.0)
    a = run_device(cuda_lib, sys0.copy(), 8.0, 10, fused=True)
    b = run_device(cuda_lib, sys0.copy(), 8.0, 10, fused=False)
    assert a[5] == b[5] and a[5] > 10 and a[6] == b[6]
    for k in range(4):
        assert np.array_equal(a[k], b[k])
    assert a[4].tobytes() == b[4].tobytes()


def test_encounter_loop_redone_after_buffer_overflow(cuda_lib):
    """With record and candidate buffers of one entry, the library's substep
    loop overflows, grows its buffers and redoes the subsystem's run from its
    starting state (the drop-in calls grow and redo each screen instead): the
    same states, records, pairs and force calls as with the default buffers."""
    sys0 = make_system(seed=4, n_particles=1500, nplanets=8, near_fraction=0.05, h=8.0)
    want = run_device(cuda_lib, sys0.copy(), 8.0, 10, fused=True)
    assert cuda_lib.mercury_b200_set_event_capacity(1) == 0
    try:
        a = run_device(cuda_lib, sys0.copy(), 8.0, 10, fused=True)
        b = run_device(cuda_lib, sys0.copy(), 8.0, 10, fused=False)
    finally:
        cuda_lib.mercury_b200_set_event_capacity(0)
    assert len(want[4]) > 1
    for got in (a, b):
        assert got[5] == want[5] and got[6] == want[6]
        for k in range(4):
            assert np.array_equal(got[k], want[k])
        assert got[4].tobytes() == want[4].tobytes()
