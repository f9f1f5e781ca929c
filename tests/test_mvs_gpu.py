"""GPU parity of the MVS path against the CPU oracle, through the C ABI.

Gates (from the path's contract): positions and velocities within 1e-12
relative of the oracle after one step; identical encounter and impact lists
(ids, kinds, order); multi-step runs within the stated drift. With
--fmad=false the kernels round every statement as the oracle does, so most
bodies agree bit for bit; the remainder differ only through CUDA's cos/pow in
the Kepler solver's seed (a few ulp)."""
import numpy as np
import pytest

from mercuda_b200.backend import Backend
from mercuda_b200.system import K2, System, make_system

pytestmark = pytest.mark.gpu

REL_ONE_STEP = 1e-12


def rel_err(a, b):
    scale = np.maximum(np.linalg.norm(b, axis=1, keepdims=True), 1e-300)
    return np.max(np.abs(a - b) / scale) if len(a) else 0.0


def event_key(ev):
    return [(int(e["i"]), int(e["j"]), int(e["kind"]), int(e["now"])) for e in ev]


def assert_events_equal(got, want, tol=1e-9):
    assert event_key(got) == event_key(want)
    for g, w in zip(got, want):
        assert abs(g["time"] - w["time"]) <= tol * max(1.0, abs(w["time"]))
        assert abs(g["distance"] - w["distance"]) <= tol * max(1e-12, abs(w["distance"]))
        if w["kind"] & 1:
            assert np.max(np.abs(g["xi"] - w["xi"])) <= tol * max(1.0, np.max(np.abs(w["xi"])))
            assert np.max(np.abs(g["xj"] - w["xj"])) <= tol * max(1.0, np.max(np.abs(w["xj"])))
        if w["kind"] == 8:
            # central-body records carry no states (value-initialised in the reference)
            assert not np.any(g["xi"]) and not np.any(g["xj"]) and g["now"] == 0


def oracle_events_one_step(oracle, sys0, h, rcen, time=0.0):
    """Oracle's records for one step, in the ABI's sorted order."""
    s = sys0.copy()
    ev, steps = oracle.mvs_run(s, time, h, 1, rcen, central=True, threads=4)
    return s, ev


@pytest.fixture()
def backend(cuda_lib):
    b = Backend("MVS", lib=cuda_lib)
    b.configure()
    yield b
    b.free()


@pytest.mark.parametrize("count", [0, 1, 31, 32, 33, 255, 256, 257, 1999, 2000, 2001, 4095, 4096, 4097])
def test_one_step_parity_block_boundaries(backend, oracle, count):
    sys0 = make_system(seed=11 + count, n_particles=count, near_fraction=0.05)
    backend.upload(sys0)
    backend.step(0.0, 8.0, dtflag=0)
    x, v = backend.download()
    ev = backend.events(8.0, 8.0, 0.005)
    ref, rev = oracle_events_one_step(oracle, sys0, 8.0, 0.005)
    assert rel_err(x, ref.x) <= REL_ONE_STEP
    assert rel_err(v, ref.v) <= REL_ONE_STEP
    assert_events_equal(ev, rev)


def test_one_step_bitwise_share(backend, oracle):
    """Most particles take drift_kepmd (no transcendental): those are bit-exact."""
    sys0 = make_system(seed=3, n_particles=20000)
    backend.upload(sys0)
    backend.step(0.0, 8.0, dtflag=0)
    x, v = backend.download()
    ref, _ = oracle_events_one_step(oracle, sys0, 8.0, 0.005)
    same = np.all(x == ref.x, axis=1) & np.all(v == ref.v, axis=1)
    assert same.mean() > 0.95
    assert rel_err(x, ref.x) <= REL_ONE_STEP


def test_per_step_loop_matches_oracle_run(backend, oracle):
    """mal_hcon-style loop: step + events each step for 46 steps of 8 d (365 d)."""
    sys0 = make_system(seed=1, n_particles=3000, near_fraction=0.02)
    backend.upload(sys0)
    got = []
    time = 0.0
    for k in range(46):
        backend.step(time, 8.0, dtflag=0 if k == 0 else 2)
        ev = backend.events(time + 8.0, 8.0, 0.005)
        got.extend((k, e) for e in ev)
        time += 8.0
    x, v = backend.download()
    ref = sys0.copy()
    rev, rsteps = oracle.mvs_run(ref, 0.0, 8.0, 46, 0.005, central=True, threads=8)
    # stated drift after 365 d: 1e-9 relative (ulp differences amplified by close encounters)
    assert rel_err(x, ref.x) < 1e-9
    assert [(k, int(e["i"]), int(e["j"]), int(e["kind"])) for k, e in got] == \
        [(int(s), int(e["i"]), int(e["j"]), int(e["kind"])) for s, e in zip(rsteps, rev)]


@pytest.mark.parametrize("spl", [1, 7, 0])
def test_fused_advance_matches_oracle(backend, oracle, spl):
    sys0 = make_system(seed=2, n_particles=5000, near_fraction=0.02)
    backend.upload(sys0)
    ev, steps = backend.mvs_advance(0.0, 8.0, 46, 0.005, steps_per_launch=spl)
    x, v = backend.download()
    ref = sys0.copy()
    rev, rsteps = oracle.mvs_run(ref, 0.0, 8.0, 46, 0.005, central=True, threads=8)
    assert rel_err(x, ref.x) < 1e-9
    assert np.array_equal(steps, rsteps)
    assert_events_equal(ev, rev, tol=1e-7)


@pytest.mark.parametrize("speed", [0.7, 1.0, 1.2])
def test_kepler_regimes_no_big_bodies(backend, oracle, speed):
    """The reference's Kepler-regime case: one massless body, no Big bodies."""
    m = np.array([K2, 0.0])
    x = np.array([[0, 0, 0], [0.5, 0, 0]], dtype=float)
    v = np.array([[0, 0, 0], [0, speed * np.sqrt(2 * K2 / 0.5), 0]], dtype=float)
    sys0 = System(m=m, x=x, v=v, nbig=1)
    backend.upload(sys0)
    ev, _ = backend.mvs_advance(0.0, 0.5, 64, 0.005)
    gx, gv = backend.download()
    ref = sys0.copy()
    oracle.mvs_run(ref, 0.0, 0.5, 64, 0.005, threads=1)
    assert rel_err(gx, ref.x) <= 1e-12 and rel_err(gv, ref.v) <= 1e-12


def test_yarkovsky_and_cometary_terms(backend, oracle):
    """MVS with non-gravitational terms (mfo_ngf in the kick, ngflag 1)."""
    sys0 = make_system(seed=9, n_particles=700)
    rng = np.random.default_rng(9)
    sys0.ngf[sys0.nbig:, 4] = rng.uniform(1e-15, 1e-13, sys0.n - sys0.nbig) * rng.choice([-1, 1], sys0.n - sys0.nbig)
    sys0.ngf[sys0.nbig::3, 0] = 1e-9
    sys0.ngf[sys0.nbig::5, 2] = 1e-9
    backend.upload(sys0)
    ev, _ = backend.mvs_advance(0.0, 8.0, 16, 0.005)
    x, v = backend.download()
    ref = sys0.copy()
    oracle.mvs_run(ref, 0.0, 8.0, 16, 0.005, threads=4)
    assert rel_err(x, ref.x) < 1e-11 and rel_err(v, ref.v) < 1e-11


def test_oblateness(backend, oracle):
    sys0 = make_system(seed=10, n_particles=500)
    sys0.jcen = np.array([1e-7, -1e-10, 1e-13])
    backend.upload(sys0)
    backend.mvs_advance(0.0, 8.0, 10, 0.005)
    x, v = backend.download()
    ref = sys0.copy()
    oracle.mvs_run(ref, 0.0, 8.0, 10, 0.005, threads=1)
    assert rel_err(x, ref.x) < 1e-11


def test_backwards_integration(backend, oracle):
    sys0 = make_system(seed=12, n_particles=800, near_fraction=0.05)
    backend.upload(sys0)
    ev, steps = backend.mvs_advance(0.0, -8.0, 20, 0.005)
    x, _ = backend.download()
    ref = sys0.copy()
    rev, rsteps = oracle.mvs_run(ref, 0.0, -8.0, 20, 0.005, threads=4)
    assert rel_err(x, ref.x) < 1e-10
    assert event_key(ev) == event_key(rev)


def test_event_buffer_growth(backend, oracle):
    """More simultaneous encounter records than the initial buffer (4,096):
    the step is redone with a larger buffer and nothing is dropped."""
    sys0 = make_system(seed=4, n_particles=20000, near_fraction=1.0, planet_kw=dict(mmin=1e-3, mmax=1e-3))
    sys0.rce[1:sys0.nbig] *= 20.0
    backend.upload(sys0)
    backend.step(0.0, 8.0, dtflag=0)
    ev = backend.events(8.0, 8.0, 0.005)
    _, rev = oracle_events_one_step(oracle, sys0, 8.0, 0.005)
    assert len(rev) > 4096
    assert event_key(ev) == event_key(rev)


def test_previous_state_download(backend):
    sys0 = make_system(seed=13, n_particles=100)
    backend.upload(sys0)
    backend.step(0.0, 8.0, dtflag=0)
    x0, v0 = backend.download(previous=True)
    assert np.array_equal(x0, sys0.x) and np.array_equal(v0, sys0.v)


def test_step_failure_is_reported(backend):
    """A body at the central body's position gives a non-finite force: the step
    must fail loudly (the bridge turns it into 'CUDA integration step failed')."""
    sys0 = make_system(seed=14, n_particles=10)
    sys0.x[sys0.nbig + 3] = sys0.x[2]   # on top of a Big body: division by zero
    backend.upload(sys0)
    with pytest.raises(Exception, match="CUDA integration step failed"):
        backend.step(0.0, 8.0, dtflag=0)


def test_per_step_loop_long_run_with_reordering(backend, oracle):
    """100 drop-in steps: the slot order is rebuilt every 32 steps (and the
    per-step previous/central buffers must follow it)."""
    sys0 = make_system(seed=15, n_particles=1500, near_fraction=0.05)
    backend.upload(sys0)
    time, got = 0.0, []
    for k in range(100):
        backend.step(time, 8.0, dtflag=0 if k == 0 else 2)
        x0, v0 = backend.download(previous=True)
        ev = backend.events(time + 8.0, 8.0, 0.005)
        got.extend((k, int(e["i"]), int(e["j"]), int(e["kind"])) for e in ev)
        time += 8.0
    x, v = backend.download()
    ref = sys0.copy()
    rev, rsteps = oracle.mvs_run(ref, 0.0, 8.0, 100, 0.005, central=True, threads=4)
    assert rel_err(x, ref.x) < 1e-9
    assert got == [(int(s), int(e["i"]), int(e["j"]), int(e["kind"])) for s, e in zip(rsteps, rev)]
    prev = sys0.copy()
    oracle.mvs_run(prev, 0.0, 8.0, 99, 0.005, central=False, threads=4)
    assert rel_err(x0, prev.x) < 1e-9


def test_per_step_loop_with_changes_between_steps(backend, oracle):
    """Per-step calls whose step size and central radius change between steps,
    with other calls in between (previous-state download, export, force): the
    next step, made ahead of the call while the host handles the records,
    must be taken only when it was made for that call. Every step's records
    and the final states match the oracle stepping the same sequence."""
    sys0 = make_system(seed=21, n_particles=2500, near_fraction=0.05)
    backend.upload(sys0)
    ref = sys0.copy()
    plan = [(8.0, 0.005)] * 5 + [(4.0, 0.005)] * 3 + [(8.0, 0.01)] * 4 + [(-8.0, 0.01)] * 2 + [(8.0, 0.005)] * 6
    time = 0.0
    for k, (h, rc) in enumerate(plan):
        backend.step(time, h, dtflag=0 if k == 0 else 2)
        if k % 4 == 1:
            backend.download(previous=True)
        if k == 9:
            backend.force()
        if k == 15:
            backend.export(h)
        ev = backend.events(time + h, h, rc)
        rev, _ = oracle.mvs_run(ref, time, h, 1, rc, central=True, threads=4)
        assert event_key(ev) == event_key(rev), k
        time += h
    x, v = backend.download()
    assert rel_err(x, ref.x) < 1e-9 and rel_err(v, ref.v) < 1e-9


def test_per_step_loop_many_records(backend, oracle):
    """Consecutive steps with more records than are read back with the status
    (1,024): the rest come from the device, every step."""
    sys0 = make_system(seed=4, n_particles=12000, near_fraction=1.0, planet_kw=dict(mmin=1e-3, mmax=1e-3))
    sys0.rce[1:sys0.nbig] *= 20.0
    backend.upload(sys0)
    ref = sys0.copy()
    time, counts = 0.0, []
    for k in range(4):
        backend.step(time, 8.0, dtflag=0 if k == 0 else 2)
        ev = backend.events(time + 8.0, 8.0, 0.005)
        rev, _ = oracle.mvs_run(ref, time, 8.0, 1, 0.005, central=True, threads=4)
        assert event_key(ev) == event_key(rev), k
        counts.append(len(ev))
        time += 8.0
    assert min(counts) > 1024


@pytest.mark.parametrize("oblate", [False, True])
def test_massive_small_bodies(backend, oracle, oblate):
    """Semi-active Small bodies under MVS, which the reference accepts
    (mercury_cuda.cu:400-401): they move as test particles and, with the
    central body's oblateness, enter the reaction term acen that every body
    feels (mfo_mvs, mercury6_2.for:5061-5068). One step at 1e-12, then a
    fused run and per-step drop-in calls against the oracle."""
    from adaptive_cases import hvar_system
    sys0 = hvar_system(massive=True, pn=0)
    if oblate:
        sys0.jcen[:] = [0.1, -1e-3, 0.0]
    assert np.count_nonzero(sys0.m[sys0.nbig:]) > 5
    backend.upload(sys0)
    backend.step(0.0, 0.5, dtflag=0)
    x, v = backend.download()
    ev = backend.events(0.5, 0.5, 0.005)
    ref, rev = oracle_events_one_step(oracle, sys0, 0.5, 0.005)
    assert rel_err(x, ref.x) <= REL_ONE_STEP and rel_err(v, ref.v) <= REL_ONE_STEP
    assert event_key(ev) == event_key(rev)
    # fused run from the start
    backend.upload(sys0)
    ev, steps = backend.mvs_advance(0.0, 0.5, 128, 0.005)
    x, v = backend.download()
    xe, ve = backend.export(0.5, physical=True)
    ref = sys0.copy()
    rev, rsteps = oracle.mvs_run(ref, 0.0, 0.5, 128, 0.005, central=True, threads=1)
    assert rel_err(x, ref.x) < 1e-11 and rel_err(v, ref.v) < 1e-11
    assert np.array_equal(steps, rsteps) and event_key(ev) == event_key(rev)
    want_x, want_v = oracle.mvs_corrector(ref, 0.5, forward=True)
    assert np.max(np.abs(xe - want_x)) < 1e-12 and np.max(np.abs(ve - want_v)) < 1e-12


def test_massive_small_bodies_particles_and_oblateness(backend, oracle):
    """A workload-sized system with a few massive Small bodies among massless
    ones and central-body oblateness: the massive ones ride in the Big-body
    CTA, the rest in particle slots, with event ids mapped through both."""
    sys0 = make_system(seed=31, n_particles=3000, near_fraction=0.03)
    sys0.m[sys0.nbig:sys0.nbig + 40:4] = 1e-9 * K2
    sys0.jcen[:] = [1e-6, -1e-9, 0.0]
    backend.upload(sys0)
    got, t = [], 0.0
    for k in range(12):
        backend.step(t, 8.0, dtflag=0 if k == 0 else 2)
        got.extend((k, int(e["i"]), int(e["j"]), int(e["kind"])) for e in backend.events(t + 8.0, 8.0, 0.005))
        t += 8.0
    x, v = backend.download()
    ref = sys0.copy()
    rev, rsteps = oracle.mvs_run(ref, 0.0, 8.0, 12, 0.005, central=True, threads=1)
    assert rel_err(x, ref.x) < 1e-11 and rel_err(v, ref.v) < 1e-11
    assert got == [(int(s), int(e["i"]), int(e["j"]), int(e["kind"])) for s, e in zip(rsteps, rev)]
    e0, l0 = backend.energy(8.0, physical=True)
    assert np.isfinite(e0) and np.isfinite(l0)


def test_fused_run_launch_schedule(backend):
    """The automatic launch choice makes a short first launch (so that the
    next launch's Big-body steps run beside its particles) and re-sorts the
    slots only after 16 steps: the records and states equal those of one
    launch of all the steps, and the launches are reported."""
    sys0 = make_system(seed=22, n_particles=20000, near_fraction=0.05)
    backend.upload(sys0)
    ev_a, st_a = backend.mvs_advance(0.0, 8.0, 20, 0.005)
    launches = backend.advance_launches()
    assert [k for k, _ in launches] == [4, 16] and all(ms > 0.0 for _, ms in launches)
    xa, va = backend.download()
    backend.upload(sys0)
    ev_b, st_b = backend.mvs_advance(0.0, 8.0, 20, 0.005, steps_per_launch=20)
    assert [k for k, _ in backend.advance_launches()] == [20]
    xb, vb = backend.download()
    assert ev_a.tobytes() == ev_b.tobytes() and np.array_equal(st_a, st_b)
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
