"""The one-call MVS run (mercury_b200_mvs_run) against the three calls it
stands for (upload, fused advance, download): with page-locked host arrays
the particles are copied, ordered and stepped in chunks, and the results
must be the same bit for bit; with pageable arrays the three calls are made
in turn. The fused advance itself is checked against the oracle elsewhere."""
import numpy as np
import pytest
import torch

from mercuda_b200.backend import Backend
from mercuda_b200.system import make_system

pytestmark = pytest.mark.gpu

_KEEP = []


def pinned(a):
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    _KEEP.append(t)
    out = t.numpy()
    out[...] = a
    return out


def pinned_system(s):
    p = s.copy()
    for name in ("m", "x", "v", "ngf", "rce", "rphys", "rcrit"):
        setattr(p, name, pinned(getattr(s, name)))
    return p


@pytest.fixture()
def backend(cuda_lib):
    b = Backend("MVS", lib=cuda_lib)
    b.configure()
    yield b
    b.free()


def three_calls(b, s, nsteps, h, rcen):
    b.upload(s)
    ev, st = b.mvs_advance(0.0, h, nsteps, rcen)
    x, v = b.download()
    return ev, st, x, v


@pytest.mark.parametrize("particles,pin", [(300_001, True), (600_000, True), (150_000, False)])
def test_run_matches_upload_advance_download(backend, particles, pin):
    sys0 = make_system(seed=31, n_particles=particles, near_fraction=0.02)
    ev0, st0, x0, v0 = three_calls(backend, sys0, 12, 8.0, 0.005)
    s = pinned_system(sys0) if pin else sys0
    out = (pinned(np.zeros((s.n, 3))), pinned(np.zeros((s.n, 3)))) if pin else None
    ev, st, x, v = backend.mvs_run(s, 0.0, 8.0, 12, 0.005, out=out)
    assert len(ev0) > 100
    assert ev.tobytes() == ev0.tobytes() and np.array_equal(st, st0)
    assert np.array_equal(x, x0) and np.array_equal(v, v0)
    # the system stays uploaded in its end state: the next run continues it
    ev1, _ = backend.mvs_advance(96.0, 8.0, 3, 0.005)
    xa, _ = backend.download()
    three_calls(backend, sys0, 12, 8.0, 0.005)
    ev2, _ = backend.mvs_advance(96.0, 8.0, 3, 0.005)
    xb, _ = backend.download()
    assert ev1.tobytes() == ev2.tobytes() and np.array_equal(xa, xb)


def test_run_with_nongravitational_forces_and_oblateness(backend):
    sys0 = make_system(seed=32, n_particles=300_000, near_fraction=0.02)
    rng = np.random.default_rng(5)
    nb = sys0.nbig
    sys0.ngf[nb:, 4] = rng.uniform(-1e-13, 1e-13, sys0.n - nb)
    sys0.jcen[:] = [1e-6, -1e-8, 0.0]
    ev0, st0, x0, v0 = three_calls(backend, sys0, 5, 8.0, 0.005)
    s = pinned_system(sys0)
    out = (pinned(np.zeros((s.n, 3))), pinned(np.zeros((s.n, 3))))
    ev, st, x, v = backend.mvs_run(s, 0.0, 8.0, 5, 0.005, out=out)
    assert ev.tobytes() == ev0.tobytes() and np.array_equal(st, st0)
    assert np.array_equal(x, x0) and np.array_equal(v, v0)


def test_run_event_buffer_overflow_is_redone(backend, cuda_lib):
    """More records than the first guess of the buffer: the run is made again
    from the uploaded states with room, and nothing is dropped."""
    sys0 = make_system(seed=4, n_particles=300_000, near_fraction=0.05, planet_kw=dict(mmin=1e-3, mmax=1e-3))
    ev0, st0, x0, v0 = three_calls(backend, sys0, 2, 8.0, 0.005)
    s = pinned_system(sys0)
    out = (pinned(np.zeros((s.n, 3))), pinned(np.zeros((s.n, 3))))
    cuda_lib.mercury_b200_set_event_capacity(1024)
    try:
        ev, st, x, v = backend.mvs_run(s, 0.0, 8.0, 2, 0.005, out=out)
    finally:
        cuda_lib.mercury_b200_set_event_capacity(0)
    assert len(ev0) > 1024
    assert ev.tobytes() == ev0.tobytes() and np.array_equal(st, st0)
    assert np.array_equal(x, x0) and np.array_equal(v, v0)


def test_run_with_massive_small_bodies(backend):
    """Massive Small bodies move the split between the Big-body CTA and the
    particle slots (with oblateness they enter its reaction term): the run
    makes the three calls in turn, with the same results."""
    sys0 = make_system(seed=33, n_particles=300_000, near_fraction=0.02)
    nb = sys0.nbig
    sys0.m[nb:nb + 7] = 1e-12
    sys0.jcen[:] = [1e-6, 0.0, 0.0]
    ev0, st0, x0, v0 = three_calls(backend, sys0, 4, 8.0, 0.005)
    s = pinned_system(sys0)
    out = (pinned(np.zeros((s.n, 3))), pinned(np.zeros((s.n, 3))))
    ev, st, x, v = backend.mvs_run(s, 0.0, 8.0, 4, 0.005, out=out)
    assert ev.tobytes() == ev0.tobytes() and np.array_equal(st, st0)
    assert np.array_equal(x, x0) and np.array_equal(v, v0)
