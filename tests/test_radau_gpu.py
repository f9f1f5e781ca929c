"""RA15 (mdt_ra15) and the heliocentric force (mfo_all) through the drop-in C
ABI on the GPU, checked against the oracle.

The force matrix restates the reference's tests/test_mercury.py:113-133
(semi-active bodies among massless ones, PR mass gating, every ngflag, with
and without 1PN); the integrations restate tests/test_gpu_algorithms.py:89-100
(semi-active Small bodies, both directions, output intervals that clip steps
and restart the RA15 sequence, 1PN with Yarkovsky and radiation pressure).
The GPU and the oracle run the same statements in the same order, so apart
from the cometary law (which calls pow) the results are expected bit for bit;
the reference's own bar, 2e-12 relative for the force, is asserted too.
"""
import numpy as np
import pytest

from adaptive_cases import compare_events, hvar_system, oracle_intervals, run_intervals
from mercuda_b200.backend import Backend, BackendError
from mercuda_b200.system import K2, System, make_system

pytestmark = pytest.mark.gpu


def force_matrix_system(pn, flag, n=200, seed=19):
    rng = np.random.default_rng(seed)
    m = np.zeros(n)
    m[:3] = [K2, 3e-6 * K2, 1e-3 * K2]
    m[3::7] = 1e-8 * K2
    x = np.vstack([np.zeros(3), rng.uniform(-4, 4, (n - 1, 3))])
    v = np.vstack([np.zeros(3), rng.uniform(-0.02, 0.02, (n - 1, 3))])
    ngf = np.zeros((n, 5))
    sign = np.array([(-1.0) ** j for j in range(n)])
    if flag & 1:
        ngf[1:, 0] = 1e-12
        ngf[1:, 1] = sign[1:] * 2e-11
        ngf[1:, 2] = 3e-13
        ngf[1:, 4] = sign[1:] * 4e-11
    if flag & 2:
        ngf[1:, 3] = 0.001
    rc = np.full(n, 0.01)
    return System(m=m, x=x, v=v, nbig=3, ngf=ngf, jcen=np.array([1e-7, -1e-10, 1e-13]), rce=rc, rphys=rc.copy(),
                  pn=int(pn))


@pytest.mark.parametrize("pn", [0, 1])
@pytest.mark.parametrize("flag", [0, 1, 2, 3])
def test_force_matrix(cuda_lib, oracle, pn, flag):
    sys = force_matrix_system(pn, flag)
    want = oracle.force(sys)
    be = Backend("RADAU", cuda_lib)
    be.configure()
    be.upload(sys)
    got = be.force()
    be.free()
    assert np.all(got[0] == 0.0)
    rel = np.max(np.abs(got[1:] - want[1:]) / np.maximum(np.abs(want[1:]), 1e-20))
    assert rel < 2e-12, (pn, flag, rel)
    if not flag & 1:  # no pow in the force laws: identical statements, identical bits
        assert np.array_equal(got, want)


@pytest.mark.parametrize("direction", [-1, 1])
@pytest.mark.parametrize("pn", [0, 1])
def test_radau_semi_active(cuda_lib, oracle, direction, pn):
    sys = hvar_system(massive=True, pn=pn)
    ref = sys.copy()
    be = Backend("RADAU", cuda_lib)
    be.configure()
    be.upload(sys)
    ev, h = run_intervals(be, sys, 0.0, direction * 32.0, 7.3, 0.5 * direction, 1e-12)
    x, v = be.download()
    forces = be.forces
    be.free()
    want_ev, want_h, steps, want_forces, _ = oracle_intervals(oracle, ref, 4, 0.0, direction * 32.0, 7.3,
                                                              0.5 * direction, 1e-12)
    assert forces == want_forces
    assert h == want_h
    assert np.array_equal(x, ref.x) and np.array_equal(v, ref.v), (
        np.max(np.abs(x - ref.x)), np.max(np.abs(v - ref.v)))
    compare_events(ev, want_ev)


def test_radau_limits_keep_history(cuda_lib, oracle):
    """mercury_cuda_limits between intervals must not restart the sequence."""
    sys = hvar_system(massive=False, pn=0, count=5)
    a = sys.copy()
    be = Backend("RADAU", cuda_lib)
    be.configure()
    be.upload(a)
    run_intervals(be, a, 0.0, 60.0, 7.3, 0.5, 1e-12, update_limits=True)
    x1, v1 = be.download()
    f1 = be.forces
    be.free()
    b = sys.copy()
    be = Backend("RADAU", cuda_lib)
    be.configure()
    be.upload(b)
    run_intervals(be, b, 0.0, 60.0, 7.3, 0.5, 1e-12)
    x2, v2 = be.download()
    assert be.forces == f1
    be.free()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)


def test_radau_particles_and_events(cuda_lib, oracle):
    """Many massless particles (slot order differs from body order) with
    planetary encounters and impacts, Yarkovsky, PR drag and 1PN."""
    sys = make_system(seed=5, n_particles=2000, nplanets=6, near_fraction=0.05, h=4.0)
    rng = np.random.default_rng(3)
    npart = sys.n - sys.nbig
    sys.ngf[sys.nbig:, 3] = rng.uniform(0.01, 0.3, npart)
    sys.ngf[sys.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
    sys.pn = 1
    ref = sys.copy()
    be = Backend("RADAU", cuda_lib)
    be.configure()
    be.upload(sys)
    ev, _, h, steps = be.hvar_run(0.0, 60.0, 4.0, 1e-12, 0.005)
    x, v = be.download()
    x0, _ = be.download(previous=True)
    be.free()
    want_ev, _, want_h, want_steps, _ = oracle.ra15_run(ref, 0.0, 60.0, 4.0, 1e-12, 0.005)
    assert steps == want_steps and h == want_h
    assert np.array_equal(x, ref.x) and np.array_equal(v, ref.v), (
        np.max(np.abs(x - ref.x)), np.max(np.abs(v - ref.v)))
    assert len(want_ev) > 0
    compare_events(ev, want_ev)
    assert not np.array_equal(x0, x)


def test_force_fails_loudly(cuda_lib):
    sys = force_matrix_system(0, 0, n=20)
    sys.x[7] = 0.0  # a body at the central body's position: mfo_grav's fail()
    be = Backend("RADAU", cuda_lib)
    be.configure()
    be.upload(sys)
    with pytest.raises(BackendError):
        be.force()
    be.free()
