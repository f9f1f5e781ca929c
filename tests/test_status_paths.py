"""Host-side failure paths of the drop-in boundary, tested without a GPU fault.

The reference tests its Fortran host's failure handling by rewriting the
return values of its CPU stub and relinking (tests/test_edges.py:18-67,
mercury_cuda_stub.cpp:1-20): configure, upload and step failures give a
nonzero status, a `MERCURY CUDA: <what>` line, and the host's fatal message
("CUDA integration step failed", ...). Here the library's own hook does the
same: MERCURY_B200_FAIL names the points that fail on purpose, before any
CUDA call, so these tests run with or without a device. The workspace guard
of the upload (the reference's 80%-of-free-memory check,
mercury_cuda.cu:384-388) is driven the same way. Also: mce_init's limits
(the host-side set-up every HYBRID and MVS test feeds the library) against
the oracle's restatement of mercury6_2.for:1285-1380.
"""
import ctypes as C
import os

import numpy as np
import pytest

from mercuda_b200.backend import Backend, BackendError, load_library
from mercuda_b200.system import make_system, mce_init


@pytest.fixture()
def lib():
    return load_library()


@pytest.fixture()
def fail(monkeypatch):
    def set_points(*points):
        monkeypatch.setenv("MERCURY_B200_FAIL", ",".join(points))
    yield set_points
    os.environ.pop("MERCURY_B200_FAIL", None)


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def upload(lib, s):
    return lib.mercury_cuda_upload(s.n, s.nbig, int(s.pn), s.ngflag, _p(s.m), _p(s.x), _p(s.v), _p(s.ngf),
                                   _p(s.jcen), _p(s.rce), _p(s.rphys))


def test_invalid_algorithm_is_refused(lib):
    """configure accepts 1, 2, 3, 4, 9 and 10 only (mercury_cuda.cu:372)."""
    for bad in (0, 5, 6, 7, 8, 11, -1):
        assert lib.mercury_cuda_configure(bad) == 1


@pytest.mark.parametrize("point", ["configure", "upload", "memory"])
def test_setup_failures_report(lib, fail, capfd, point):
    fail(point)
    s = make_system(seed=1, n_particles=10)
    rc = lib.mercury_cuda_configure(1) if point == "configure" else upload(lib, s)
    assert rc == 1
    err = capfd.readouterr().err
    want = "Insufficient device workspace memory" if point == "memory" else f"injected failure: {point}"
    assert f"MERCURY CUDA: {want}" in err


def test_call_failures_report(lib, fail, capfd):
    """Every step-time entry point turns a failure into status 1 and one line."""
    D, I = C.c_double, C.c_int
    fail("step", "events", "download", "export", "force", "limits", "advance", "hybrid_begin", "hybrid_finish",
         "encounter_enter", "encounter_update")
    x = np.zeros((4, 3))
    hh, hd = D(8.0), D(0.0)
    nf, nr = C.c_int64(0), C.c_int64(0)
    ptr, cnt = C.c_void_p(), I(0)
    ii = np.zeros(4, dtype=np.int32)
    pi = ii.ctypes.data_as(C.POINTER(I))
    calls = {
        "step": lambda: lib.mercury_cuda_step(0.0, C.byref(hh), C.byref(hd), 0.0, C.byref(nf), C.byref(nr)),
        "events": lambda: lib.mercury_cuda_events(8.0, 8.0, 0.005, C.byref(ptr), C.byref(cnt)),
        "download": lambda: lib.mercury_cuda_download(_p(x), _p(x), 0),
        "export": lambda: lib.mercury_cuda_export(8.0, 1, _p(x), _p(x)),
        "force": lambda: lib.mercury_cuda_force(_p(x)),
        "limits": lambda: lib.mercury_cuda_limits(_p(x)),
        "advance": lambda: lib.mercury_b200_mvs_advance(0.0, 8.0, 4, 0.005, 0, C.byref(cnt)),
        "hybrid_begin": lambda: lib.mercury_cuda_hybrid_begin(8.0, _p(x), 0, 4, pi, C.byref(cnt), pi, pi, _p(x),
                                                              _p(x), C.byref(nf)),
        "hybrid_finish": lambda: lib.mercury_cuda_hybrid_finish(8.0, _p(x), _p(x), _p(x), C.byref(nf)),
        "encounter_enter": lambda: lib.mercury_cuda_encounter_enter(2, 1, _p(x), _p(x), _p(x), _p(x), _p(x), _p(x),
                                                                    0, pi, pi),
        "encounter_update": lambda: lib.mercury_cuda_encounter_update(_p(x), _p(x), _p(x)),
    }
    for point, call in calls.items():
        assert call() == 1, point
        assert f"MERCURY CUDA: injected failure: {point}" in capfd.readouterr().err
    lib.mercury_cuda_encounter_exit()


def test_host_mirror_messages(lib, fail, monkeypatch):
    """The host-side mirror of mercury_gpu.f90 raises the bridge's own fatal
    messages (mercury_gpu.f90:128-179): no silent fallback."""
    b = Backend("MVS", lib)
    monkeypatch.setattr(b, "available", lambda: True)
    fail("configure")
    with pytest.raises(BackendError, match="CUDA algorithm initialization failed"):
        b.configure()
    fail("upload")
    with pytest.raises(BackendError, match="CUDA state upload failed"):
        b.upload(make_system(seed=2, n_particles=5))
    fail("step", "events", "download")
    with pytest.raises(BackendError, match="CUDA integration step failed"):
        b.step(0.0, 8.0)
    with pytest.raises(BackendError, match="CUDA event screening failed"):
        b.events(8.0, 8.0, 0.005)
    b.n = 3
    with pytest.raises(BackendError, match="CUDA download failed"):
        b.download()
    with pytest.raises(BackendError, match="CUDA previous state download failed"):
        b.download(previous=True)


def test_unavailable_device_is_an_error(lib, monkeypatch):
    """`execution backend = cuda` without a device is fatal (mercury_gpu.f90:121)."""
    b = Backend("MVS", lib)
    monkeypatch.setattr(b, "available", lambda: False)
    with pytest.raises(BackendError, match="no CUDA device/build is available"):
        b.configure()


@pytest.mark.parametrize("seed,h", [(1, 8.0), (2, -4.0), (3, 0.5)])
def test_mce_init_matches_oracle(oracle, seed, h):
    """system.mce_init == the oracle's mce_init (mce_hill with mco_x2a, the
    rce/rphys/rcrit statements) bit for bit, unbound bodies included."""
    s = make_system(seed=seed, n_particles=500, near_fraction=0.05, h=h)
    s.v[s.nbig:s.nbig + 5] *= 2.0           # unbound: a from the current distance
    s.rceh[s.nbig::7] = 2.5
    s.rho[1:] = np.linspace(1.0, 3.0, s.n - 1) * s.rho[1]
    mce_init(s, h, 3.0)
    rce, rphys, rcrit = oracle.mce_init(s.m, s.x, s.v, s.rho, s.rceh, h, 3.0)
    assert np.array_equal(s.rce[1:], rce[1:])
    assert np.array_equal(s.rphys[1:], rphys[1:])
    assert np.array_equal(s.rcrit[1:], rcrit[1:])
