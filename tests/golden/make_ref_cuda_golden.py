"""Generate the golden fixtures of the reference's own CUDA backend.

The reference backend (mercury_cuda.cu, built unchanged for sm_100a by
`make -C oracle ref` into oracle/_ref/libmercury_cuda_ref.so) is driven through
its C ABI exactly as its Fortran host and its own test harness drive it
(mercury_gpu.f90's gpu_* calls; tests/force_library.py, tests/test_mercury.py,
tests/test_gpu_algorithms.py), on seeded systems. The stored inputs and outputs
pin the CPU oracle to the reference's code.

Two groups:
  mvs    -> tests/golden/ref_cuda_mvs.npz   MVS runs (algorithm 1)
  paths  -> tests/golden/ref_cuda_paths.npz the other paths: the force matrix
            (mercury_cuda_force), RADAU/BS/BS2 runs (mercury_cuda_step +
            _events as mal_hvar makes them), HYBRID runs (hybrid_begin, the
            encounter subsystem as mdt_hkce drives it, hybrid_finish), the
            output corrector (export(h, 1)), MVS with oblateness, with massive
            Small bodies, and the TEST algorithm.

Needs a CUDA device; run from the repository root:
    python tests/golden/make_ref_cuda_golden.py [mvs|paths] [out.npz]
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
from mercuda_b200.system import K2, System, make_system, mce_init  # noqa: E402

D, I = C.c_double, C.c_int
PD = C.POINTER(D)
PI = C.POINTER(I)
PI64 = C.POINTER(C.c_int64)
EV = np.dtype([("i", np.int32), ("j", np.int32), ("kind", np.int32), ("now", np.int32), ("distance", np.float64),
               ("time", np.float64), ("xi", np.float64, 6), ("xj", np.float64, 6)])
REF = ROOT / "oracle/_ref/libmercury_cuda_ref.so"


def p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(PD)


def load():
    """The reference library with the argument types of its 16 entry points
    (mercury_cuda.h:12-34) and nothing else."""
    L = C.CDLL(str(REF))
    L.mercury_cuda_available.restype = I
    L.mercury_cuda_configure.argtypes = [I]
    L.mercury_cuda_reset.argtypes = [I]
    L.mercury_cuda_reset.restype = None
    L.mercury_cuda_limits.argtypes = [PD]
    L.mercury_cuda_export.argtypes = [D, I, PD, PD]
    L.mercury_cuda_upload.argtypes = [I, I, I, I, PD, PD, PD, PD, PD, PD, PD]
    L.mercury_cuda_step.argtypes = [D, PD, PD, D, PI64, PI64]
    L.mercury_cuda_download.argtypes = [PD, PD, I]
    L.mercury_cuda_events.argtypes = [D, D, D, C.POINTER(C.c_void_p), PI]
    L.mercury_cuda_force.argtypes = [PD]
    L.mercury_cuda_hybrid_begin.argtypes = [D, PD, I, I, PI, PI, PI, PI, PD, PD, PI64]
    L.mercury_cuda_hybrid_finish.argtypes = [D, PD, PD, PD, PI64]
    L.mercury_cuda_encounter_enter.argtypes = [I, I, PD, PD, PD, PD, PD, PD, I, PI, PI]
    L.mercury_cuda_encounter_update.argtypes = [PD, PD, PD]
    L.mercury_cuda_encounter_exit.restype = None
    L.mercury_cuda_free.restype = None
    return L


def run_mvs(L, s, h, nsteps, rcen, algorithm=1):
    assert L.mercury_cuda_configure(algorithm) == 0
    assert L.mercury_cuda_upload(s.n, s.nbig, 0, s.ngflag, p(s.m), p(s.x), p(s.v), p(s.ngf), p(s.jcen), p(s.rce),
                                 p(s.rphys)) == 0
    events, steps = [], []
    time = 0.0
    for k in range(nsteps):
        L.mercury_cuda_reset(0 if k == 0 else 2)
        hh, hd = D(h), D(0)
        nf, nr = C.c_int64(0), C.c_int64(0)
        assert L.mercury_cuda_step(time, C.byref(hh), C.byref(hd), 0.0, C.byref(nf), C.byref(nr)) == 0
        ptr, cnt = C.c_void_p(), I(0)
        assert L.mercury_cuda_events(time + h, h, rcen, C.byref(ptr), C.byref(cnt)) == 0
        if cnt.value:
            raw = (C.c_char * (cnt.value * 128)).from_address(ptr.value)
            ev = np.frombuffer(bytes(raw), dtype=EV).copy()
            events.append(ev)
            steps.append(np.full(len(ev), k, dtype=np.int32))
        time = time + h
    x = np.zeros((s.n, 3))
    v = np.zeros((s.n, 3))
    assert L.mercury_cuda_download(p(x), p(v), 0) == 0
    xe = np.zeros((s.n, 3))
    ve = np.zeros((s.n, 3))
    assert L.mercury_cuda_export(h, 1, p(xe), p(ve)) == 0
    L.mercury_cuda_free()
    ev = np.concatenate(events) if events else np.zeros(0, EV)
    st = np.concatenate(steps) if steps else np.zeros(0, np.int32)
    return x, v, ev, st, xe, ve


def store_system(data, name, s):
    for key in ("m", "x", "v", "ngf", "jcen", "rce", "rphys", "rcrit"):
        data[f"{name}/{key}0" if key in ("x", "v") else f"{name}/{key}"] = np.array(getattr(s, key))
    data[f"{name}/nbig"] = np.array(s.nbig)
    data[f"{name}/pn"] = np.array(int(s.pn))


def main_mvs(out):
    L = load()
    assert L.mercury_cuda_available()
    data = {}
    cases = {
        "c0": (make_system(seed=21, n_particles=2000, near_fraction=0.02), 8.0, 46),
        "c0_one": (make_system(seed=22, n_particles=3000, near_fraction=0.03), 8.0, 1),
        "back": (make_system(seed=23, n_particles=500, near_fraction=0.05), -8.0, 20),
    }
    # Kepler regimes: one massless body, no Big bodies (reference test_gpu_algorithms.py:143-153)
    for speed in (0.7, 1.0, 1.2):
        m = np.array([K2, 0.0])
        x = np.array([[0, 0, 0], [0.5, 0, 0]], dtype=float)
        v = np.array([[0, 0, 0], [0, speed * np.sqrt(2 * K2 / 0.5), 0]], dtype=float)
        cases[f"kepler_{speed}"] = (System(m=m, x=x, v=v, nbig=1), 0.5, 64)
    for name, (s, h, nsteps) in cases.items():
        x, v, ev, st, _, _ = run_mvs(L, s, h, nsteps, 0.005)
        for key, val in [("m", s.m), ("x0", s.x), ("v0", s.v), ("rce", s.rce), ("rphys", s.rphys)]:
            data[f"{name}/{key}"] = val
        data[f"{name}/nbig"] = np.array(s.nbig)
        data[f"{name}/h"] = np.array(h)
        data[f"{name}/nsteps"] = np.array(nsteps)
        data[f"{name}/x"] = x
        data[f"{name}/v"] = v
        data[f"{name}/events"] = ev
        data[f"{name}/event_steps"] = st
        print(name, s.n, "bodies,", nsteps, "steps,", len(ev), "events")
    np.savez_compressed(out, **data)


def reference_backend(L, algorithm):
    """The repository's host-side mirror of mercury_gpu.f90 (Backend) bound to
    the reference library: only drop-in entry points are called."""
    from mercuda_b200.backend import Backend
    return Backend(algorithm, lib=L)


def main_paths(out):
    from adaptive_cases import hvar_system, planar_body, run_intervals
    from test_radau_gpu import force_matrix_system

    L = load()
    assert L.mercury_cuda_available()
    data = {}

    # mercury_cuda_force across 1PN x ngflag with J2-J6 (reference tests/test_mercury.py:113-133)
    for pn in (0, 1):
        for flag in range(4):
            s = force_matrix_system(pn, flag)
            name = f"force_pn{pn}_ng{flag}"
            assert L.mercury_cuda_configure(2) == 0
            assert L.mercury_cuda_upload(s.n, s.nbig, pn, flag, p(s.m), p(s.x), p(s.v), p(s.ngf), p(s.jcen),
                                         p(s.rce), p(s.rphys)) == 0
            a = np.zeros((s.n, 3))
            assert L.mercury_cuda_force(p(a)) == 0
            L.mercury_cuda_free()
            store_system(data, name, s)
            data[f"{name}/a"] = a
            print(name)

    # RADAU, BS, BS2 (reference tests/test_gpu_algorithms.py:89-110): three planets,
    # 33 planar Small bodies (every third semi-active), output interval 7.3 d
    adaptive = []
    for direction in (-1, 1):
        for pn in (0, 1):
            adaptive.append(("RADAU", True, pn, direction))
        for massive in (False, True):
            adaptive.append(("BS2", massive, 0, direction))
        adaptive.append(("BS", True, 1, direction))
    for alg, massive, pn, direction in adaptive:
        s = hvar_system(massive=massive, pn=pn)
        name = f"hvar_{alg}_m{int(massive)}_pn{pn}_d{direction}"
        store_system(data, name, s)
        be = reference_backend(L, alg)
        be.configure()
        be.upload(s)
        ev, hnext = run_intervals(be, s, 0.0, 32.0 * direction, 7.3, 0.5, 1e-12)
        x, v = be.download()
        be.free()
        data[f"{name}/x"] = x
        data[f"{name}/v"] = v
        data[f"{name}/events"] = np.asarray(ev, dtype=EV) if len(ev) else np.zeros(0, EV)
        data[f"{name}/h"] = np.array(hnext)
        print(name, len(ev), "events")

    # The oblateness of the reference's test (J2 = 0.1, J4 = -1e-3 with
    # rcen = 0.005 AU, tests/test_gpu_algorithms.py:79-87) as its Fortran host
    # passes it to the backend: mio_in scales J_2n by rcen^2n
    # (mercury6_2.for:6171-6173).
    rcen = 0.005
    jcen_test = [0.1 * rcen ** 2, -1e-3 * rcen ** 4, 0.0]

    # HYBRID (reference tests/test_gpu_algorithms.py:34-41, 166-177): semi-active
    # and massless Small bodies both ways, a close Big pair that forces the BS2
    # subsystem, no Big bodies, the oblateness reaction, and particles near planets
    def close_pair(count=3, jcen=None):
        bodies = [(K2, [0.0] * 3, [0.0] * 3), planar_body(1e-5, 1.0, 0.0, 0.0), planar_body(1e-5, 1.02, 0.0, 0.02)]
        bodies += [planar_body(0.0, 1.6 + j * 0.012, 0.12, j * 0.37) for j in range(count)]
        n = len(bodies)
        s = System(m=np.array([b[0] for b in bodies]), x=np.array([b[1] for b in bodies]),
                   v=np.array([b[2] for b in bodies]), nbig=3, rce=np.full(n, 0.01), rphys=np.full(n, 1e-5))
        if jcen is not None:
            s.jcen[:] = jcen
        return mce_init(s, 0.5, 3.0)

    def no_big(count):
        bodies = [(K2, [0.0] * 3, [0.0] * 3)] + [planar_body(0.0, 1.6 + j * 0.012, 0.12, j * 0.37)
                                                 for j in range(count)]
        s = System(m=np.array([b[0] for b in bodies]), x=np.array([b[1] for b in bodies]).reshape(-1, 3),
                   v=np.array([b[2] for b in bodies]).reshape(-1, 3), nbig=1)
        return mce_init(s, 0.5, 3.0)

    def oblate(massive, jcen):
        bodies = [(K2, [0.0] * 3, [0.0] * 3), planar_body(1e-3, 0.3, 0.02, 0.0), planar_body(1e-3, 5.2, 0.04, 0.0)]
        bodies += [planar_body(1e-8 if massive and j % 3 == 0 else 0.0, 1.6 + j * 0.012, 0.12, j * 0.37)
                   for j in range(33)]
        n = len(bodies)
        s = System(m=np.array([b[0] for b in bodies]), x=np.array([b[1] for b in bodies]),
                   v=np.array([b[2] for b in bodies]), nbig=3, rce=np.full(n, 0.05), rphys=np.full(n, 1e-4))
        s.jcen[:] = jcen
        return s

    hybrid = [
        ("hy_semi_m0_dm", mce_init(hvar_system(massive=False, pn=0), 0.5, 3.0), -0.5, 60),
        ("hy_semi_m0_dp", mce_init(hvar_system(massive=False, pn=0), 0.5, 3.0), 0.5, 60),
        ("hy_semi_m1_dm", mce_init(hvar_system(massive=True, pn=0), 0.5, 3.0), -0.5, 60),
        ("hy_semi_m1_dp", mce_init(hvar_system(massive=True, pn=0), 0.5, 3.0), 0.5, 60),
        ("hy_close_pair", close_pair(), 0.5, 16),
        ("hy_close_pair_oblate", close_pair(jcen=jcen_test), 0.5, 16),
        ("hy_no_big_257", no_big(257), 0.5, 32),
        ("hy_oblate_m1", mce_init(oblate(True, jcen_test), 0.5, 3.0), 0.5, 128),
        ("hy_particles", make_system(seed=3, n_particles=1500, nplanets=8, near_fraction=0.05, h=8.0), 8.0, 10),
    ]
    for name, s, h, nsteps in hybrid:
        store_system(data, name, s)
        be = reference_backend(L, "HYBRID")
        be.configure()
        be.upload(s)
        state = {"dtflag": 0}
        events, pairs, t = [], 0, 0.0
        for _ in range(nsteps):
            ev, npair = be.hybrid_step(s, t, h, 1e-12, state, 0.005, fused=False)
            pairs += npair
            t = t + h
            events.append(ev)
            events.append(be.events(t, h, 0.005))
        x, v = be.download()
        xe, ve = be.export(h, physical=True)
        be.free()
        ev = np.concatenate(events) if events else np.zeros(0, EV)
        data[f"{name}/x"] = x
        data[f"{name}/v"] = v
        data[f"{name}/xe"] = xe
        data[f"{name}/ve"] = ve
        data[f"{name}/events"] = np.asarray(ev, dtype=EV)
        data[f"{name}/h"] = np.array(h)
        data[f"{name}/nsteps"] = np.array(nsteps)
        data[f"{name}/pairs"] = np.array(pairs)
        data[f"{name}/forces"] = np.array(be.forces)
        print(name, pairs, "pairs", len(ev), "events")

    # MVS beyond the plain workload: the oblateness reaction (reference
    # tests/test_gpu_algorithms.py:159-165), massive Small bodies with and
    # without it, non-gravitational terms, both directions, the TEST algorithm;
    # the corrected state export(h, 1) of each
    def with_ngf(s):
        s.ngf[s.nbig:, 0] = 1e-9
        s.ngf[s.nbig:, 2] = 1e-9
        return s

    mvs = [
        ("mvs_oblate", oblate(False, jcen_test), 0.5, 128, 1),
        ("mvs_oblate_massive", oblate(True, jcen_test), 0.5, 128, 1),
        # J2 r^-2 = 1.1 at the inner planet's orbit: the reaction as large as
        # the Kepler term
        ("mvs_oblate_strong", oblate(True, [0.1, -1e-3, 0.0]), 0.5, 128, 1),
        ("mvs_massive", hvar_system(massive=True, pn=0), 0.5, 64, 1),
        ("mvs_back", hvar_system(massive=False, pn=0), -0.5, 256, 1),
        ("mvs_ngf", with_ngf(hvar_system(massive=False, pn=0)), 0.5, 256, 1),
        ("mvs_test_alg", hvar_system(massive=False, pn=0), 0.5, 64, 9),
        ("mvs_workload", make_system(seed=24, n_particles=3000, near_fraction=0.02), 8.0, 46, 1),
    ]
    for name, s, h, nsteps, alg in mvs:
        store_system(data, name, s)
        x, v, ev, st, xe, ve = run_mvs(L, s, h, nsteps, 0.005, alg)
        data[f"{name}/x"] = x
        data[f"{name}/v"] = v
        data[f"{name}/xe"] = xe
        data[f"{name}/ve"] = ve
        data[f"{name}/events"] = ev
        data[f"{name}/event_steps"] = st
        data[f"{name}/h"] = np.array(h)
        data[f"{name}/nsteps"] = np.array(nsteps)
        data[f"{name}/algorithm"] = np.array(alg)
        print(name, len(ev), "events")
    np.savez_compressed(out, **data)


if __name__ == "__main__":
    group = sys.argv[1] if len(sys.argv) > 1 else "mvs"
    default = ROOT / ("tests/golden/ref_cuda_mvs.npz" if group == "mvs" else "tests/golden/ref_cuda_paths.npz")
    target = sys.argv[2] if len(sys.argv) > 2 else default
    (main_mvs if group == "mvs" else main_paths)(target)
