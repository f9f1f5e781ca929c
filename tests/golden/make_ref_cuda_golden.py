"""Generate tests/golden/ref_cuda_mvs.npz from the reference's own CUDA backend.

The reference backend (mercury_cuda.cu, built unchanged for sm_100a by
`make -C oracle ref` into oracle/_ref/libmercury_cuda_ref.so) is driven through
its C ABI exactly as its own test harness does (upload, configure, step,
events, download), on seeded systems of this path's workload generator.
The stored inputs and outputs pin the CPU oracle to the reference's code.

Needs a CUDA device; run from the repository root:
    python tests/golden/make_ref_cuda_golden.py [out.npz]
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from mercuda_b200.system import K2, System, make_system  # noqa: E402

D, I = C.c_double, C.c_int
PD = C.POINTER(D)
EV = np.dtype([("i", np.int32), ("j", np.int32), ("kind", np.int32), ("now", np.int32), ("distance", np.float64),
               ("time", np.float64), ("xi", np.float64, 6), ("xj", np.float64, 6)])


def p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(PD)


def load():
    L = C.CDLL(str(ROOT / "oracle/_ref/libmercury_cuda_ref.so"))
    L.mercury_cuda_upload.argtypes = [I, I, I, I, PD, PD, PD, PD, PD, PD, PD]
    L.mercury_cuda_step.argtypes = [D, PD, PD, D, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.mercury_cuda_download.argtypes = [PD, PD, I]
    L.mercury_cuda_events.argtypes = [D, D, D, C.POINTER(C.c_void_p), C.POINTER(I)]
    L.mercury_cuda_force.argtypes = [PD]
    L.mercury_cuda_reset.argtypes = [I]
    return L


def run_mvs(L, s, h, nsteps, rcen):
    assert L.mercury_cuda_configure(1) == 0
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
    L.mercury_cuda_free()
    ev = np.concatenate(events) if events else np.zeros(0, EV)
    st = np.concatenate(steps) if steps else np.zeros(0, np.int32)
    return x, v, ev, st


def main(out):
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
        x, v, ev, st = run_mvs(L, s, h, nsteps, 0.005)
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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else ROOT / "tests/golden/ref_cuda_mvs.npz")
