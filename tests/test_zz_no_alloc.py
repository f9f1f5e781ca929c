"""The allocation-free MVS step against the library's regular drop-in step.

mercury_b200_mvs_step_noalloc serves hosts that cannot call cudaMalloc (their
device memory belongs to another allocator or budget, or they cannot accept
the implicit device-wide synchronization of cudaMalloc/cudaFree): the caller
owns every array (here torch allocates them, standing in for such a host) and
the step's scratch lives in a static device array inside the library. Two
calls in a row (the first recomputing the cached accelerations, the second
reusing them) must give the same states and pair records as two
mercury_cuda_step + mercury_cuda_events calls on the same system.

This file is collected last so that a run stopping at its first failure has
already run every other test; it passes alone in a fresh process too (the
first call then performs the per-device set-up).
"""
import ctypes as C

import numpy as np
import pytest

from mercuda_b200.backend import EVENT_DTYPE, Backend
from mercuda_b200.system import make_system

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12   # the parity tolerance of the one-step tests
H = 8.0
RCEN = 0.005
EVENT_CAP = 8192


def _key(ev):
    return [(min(int(e["i"]), int(e["j"])), max(int(e["i"]), int(e["j"])), int(e["kind"]), int(e["now"]))
            for e in ev]


def _sorted(ev):
    order = sorted(range(len(ev)), key=lambda k: (min(ev[k]["i"], ev[k]["j"]), max(ev[k]["i"], ev[k]["j"])))
    return ev[order]


def _rel(a, b):
    scale = np.maximum(np.linalg.norm(b, axis=1, keepdims=True), 1e-300)
    return float(np.max(np.abs(a - b) / scale))


def test_noalloc_step_matches_drop_in_step(cuda_lib):
    import torch

    sys0 = make_system(seed=41, n_particles=3001, near_fraction=0.03)
    nbig, n = sys0.nbig, sys0.n
    npart = n - nbig
    npcap = max(2, npart + (npart & 1))

    # Reference: the existing drop-in entry points, two steps.
    b = Backend("MVS", lib=cuda_lib)
    b.configure()
    b.upload(sys0)
    want = []
    time = 0.0
    for k in range(2):
        b.step(time, H, dtflag=0 if k == 0 else 2)
        x, v = b.download()
        ev = b.events(time + H, H, RCEN)
        want.append((x, v, ev[ev["kind"] != 8]))
        time += H
    b.free()

    # The caller's device arrays (SoA, particle columns padded to npcap).
    dev = torch.device("cuda:0")

    def dev_array(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)

    big = np.zeros((9, nbig))
    big[0:3] = sys0.x[:nbig].T
    big[3:6] = sys0.v[:nbig].T
    part = np.zeros((9, npcap))
    part[0:3, :npart] = sys0.x[nbig:].T
    part[3:6, :npart] = sys0.v[nbig:].T
    const = np.zeros((8, npcap))
    const[0, :npart] = sys0.m[nbig:]
    const[1, :npart] = sys0.rce[nbig:]
    const[2, :npart] = sys0.rphys[nbig:]
    const[3:8, :npart] = sys0.ngf[nbig:].T
    mbig, rcebig, rphysbig = dev_array(sys0.m[:nbig]), dev_array(sys0.rce[:nbig]), dev_array(sys0.rphys[:nbig])
    ngfbig = dev_array(sys0.ngf[:nbig])
    bigbuf = [dev_array(big), torch.zeros((9, nbig), dtype=torch.float64, device=dev)]
    partbuf = [dev_array(part), torch.zeros((9, npcap), dtype=torch.float64, device=dev)]
    constd = dev_array(const)
    events = torch.zeros(EVENT_CAP * EVENT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def ptr(t):
        return C.c_void_p(t.data_ptr())

    time = 0.0
    for k in range(2):
        src, dst = k % 2, 1 - k % 2
        count = C.c_int(-1)
        rc = cuda_lib.mercury_b200_mvs_step_noalloc(
            nbig, npart, ptr(mbig), ptr(rcebig), ptr(rphysbig), ptr(ngfbig), ptr(bigbuf[src]), ptr(bigbuf[dst]),
            ptr(partbuf[src]), ptr(partbuf[dst]), ptr(constd), sys0.ngflag, time, H, 1 if k == 0 else 0,
            ptr(events), EVENT_CAP, C.byref(count), stream)
        assert rc == 0
        big_out = bigbuf[dst].cpu().numpy()
        part_out = partbuf[dst].cpu().numpy()
        x = np.concatenate([big_out[0:3].T, part_out[0:3, :npart].T])
        v = np.concatenate([big_out[3:6].T, part_out[3:6, :npart].T])
        wx, wv, wev = want[k]
        assert _rel(x, wx) <= REL_TOL and _rel(v, wv) <= REL_TOL
        assert 0 <= count.value <= EVENT_CAP
        raw = events[: count.value * EVENT_DTYPE.itemsize].cpu().numpy().tobytes()
        got = _sorted(np.frombuffer(raw, dtype=EVENT_DTYPE))
        assert _key(got) == _key(wev)
        for g, w in zip(got, wev):
            assert abs(g["time"] - w["time"]) <= 1e-9 * max(1.0, abs(w["time"]))
            assert abs(g["distance"] - w["distance"]) <= 1e-9 * max(1e-12, w["distance"])
        time += H


def _noalloc_args(sys0, dev, event_cap):
    """Device arrays of sys0 as the allocation-free step takes them."""
    import torch
    nbig, n = sys0.nbig, sys0.n
    npart = n - nbig
    npcap = max(2, npart + (npart & 1))

    def dev_array(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)

    big = np.zeros((9, nbig))
    big[0:3] = sys0.x[:nbig].T
    big[3:6] = sys0.v[:nbig].T
    part = np.zeros((9, npcap))
    part[0:3, :npart] = sys0.x[nbig:].T
    part[3:6, :npart] = sys0.v[nbig:].T
    const = np.zeros((8, npcap))
    const[0, :npart] = sys0.m[nbig:]
    const[1, :npart] = sys0.rce[nbig:]
    const[2, :npart] = sys0.rphys[nbig:]
    const[3:8, :npart] = sys0.ngf[nbig:].T
    keep = dict(mbig=dev_array(sys0.m[:nbig]), rce=dev_array(sys0.rce[:nbig]), rphys=dev_array(sys0.rphys[:nbig]),
                ngf=dev_array(sys0.ngf[:nbig]), big_in=dev_array(big),
                big_out=torch.zeros((9, nbig), dtype=torch.float64, device=dev), part_in=dev_array(part),
                part_out=torch.zeros((9, npcap), dtype=torch.float64, device=dev), const=dev_array(const),
                events=torch.zeros(max(1, event_cap) * EVENT_DTYPE.itemsize, dtype=torch.uint8, device=dev))
    return keep, npart


def _call(cuda_lib, sys0, keep, npart, event_cap, count, stream, time=0.0, reset=1):
    p = lambda t: C.c_void_p(t.data_ptr())
    return cuda_lib.mercury_b200_mvs_step_noalloc(
        sys0.nbig, npart, p(keep["mbig"]), p(keep["rce"]), p(keep["rphys"]), p(keep["ngf"]), p(keep["big_in"]),
        p(keep["big_out"]), p(keep["part_in"]), p(keep["part_out"]), p(keep["const"]), sys0.ngflag, time, H, reset,
        p(keep["events"]), event_cap, C.byref(count), stream)


def test_noalloc_limits_overflow_and_memory(cuda_lib, capfd):
    """Sizes beyond the stated limits are refused with a message before any
    device work; a record buffer smaller than the step's records fails the
    call and reports the records' total; a system of Big bodies only steps;
    and calls after the first leave the device's free memory unchanged."""
    import torch
    dev = torch.device("cuda:0")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    null = C.c_void_p(0)
    count = C.c_int(-1)
    for nbig, np_, cap, msg in [(65, 10, 16, "nbig must be 1..64"), (9, 262145, 16, "at most 262144 particles"),
                                (9, 10, 8193, "event_cap must be 0..8192")]:
        rc = cuda_lib.mercury_b200_mvs_step_noalloc(nbig, np_, null, null, null, null, null, null, null, null,
                                                    null, 0, 0.0, H, 1, null, cap, C.byref(count), stream)
        assert rc == 1 and msg in capfd.readouterr().err
    # encounter records beyond a small event buffer
    sys0 = make_system(seed=42, n_particles=4001, near_fraction=0.2)
    keep, npart = _noalloc_args(sys0, dev, 2)
    rc = _call(cuda_lib, sys0, keep, npart, 2, count, stream)
    assert rc == 1 and count.value > 2
    assert "capacity exceeded" in capfd.readouterr().err
    # no test particles at all
    big_only = make_system(seed=43, n_particles=0)
    keep0, np0 = _noalloc_args(big_only, dev, 16)
    assert _call(cuda_lib, big_only, keep0, np0, 16, count, stream) == 0
    # the same steps again and again: the device's free memory does not move
    keep, npart = _noalloc_args(sys0, dev, EVENT_CAP)
    assert _call(cuda_lib, sys0, keep, npart, EVENT_CAP, count, stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in range(5):
        assert _call(cuda_lib, sys0, keep, npart, EVENT_CAP, count, stream, reset=0) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
