"""ctypes front end of ``libmercury_cuda.so``, mirroring the Fortran bridge.

The reference host drives its CUDA backend through the ``gpu_*`` wrappers of
mercury_gpu.f90 (gpu_select, gpu_push, gpu_advance, gpu_find_events,
gpu_central, gpu_pull, gpu_old, gpu_bcoord/gpu_export, gpu_limits, gpu_free).
:class:`Backend` exposes the same calls with the same argument meaning and
failure behaviour (a nonzero status from the library raises
:class:`BackendError` carrying the bridge's message, e.g. "CUDA integration
step failed"), plus the library's multi-step extension.

There is no CPU fallback here: if the library cannot be loaded, or no CUDA
device is present when one is needed, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

from .system import System

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmercury_cuda.so"

D = C.c_double
I = C.c_int
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int)
PI64 = C.POINTER(C.c_int64)

ALGORITHMS = {"MVS": 1, "BS": 2, "BS2": 3, "RADAU": 4, "TEST": 9, "HYBRID": 10}

EVENT_DTYPE = np.dtype([("i", np.int32), ("j", np.int32), ("kind", np.int32), ("now", np.int32),
                        ("distance", np.float64), ("time", np.float64),
                        ("xi", np.float64, 6), ("xj", np.float64, 6)])

# Every symbol include/mercury_cuda.h and include/mercury_b200.h declare.
DROP_IN_SYMBOLS = [
    "mercury_cuda_available", "mercury_cuda_configure", "mercury_cuda_reset", "mercury_cuda_limits",
    "mercury_cuda_export", "mercury_cuda_upload", "mercury_cuda_step", "mercury_cuda_download",
    "mercury_cuda_events", "mercury_cuda_force", "mercury_cuda_hybrid_begin", "mercury_cuda_hybrid_finish",
    "mercury_cuda_encounter_enter", "mercury_cuda_encounter_update", "mercury_cuda_encounter_exit",
    "mercury_cuda_free",
]
EXTENSION_SYMBOLS = ["mercury_b200_mvs_advance", "mercury_b200_mvs_run", "mercury_b200_advance_launches",
                     "mercury_b200_events", "mercury_b200_timing",
                     "mercury_b200_set_launch", "mercury_b200_fp64_peak", "mercury_b200_mvs_step_noalloc",
                     "mercury_b200_dropin_time", "mercury_b200_batch_upload", "mercury_b200_batch_advance",
                     "mercury_b200_batch_events", "mercury_b200_batch_download", "mercury_b200_batch_set",
                     "mercury_b200_batch_timing", "mercury_b200_batch_free", "mercury_b200_adjoint_forward",
                     "mercury_b200_adjoint_backward", "mercury_b200_adjoint_timing", "mercury_b200_adjoint_free",
                     "mercury_b200_energy", "mercury_b200_hybrid_adjoint_forward",
                     "mercury_b200_hybrid_adjoint_backward", "mercury_b200_hybrid_adjoint_timing",
                     "mercury_b200_hybrid_adjoint_free", "mercury_b200_ejections",
                     "mercury_b200_encode_ce", "mercury_b200_set_step_reduce",
                     "mercury_b200_encounter_run", "mercury_b200_hybrid_members", "mercury_b200_hybrid_member_list",
                     "mercury_b200_epoch_order",
                     "mercury_b200_sync_epochs", "mercury_b200_set_event_capacity"]

# fn(values, count, user) of mercury_b200_set_step_reduce
REDUCE_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.c_int, C.c_void_p)


class BackendError(RuntimeError):
    pass


_lib: C.CDLL | None = None


def load_library(path: Path | str | None = None) -> C.CDLL:
    """Load the CUDA library (built in-tree by mercuda_b200.build)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise BackendError(f"{p} is missing: run `python -m mercuda_b200.build`")
    L = C.CDLL(str(p))
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
    L.mercury_b200_mvs_advance.argtypes = [D, D, I, D, I, PI]
    L.mercury_b200_mvs_run.argtypes = [I, I, I, I, PD, PD, PD, PD, PD, PD, PD, D, D, I, D, I, PD, PD, PI]
    L.mercury_b200_events.argtypes = [C.c_void_p, PI, I]
    L.mercury_b200_timing.argtypes = [PD, PD, PI, PI]
    L.mercury_b200_advance_launches.argtypes = [PI, PD, I]
    L.mercury_b200_set_launch.argtypes = [I, I]
    L.mercury_b200_fp64_peak.argtypes = [PD, PD]
    L.mercury_b200_dropin_time.argtypes = [PD, PI64, I]
    L.mercury_b200_energy.argtypes = [D, I, PD, PD, PD]
    L.mercury_b200_ejections.argtypes = [D, I, D, I, PI, I, PI]
    L.mercury_b200_encode_ce.argtypes = [C.c_void_p, I, D, D, D, C.c_void_p, PI]
    L.mercury_b200_set_step_reduce.argtypes = [C.c_void_p, C.c_void_p]
    L.mercury_b200_set_event_capacity.argtypes = [C.c_int]
    L.mercury_b200_encounter_run.argtypes = [D, D, D, D, PD, PI64, PI]
    L.mercury_b200_hybrid_members.argtypes = [PI, I]
    L.mercury_b200_hybrid_member_list.argtypes = [PI, I]
    L.mercury_b200_epoch_order.argtypes = [I, PD, D, PI]
    L.mercury_b200_sync_epochs.argtypes = [PD, PD, D, D, D, PI]
    L.mercury_b200_batch_upload.argtypes = [I, PI, PI, PD, PD, PD, PD, PD, PD]
    L.mercury_b200_batch_advance.argtypes = [D, I, D, PI]
    L.mercury_b200_batch_events.argtypes = [C.c_void_p, PI, PI, I]
    L.mercury_b200_batch_download.argtypes = [PD, PD]
    L.mercury_b200_batch_set.argtypes = [I, I, I]
    L.mercury_b200_batch_timing.argtypes = [PD, PI, PI, PI]
    L.mercury_b200_batch_free.restype = None
    VP_ = C.c_void_p
    L.mercury_b200_adjoint_forward.argtypes = [I, PD, PD, PD, I, VP_, VP_, VP_, D, I, I, VP_, VP_]
    L.mercury_b200_adjoint_backward.argtypes = [VP_, VP_, VP_, VP_, VP_]
    L.mercury_b200_adjoint_timing.argtypes = [PD, PD]
    L.mercury_b200_adjoint_free.restype = None
    L.mercury_b200_hybrid_adjoint_forward.argtypes = [I, PD, PD, PD, PD, I, VP_, VP_, VP_, PD, D, D, I, I, VP_, VP_]
    L.mercury_b200_hybrid_adjoint_backward.argtypes = [VP_, VP_, VP_, VP_, VP_]
    L.mercury_b200_hybrid_adjoint_timing.argtypes = [PD, PD, PI64]
    L.mercury_b200_hybrid_adjoint_free.restype = None
    VP = C.c_void_p
    L.mercury_b200_mvs_step_noalloc.argtypes = [I, I, VP, VP, VP, VP, VP, VP, VP, VP, VP, I, D, D, I, VP, I,
                                                PI, VP]
    if path is None:
        _lib = L
    return L


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous, "float64 C-contiguous array required"
    return a.ctypes.data_as(PD)


def epoch_order(epochs: np.ndarray, tstart: float, lib: C.CDLL | None = None) -> np.ndarray:
    """mxx_sync's order of the Small bodies: order[k] = the Small body at position k."""
    L = lib or load_library()
    e = np.ascontiguousarray(epochs, dtype=np.float64)
    order = np.zeros(max(1, len(e)), dtype=np.int32)
    if L.mercury_b200_epoch_order(len(e), _p(e), tstart, order.ctypes.data_as(PI)) != 0:
        raise BackendError("epoch ordering failed")
    return order[:len(e)].copy()


def encode_ce(events: np.ndarray, mcen: float, rcen: float, rmax: float, lib: C.CDLL | None = None) -> np.ndarray:
    """mio_ce's 70-character record bodies of the close encounters (kind bit 1)
    among `events` (EVENT_DTYPE records), encoded on the device: uint8 (count, 70)."""
    L = lib or load_library()
    ev = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    lines = np.zeros((max(1, len(ev)), 70), dtype=np.uint8)
    count = C.c_int(0)
    if L.mercury_b200_encode_ce(ev.ctypes.data_as(C.c_void_p), len(ev), mcen, rcen, rmax,
                                lines.ctypes.data_as(C.c_void_p), C.byref(count)) != 0:
        raise BackendError("close-encounter encoding failed")
    return lines[:count.value].copy()


class Backend:
    """One device context of libmercury_cuda.so, driven like mercury_gpu.f90."""

    def __init__(self, algorithm: str | int = "MVS", lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        self.algorithm = ALGORITHMS[algorithm] if isinstance(algorithm, str) else int(algorithm)
        self.n = 0
        self.nbig = 0
        self.forces = 0
        self.rejected = 0

    # gpu_select (mercury_gpu.f90:115-138)
    def available(self) -> bool:
        return bool(self.lib.mercury_cuda_available())

    def configure(self) -> None:
        if not self.available():
            raise BackendError("CUDA was requested but no CUDA device/build is available")
        if self.lib.mercury_cuda_configure(self.algorithm) != 0:
            raise BackendError("CUDA algorithm initialization failed")

    # gpu_push (mercury_gpu.f90:139-151)
    def upload(self, sys: System, ngflag: int | None = None) -> None:
        """ngflag: the force-law flag that mio_in derives from the input once
        (mercury6_2.for:6360-6371); None derives it from sys.ngf here."""
        self.n, self.nbig = sys.n, sys.nbig
        flag = sys.ngflag if ngflag is None else int(ngflag)
        rc = self.lib.mercury_cuda_upload(sys.n, sys.nbig, int(sys.pn), flag, _p(sys.m), _p(sys.x), _p(sys.v),
                                          _p(sys.ngf), _p(sys.jcen), _p(sys.rce), _p(sys.rphys))
        if rc != 0:
            raise BackendError("CUDA state upload failed")

    def reset(self, dtflag: int = 0) -> None:
        self.lib.mercury_cuda_reset(int(dtflag))

    # gpu_advance (mercury_gpu.f90:168-179)
    def step(self, time: float, h: float, tol: float = 0.0, dtflag: int = 2):
        self.reset(dtflag)
        hh, hdid = D(h), D(0.0)
        nf, nr = C.c_int64(0), C.c_int64(0)
        if self.lib.mercury_cuda_step(time, C.byref(hh), C.byref(hdid), tol, C.byref(nf), C.byref(nr)) != 0:
            raise BackendError("CUDA integration step failed")
        self.forces += nf.value
        self.rejected += nr.value
        return hdid.value, hh.value

    # gpu_refresh_events (mercury_gpu.f90:108-114)
    def events(self, time: float, h: float, rcen: float) -> np.ndarray:
        ptr, count = C.c_void_p(), I(0)
        if self.lib.mercury_cuda_events(time, h, rcen, C.byref(ptr), C.byref(count)) != 0:
            raise BackendError("CUDA event screening failed")
        if count.value == 0:
            return np.zeros(0, dtype=EVENT_DTYPE)
        buf = (C.c_char * (count.value * EVENT_DTYPE.itemsize)).from_address(ptr.value)
        return np.frombuffer(bytes(buf), dtype=EVENT_DTYPE).copy()

    # gpu_pull / gpu_old (mercury_gpu.f90:180-185, 202-205)
    def download(self, previous: bool = False, out=None):
        """(x, v) of every body; `out` = (x, v) float64 (n, 3) arrays to fill
        (page-locked host arrays are written directly by DMA)."""
        if out is not None:
            x, v = out
            assert x.shape == v.shape == (self.n, 3) and x.dtype == v.dtype == np.float64
            assert x.flags.c_contiguous and v.flags.c_contiguous
        else:
            x = np.empty((self.n, 3))
            v = np.empty((self.n, 3))
        if self.lib.mercury_cuda_download(_p(x), _p(v), int(previous)) != 0:
            raise BackendError("CUDA previous state download failed" if previous else "CUDA download failed")
        return x, v

    # gpu_export (mercury_gpu.f90:186-191)
    def export(self, h: float, physical: bool = True):
        x = np.zeros((self.n, 3))
        v = np.zeros((self.n, 3))
        if self.lib.mercury_cuda_export(h, int(physical), _p(x), _p(v)) != 0:
            raise BackendError("CUDA coordinate export failed")
        return x, v

    # gpu_limits (mercury_gpu.f90:88-92)
    def limits(self, rce: np.ndarray) -> None:
        if self.lib.mercury_cuda_limits(_p(np.ascontiguousarray(rce, dtype=np.float64))) != 0:
            raise BackendError("CUDA encounter-radius update failed")

    def force(self) -> np.ndarray:
        a = np.zeros((self.n, 3))
        if self.lib.mercury_cuda_force(_p(a)) != 0:
            raise BackendError("CUDA force evaluation failed")
        return a

    def free(self) -> None:
        self.lib.mercury_cuda_free()

    # gpu_hybrid_begin / gpu_hybrid_finish (mercury_gpu.f90:93-107)
    def hybrid_begin(self, h: float, rcrit: np.ndarray, flag: int, x: np.ndarray, v: np.ndarray, cap: int = 1 << 20):
        """Kick, solar drift, Kepler drift and mce_snif. Returns (ce, pi, pj); the
        members' rows of x, v receive their pre-drift states."""
        n = self.n
        # work arrays kept between steps: the library writes ce and the pair
        # lists only when there are pairs, and reads back only members' rows
        buf = getattr(self, "_begin_buf", None)
        if buf is None or len(buf[0]) != n or len(buf[1]) != cap:
            buf = (np.zeros(n, dtype=np.int32), np.zeros(cap, dtype=np.int32), np.zeros(cap, dtype=np.int32))
            self._begin_buf = buf
        ce, pi, pj = buf
        count, nf = I(0), C.c_int64(0)
        rc = self.lib.mercury_cuda_hybrid_begin(h, _p(np.ascontiguousarray(rcrit, dtype=np.float64)), int(flag),
                                                cap, ce.ctypes.data_as(PI), C.byref(count), pi.ctypes.data_as(PI),
                                                pj.ctypes.data_as(PI), _p(x), _p(v), C.byref(nf))
        if rc != 0:
            raise BackendError("CUDA hybrid drift failed")
        self.forces += nf.value
        return ce, pi[:count.value].copy(), pj[:count.value].copy()

    def hybrid_member_list(self) -> np.ndarray:
        """The bodies (0-based, ascending, no central body) whose rows
        hybrid_finish takes in the current HYBRID step."""
        count = self.lib.mercury_b200_hybrid_member_list(None, 0)
        if count < 0:
            raise BackendError("no HYBRID step begun")
        ids = np.empty(count, dtype=np.int32)
        if count:
            self.lib.mercury_b200_hybrid_member_list(ids.ctypes.data_as(PI), count)
        return ids.astype(np.int64)

    def hybrid_finish(self, h: float, m: np.ndarray, x: np.ndarray, v: np.ndarray) -> None:
        nf = C.c_int64(0)
        if self.lib.mercury_cuda_hybrid_finish(h, _p(m), _p(x), _p(v), C.byref(nf)) != 0:
            raise BackendError("CUDA hybrid kick failed")
        self.forces += nf.value

    # mdt_hy's CUDA branch with mdt_hkce's (mercury6_2.for:3646-3659, 3798-3940)
    def hybrid_step(self, sys: System, time: float, h: float, tol: float, state: dict, rcen: float = 0.005,
                    fused: bool = True):
        """One HYBRID step of sys (democratic-heliocentric masses/radii/rcrit on
        the host; positions live on the device). `state` carries dtflag and hrec
        between calls. Returns the encounter records of the subsystem (global
        1-based ids) and the number of encounter pairs. The encounter
        subsystem's substeps run inside the library (mercury_b200_encounter_run)
        or, with fused=False, one drop-in call at a time from here as
        mercury_gpu.f90's host loop makes them; the results are the same."""
        if state.get("dtflag", 0) == 0:
            state["hrec"] = h
        # host rows of the members only pass through x, v (kept between steps)
        rows = getattr(self, "_step_rows", None)
        if rows is None or rows[0].shape[0] != sys.n:
            rows = (np.zeros((sys.n, 3)), np.zeros((sys.n, 3)))
            self._step_rows = rows
        x, v = rows
        ce, pi, pj = self.hybrid_begin(h, sys.rcrit, state.get("dtflag", 0), x, v)
        state["dtflag"] = 2
        events = np.zeros(0, dtype=EVENT_DTYPE)
        if len(pi):
            # the members as the library collected them from the pairs (the
            # bodies that ce flags, without a scan of ce); a library with the
            # drop-in calls alone (the reference's) is scanned
            if hasattr(self.lib, "mercury_b200_hybrid_member_list"):
                members = self.hybrid_member_list()
            else:
                members = np.nonzero(ce[1:])[0] + 1
            sub = np.concatenate([[0], members])
            xbs, vbs, events = self.encounter_subsystem(sub, sys.nbig, sys.m[sub], x[sub], v[sub], sys.rcrit[sub],
                                                         sys.rce[sub], sys.rphys[sub], pi, pj, time, h, tol, state,
                                                         rcen, fused)
            x[sub[1:]] = xbs[1:]
            v[sub[1:]] = vbs[1:]
        self.hybrid_finish(h, sys.m, x, v)
        return events, len(pi)

    def encounter_subsystem(self, sub, nbig, m, x, v, rcrit, rce, rphys, pi, pj, time, h, tol, state, rcen,
                            fused=True):
        """mdt_hkce (mercury6_2.for:3798-3940) through the drop-in calls: the
        central body and the members sub[1:] (sorted global 0-based indices;
        sub[0] = 0) with masses, pre-drift states and radii in the same order
        (row 0 is ignored), encounter pairs pi/pj (global 1-based). Returns the
        members' end states (rows as sub) and the close-encounter records
        with global 1-based ids (an EVENT_DTYPE array)."""
        sub = np.asarray(sub)
        index = sub.tolist()
        nbs = len(sub)
        nbsbig = 1 + int(np.count_nonzero(sub[1:] < nbig))
        mbs = np.ascontiguousarray(m, dtype=np.float64).copy()
        xbs = np.array(x, dtype=np.float64)
        vbs = np.array(v, dtype=np.float64)
        xbs[0] = 0.0
        vbs[0] = 0.0
        rcritbs = np.array(rcrit, dtype=np.float64)
        rcebs = np.array(rce, dtype=np.float64)
        rphybs = np.array(rphys, dtype=np.float64)
        rcritbs[0] = rcebs[0] = rphybs[0] = 0.0
        # subsystem index of each pair member (sub is sorted)
        ibs = np.ascontiguousarray(np.searchsorted(sub, np.asarray(pi) - 1) + 1, dtype=np.int32)
        jbs = np.ascontiguousarray(np.searchsorted(sub, np.asarray(pj) - 1) + 1, dtype=np.int32)
        if self.lib.mercury_cuda_encounter_enter(nbs, nbsbig, _p(mbs), _p(xbs), _p(vbs), _p(rcritbs), _p(rcebs),
                                                 _p(rphybs), len(ibs), ibs.ctypes.data_as(PI),
                                                 jbs.ctypes.data_as(PI)) != 0:
            raise BackendError("CUDA encounter initialization failed")
        records = []
        outer_n = self.n
        self.n = nbs
        try:
            if fused:
                # the same drop-in calls, looped inside the library
                hrec, nf, nrec = D(state["hrec"]), C.c_int64(0), I(0)
                if self.lib.mercury_b200_encounter_run(time, h, tol, rcen, C.byref(hrec), C.byref(nf),
                                                       C.byref(nrec)) != 0:
                    raise BackendError("CUDA integration step failed")
                state["hrec"] = hrec.value
                self.forces += nf.value
                sub_ev = np.zeros(nrec.value, dtype=EVENT_DTYPE)
                if nrec.value:
                    self.lib.mercury_b200_events(sub_ev.ctypes.data_as(C.c_void_p), None, nrec.value)
                    # subsystem ids -> global ids
                    sub_ev["i"] = sub[sub_ev["i"] - 1] + 1
                    sub_ev["j"] = sub[sub_ev["j"] - 1] + 1
                records = sub_ev
                xbs, vbs = self.download()
            else:
                dtflag, tlocal, hlocal = 1, 0.0, math.copysign(state["hrec"], h)
                while True:
                    tmp0 = abs(h) - abs(tlocal)
                    state["hrec"] = hlocal
                    if abs(hlocal) > tmp0:
                        hlocal = math.copysign(tmp0, h)
                    hdid, hlocal = self.step(tlocal, hlocal, tol, dtflag)
                    dtflag = 2
                    xbs, vbs = self.download()
                    tlocal = tlocal + hdid
                    for e in self.events(time + tlocal, hdid, rcen):
                        if e["kind"] & 8:
                            continue
                        e = e.copy()
                        e["i"] = index[e["i"] - 1] + 1
                        e["j"] = index[e["j"] - 1] + 1
                        records.append(e)
                    if not (tlocal - h) * h < 0.0:
                        break
        finally:
            self.lib.mercury_cuda_encounter_exit()
            self.n = outer_n
        if not isinstance(records, np.ndarray):
            records = np.array(records, dtype=EVENT_DTYPE) if records else np.zeros(0, dtype=EVENT_DTYPE)
        return xbs, vbs, records

    def sync_epochs(self, epoch: np.ndarray, time: float, h0: float, tol: float, dtout: float):
        """mxx_sync's integration of the uploaded system (in its order, see
        epoch_order): returns (the common epoch reached, BS steps)."""
        ep = np.ascontiguousarray(epoch, dtype=np.float64)
        t, steps = D(time), I(0)
        if self.lib.mercury_b200_sync_epochs(_p(ep), C.byref(t), h0, tol, dtout, C.byref(steps)) != 0:
            raise BackendError("epoch synchronisation failed")
        return t.value, steps.value

    def hybrid_members(self, ids) -> None:
        """The bodies (0-based) whose rows hybrid_finish takes from x, v."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        if self.lib.mercury_b200_hybrid_members(ids.ctypes.data_as(PI), len(ids)) != 0:
            raise BackendError("CUDA hybrid member list rejected")

    # mal_hvar's step loop (mercury6_2.for:423-470) through the drop-in calls:
    # steps clipped to tstop, dtflag = 1 (a fresh RA15 sequence) when a clipped
    # step changes h, events screened after every step.
    def hvar_run(self, time0: float, tstop: float, h: float, tol: float, rcen: float, max_steps: int = 1_000_000):
        """Returns (events, step index of each event, h after the last step, steps taken)."""
        time, dtflag, steps = time0, 0, 0
        events, where = [], []
        while steps < max_steps:
            if abs(tstop - time) <= 0.0:
                break
            step = math.copysign(min(abs(tstop - time), abs(h)), tstop - time)
            if not math.isfinite(step) or time + step == time:
                break
            if step != h and dtflag != 0:
                dtflag = 1
            h = step
            hdid, h = self.step(time, h, tol, dtflag)
            dtflag = 2
            time = time + hdid
            ev = self.events(time, hdid, rcen)
            if len(ev):
                events.append(ev)
                where.append(np.full(len(ev), steps, dtype=np.int32))
            steps += 1
        if events:
            return np.concatenate(events), np.concatenate(where), h, steps
        return np.zeros(0, dtype=EVENT_DTYPE), np.zeros(0, dtype=np.int32), h, steps

    # extension: fused multi-step MVS run
    def mvs_advance(self, time: float, h: float, nsteps: int, rcen: float, steps_per_launch: int = 0):
        nev = I(0)
        if self.lib.mercury_b200_mvs_advance(time, h, int(nsteps), rcen, int(steps_per_launch), C.byref(nev)) != 0:
            raise BackendError("CUDA integration step failed")
        # every record is written by the library: no need to clear the arrays
        events = np.empty(nev.value, dtype=EVENT_DTYPE)
        steps = np.empty(nev.value, dtype=np.int32)
        if nev.value:
            self.lib.mercury_b200_events(events.ctypes.data_as(C.c_void_p), steps.ctypes.data_as(PI), nev.value)
        return events, steps

    def mvs_run(self, sys: System, time: float, h: float, nsteps: int, rcen: float, steps_per_launch: int = 0,
                ngflag: int | None = None, out=None):
        """upload(sys) + mvs_advance + download() in one library call
        (mercury_b200_mvs_run): with page-locked host arrays (sys's and `out`'s)
        the particles' copies overlap their steps. Returns (events, steps, x, v)."""
        self.n, self.nbig = sys.n, sys.nbig
        flag = sys.ngflag if ngflag is None else int(ngflag)
        if out is None:
            out = (np.empty((sys.n, 3)), np.empty((sys.n, 3)))
        x, v = out
        assert x.shape == v.shape == (sys.n, 3) and x.dtype == v.dtype == np.float64
        nev = I(0)
        if self.lib.mercury_b200_mvs_run(sys.n, sys.nbig, int(sys.pn), flag, _p(sys.m), _p(sys.x), _p(sys.v),
                                         _p(sys.ngf), _p(sys.jcen), _p(sys.rce), _p(sys.rphys), time, h,
                                         int(nsteps), rcen, int(steps_per_launch), _p(x), _p(v),
                                         C.byref(nev)) != 0:
            raise BackendError("CUDA integration step failed")
        events = np.empty(nev.value, dtype=EVENT_DTYPE)
        steps = np.empty(nev.value, dtype=np.int32)
        if nev.value:
            self.lib.mercury_b200_events(events.ctypes.data_as(C.c_void_p), steps.ctypes.data_as(PI), nev.value)
        return events, steps, x, v

    def timing(self):
        a, k, n, L = D(0.0), D(0.0), I(0), I(0)
        self.lib.mercury_b200_timing(C.byref(a), C.byref(k), C.byref(n), C.byref(L))
        return {"advance_ms": a.value, "particle_kernel_ms": k.value, "particle_launches": n.value,
                "kernel_launches": L.value}

    def advance_launches(self):
        """[(steps, particle-kernel ms)] of each launch of the last fused run."""
        n = self.lib.mercury_b200_advance_launches(None, None, 0)
        steps = np.zeros(max(1, n), dtype=np.int32)
        ms = np.zeros(max(1, n))
        self.lib.mercury_b200_advance_launches(steps.ctypes.data_as(PI), _p(ms), n)
        return [(int(steps[k]), float(ms[k])) for k in range(n)]

    def dropin_time(self, reset: bool = False):
        """(device ms, kernels launched) of the drop-in step/events calls since the last reset."""
        ms, n = D(0.0), C.c_int64(0)
        self.lib.mercury_b200_dropin_time(C.byref(ms), C.byref(n), int(reset))
        return ms.value, n.value

    def energy(self, h: float = 0.0, physical: bool = False, spin: np.ndarray | None = None):
        """(e, l2) of mxx_en on the state export(h, physical) returns; spin is
        (n, 3) or None."""
        e, l2 = D(0.0), D(0.0)
        sp = None if spin is None else np.ascontiguousarray(spin, dtype=np.float64)
        if self.lib.mercury_b200_energy(float(h), int(physical), _p(sp) if sp is not None else None,
                                        C.byref(e), C.byref(l2)) != 0:
            raise BackendError("energy check failed")
        return e.value, l2.value

    def ejections(self, h: float, physical: bool, rmax: float, i0: int = 2, cap: int | None = None) -> np.ndarray:
        """mxx_ejec's test on the device: ascending 1-based ids of the bodies
        j >= i0 beyond rmax (positions as export(h, physical) returns them)."""
        cap = self.n if cap is None else cap
        ids = np.zeros(max(1, cap), dtype=np.int32)
        count = C.c_int(0)
        if self.lib.mercury_b200_ejections(h, int(physical), rmax, i0, ids.ctypes.data_as(PI), cap,
                                           C.byref(count)) != 0:
            raise BackendError("ejection screen failed")
        return ids[:min(count.value, cap)].copy()

    def set_step_reduce(self, fn) -> None:
        """Install (a REDUCE_FN callback, kept alive by the caller) or clear
        (None) the cross-process reduction of the adaptive step control."""
        self._reduce = fn
        self.lib.mercury_b200_set_step_reduce(C.cast(fn, C.c_void_p) if fn is not None else None, None)

    def fp64_peak(self):
        tf, ms = D(0.0), D(0.0)
        if self.lib.mercury_b200_fp64_peak(C.byref(tf), C.byref(ms)) != 0:
            raise BackendError("FP64 peak probe failed")
        return tf.value

    def set_launch(self, threads: int = -1, steps_per_launch: int = -1) -> None:
        if self.lib.mercury_b200_set_launch(int(threads), int(steps_per_launch)) != 0:
            raise BackendError("invalid launch shape")


class Batch:
    """Batched MVS systems (the mercury_b200_batch_* extension): many
    independent systems, each with its own Big bodies, particles and step,
    advanced together. Systems are given as System objects (massless Small
    bodies, no non-gravitational forces, no oblateness)."""

    def __init__(self, systems, h, lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        self.systems = list(systems)
        self.h = np.ascontiguousarray(h, dtype=np.float64)
        sizes = [s.n for s in self.systems]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
        self.nbig = np.array([s.nbig for s in self.systems], dtype=np.int32)
        cat = lambda name: np.ascontiguousarray(np.concatenate([getattr(s, name) for s in self.systems]))
        self.m, self.x, self.v = cat("m"), cat("x"), cat("v")
        self.rce, self.rphys = cat("rce"), cat("rphys")
        rc = self.lib.mercury_b200_batch_upload(len(self.systems), self.offsets.ctypes.data_as(PI),
                                                self.nbig.ctypes.data_as(PI), _p(self.h), _p(self.m), _p(self.x),
                                                _p(self.v), _p(self.rce), _p(self.rphys))
        if rc != 0:
            raise BackendError("batched upload failed")

    def set(self, threads: int = -1, steps_per_launch: int = -1, graph: int = -1) -> None:
        if self.lib.mercury_b200_batch_set(int(threads), int(steps_per_launch), int(graph)) != 0:
            raise BackendError("invalid batched launch shape")

    def advance(self, time: float, nsteps: int, rcen: float):
        """Returns (events, system of each, step of each)."""
        nev = I(0)
        if self.lib.mercury_b200_batch_advance(time, int(nsteps), rcen, C.byref(nev)) != 0:
            raise BackendError("batched advance failed")
        ev = np.zeros(nev.value, dtype=EVENT_DTYPE)
        sy = np.zeros(nev.value, dtype=np.int32)
        st = np.zeros(nev.value, dtype=np.int32)
        if nev.value:
            self.lib.mercury_b200_batch_events(ev.ctypes.data_as(C.c_void_p), sy.ctypes.data_as(PI),
                                               st.ctypes.data_as(PI), nev.value)
        return ev, sy, st

    def download(self):
        """(x, v) of every system, as a list of (n_s, 3) array pairs."""
        x = np.zeros_like(self.x)
        v = np.zeros_like(self.v)
        if self.lib.mercury_b200_batch_download(_p(x), _p(v)) != 0:
            raise BackendError("batched download failed")
        o = self.offsets
        return [(x[o[k]:o[k + 1]], v[o[k]:o[k + 1]]) for k in range(len(self.systems))]

    def timing(self):
        ms, n, t, k = D(0.0), I(0), I(0), I(0)
        self.lib.mercury_b200_batch_timing(C.byref(ms), C.byref(n), C.byref(t), C.byref(k))
        return {"ms": ms.value, "launches": n.value, "threads": t.value, "steps_per_launch": k.value}

    def free(self) -> None:
        self.lib.mercury_b200_batch_free()
