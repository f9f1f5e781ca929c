"""Throughput of the MVS test-particle step on B200 (one JSON line on rank 0).

Workload: the 1,000,000-particle FP64 MVS system of the path's benchmark
configuration (central mass 1 Msun, 8 Big bodies log-uniform 1.7e-7..1e-3
Msun at a 0.39..30 AU, particles a U[0.5,5] AU e U[0,0.2] i U[0,10 deg], 1%
placed inside 5 Hill radii of a planet, h = 8 d, close-encounter screen at 3
Hill radii, central-impact screen at rcen = 0.005 AU), seeded synthetic data.
A bench "step" is one MVS step (kick, Kepler drift, mce_stat/mce_cent screen,
kick) of every particle, events included.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload mvs|radau|bs|bs2]

--impl reference times the reference's CPU algorithm for this path (the C++
restatement of mercury6_2.for in oracle/, all host cores) on the same
workload; under torchrun only rank 0 runs it.

--workload hybrid measures HYBRID (mdt_hy through mercury_cuda_hybrid_begin /
_finish, the encounter members' BS2 subsystem driven as mdt_hkce drives it,
central-impact screen every step) on the MVS workload's system, rcrit from
mce_init (cefac 3); a step is one HYBRID step.

--workload dropin measures the per-step drop-in calls on the MVS workload
(mercury_cuda_step + mercury_cuda_events per step, as mal_hcon makes them;
wall clock), with the reference's CUDA backend making the same calls beside
it.

--workload batch measures the batched extension: 4096 independent systems
(1-8 planets, log-uniform 10-5000 particles, h uniform 4-16 d, 3.3M particles
in all) advanced together; the plain loop over systems through the
single-system path is timed on a sample beside it.

--workload adjoint measures the gradient of sum |x_final|^2 with respect to
every particle's initial state and Yarkovsky coefficient (forward with a
checkpoint every 50 steps, then the reverse sweep) on 100,000 particles for
--steps MVS steps (1,000 for the gradient benchmark); a step is one forward
plus one backward particle-step.

--workload radau|bs|bs2 measures the adaptive integrators instead (mdt_ra15,
mdt_bs1, mdt_bs2 through the drop-in step/events calls, as mal_hvar drives
them) on the 100,000-particle system of the same generator with 1PN,
radiation pressure (beta U[0.01,0.3]) and Yarkovsky (yar log-U[1e-15,1e-13],
random sign), tol 1e-12; a step is one accepted integrator step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from mercuda_b200.shards import Ranks, ShardedRun  # noqa: E402

METRIC = "MVS particle-steps/s"
UNIT = "particle-steps/s"
H = 8.0
RCEN = 0.005
# Algorithmic FP64 operations per particle-step of this workload (each +,-,*,/,
# sqrt counts one), tallied by running the oracle with its counting scalar on
# 20,000 particles of the same generator for 20 steps (oracle.count_mvs):
# 158.4 add + 178.5 mul + 26.6 div + 12.5 sqrt (+0.034 libm calls).
FLOPS_PER_PARTICLE_STEP = 376.06
# Bytes per particle-step if every step read and wrote x, v (and nothing else).
BYTES_PER_PARTICLE_STEP = 96.0
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum, MB) of one
# launch of the particle kernel on this 1M-particle workload, by steps per
# launch, from ncu captures of this bench's own command (the launch list and
# traffic summary of the particle kernel are kept beside the sources).
TRAFFIC_MB_PER_LAUNCH = {31: (99.764224, 157.014528), 20: (99.714304, 127.000576), 16: (99.467776, 104.21376)}
# The FP64 pipe of the same captures: sm__pipe_fp64_cycles_active (fraction
# of peak sustained), sm__inst_executed_pipe_fp64 per particle-step (warp
# instructions x 32), smsp__issue_active (fraction), by steps per launch.
FP64_PIPE_BY_K = {20: (0.4949, 730.4, 0.5463), 16: (0.4981, 729.3, 0.5397)}
CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def compact_steps(steps):
    """Launch sizes as runs: [7, 31, 31, 6] -> "7 + 2x31 + 6"."""
    parts, k = [], 0
    while k < len(steps):
        j = k
        while j < len(steps) and steps[j] == steps[k]:
            j += 1
        parts.append(f"{j - k}x{steps[k]}" if j - k > 1 else str(steps[k]))
        k = j
    return " + ".join(parts)


def config_of(args, text, **extra):
    """The workload's config, the same dict in both arms (the reference arm
    states the sample it could time in its cpu_baseline instead)."""
    cfg = {"workload": text, "particles_per_gpu": args.particles, "seed": args.seed}
    cfg.update(extra)
    return cfg


MVS_TEXT = ("MVS, {n} massless particles + 8 planets per GPU, h=8 d, 1% near planets, encounter + central screens "
            "every step")
MVS_L2 = "state 9 doubles/particle double-buffered (144 MB) > 126 MB L2; each launch reads and writes it once"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=4570)
    p.add_argument("--warmup", type=int, default=46)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--particles", type=int, default=1_000_000)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--steps-per-launch", type=int, default=0)
    p.add_argument("--threads", type=int, default=0)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the batched and adjoint summaries of the default MVS line and the reference-GPU "
                        "comparisons of the adaptive and HYBRID lines")
    p.add_argument("--workload", default="mvs", choices=["mvs", "dropin", "radau", "bs", "bs2", "hybrid", "batch",
                                                         "adjoint", "hybrid_adjoint"])
    p.add_argument("--checkpoint-every", type=int, default=50)
    p.add_argument("--systems", type=int, default=4096)
    args = p.parse_args()
    if args.workload in ADAPTIVE and args.particles == 1_000_000:
        args.particles = 100_000
    if args.workload == "adjoint" and args.particles == 1_000_000:
        args.particles = 100_000
    if args.workload == "hybrid_adjoint" and args.particles == 1_000_000:
        args.particles = 20_000
    return args


def workload(particles: int, seed: int, near_fraction: float = 0.01, rank: int = 0):
    """Rank `rank`'s shard of the job's system: the planets of `seed` on every
    rank, the particles of rank 0 from the same generator (the one-GPU
    workload) and those of rank r > 0 from the seed (seed, r)."""
    from mercuda_b200.system import make_system
    return make_system(seed=seed, n_particles=particles, near_fraction=near_fraction, h=H,
                       particle_seed=None if rank == 0 else (seed, rank))


# HYBRID's encounter members go through BS2 at tol 1e-12 without collision
# handling; the MVS workload's deep near-planet placements (down to a small
# fraction of a Hill radius) make that subsystem crawl, so HYBRID runs the same
# generator without them: its encounters are the natural ones (about 1% of the
# particles within rcrit of a planet each step).
HYBRID_NEAR = 0.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={CLOCK_QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(particles: int, steps: int, seed: int):
    """The oracle (CPU restatement of the reference path) on all host cores."""
    from oracle import oracle as O
    sysc = workload(particles, seed)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    O.mvs_run(sysc, 0.0, H, steps, RCEN, central=True, threads=cores)
    dt = time.perf_counter() - t0
    return particles * steps / dt, cores, dt


_PINNED_KEEP = []


def pinned_like(a: np.ndarray) -> np.ndarray:
    """A copy of a in page-locked host memory (torch's pinned allocator), the
    host buffers of the end-to-end measurement: their copies run by DMA."""
    import torch
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    _PINNED_KEEP.append(t)
    out = t.numpy()
    out[...] = a
    return out


def pinned_system(s):
    """The system with its host arrays in page-locked memory."""
    p = s.copy()
    for name in ("m", "x", "v", "ngf", "rce", "rphys", "rcrit"):
        setattr(p, name, pinned_like(getattr(s, name)))
    return p


def h2d_bytes(s) -> int:
    """Bytes mercury_cuda_upload copies host -> device: x, v, m, rce, rphys,
    and ngf when a force law reads it (ngflag != 0)."""
    return s.n * (3 + 3 + 1 + 1 + 1 + (5 if s.ngflag else 0)) * 8


def one_step_parity(lib, particles: int, seed: int):
    """Parity of this run's workload, checked beside the CPU leg: the whole
    system stepped once through the drop-in calls (step + events) against the
    oracle's step of the same arrays. Returns the worst relative error of the
    states, the share of bodies bit-identical to the oracle, and whether the
    event lists (ids, kinds, order) are identical."""
    from mercuda_b200.backend import Backend
    from oracle import oracle as O
    sysw = workload(particles, seed)
    b = Backend("MVS", lib=lib)
    b.configure()
    b.upload(sysw)
    b.step(0.0, H, dtflag=0)
    x, v = b.download()
    ev = b.events(H, H, RCEN)
    b.free()
    ref = sysw.copy()
    rev, _ = O.mvs_run(ref, 0.0, H, 1, RCEN, central=True, threads=os.cpu_count() or 1)

    def rel(a, r):
        scale = np.maximum(np.linalg.norm(r, axis=1, keepdims=True), 1e-300)
        return float(np.max(np.abs(a - r) / scale))

    key = lambda e: (int(e["i"]), int(e["j"]), int(e["kind"]), int(e["now"]))
    same = np.all(x == ref.x, axis=1) & np.all(v == ref.v, axis=1)
    return {"max_rel_err_one_step": max(rel(x, ref.x), rel(v, ref.v)), "bitwise_fraction": float(same.mean()),
            "pairs_equal": [key(e) for e in ev] == [key(e) for e in rev], "events": int(len(rev)),
            "n_checked": int(sysw.n), "bar": 1e-12}


def run_reference(args, rank, metric: str | None = None):
    if rank != 0:
        return
    metric = metric or METRIC
    cores = os.cpu_count() or 1
    # Bounded sample of the workload per timed run: at ~4.5e6 particle-steps/s
    # per core the full 1M-particle system would take K*0.22 s/cores.
    budget_s = 120.0
    est = args.particles * (args.steps + args.warmup) / (4.0e6 * cores)
    particles = args.particles if est <= budget_s else max(1000, int(args.particles * budget_s / est))
    from oracle import oracle as O
    sysc = workload(particles, args.seed)
    O.mvs_run(sysc, 0.0, H, args.warmup, RCEN, central=True, threads=cores)
    t0 = time.perf_counter()
    O.mvs_run(sysc, args.warmup * H, H, args.steps, RCEN, central=True, threads=cores)
    dt = time.perf_counter() - t0
    value = particles * args.steps / dt
    sample = f"{particles} particles of the same generator x {args.steps} steps (after {args.warmup} warm-up)"
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_of(args, MVS_TEXT.format(n=args.particles), h_days=H, l2=MVS_L2),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    gpu = reference_cuda_rate(args)
    if gpu is not None:
        line["reference_cuda"] = gpu
    print(json.dumps(line), flush=True)


REF_CUDA = Path(__file__).resolve().parent / "oracle" / "_ref" / "libmercury_cuda_ref.so"
DROPIN_STEPS = 46


def dropin_steps(lib, sysw, nsteps, warm=2):
    """Upload sysw and time nsteps drop-in MVS steps (mercury_cuda_step +
    mercury_cuda_events per step, as mal_hcon makes them) by wall clock: the
    calls are synchronous. Returns particle-steps/s of the massless bodies."""
    import ctypes
    D_, I_ = ctypes.c_double, ctypes.c_int
    PD_ = ctypes.POINTER(D_)
    lib.mercury_cuda_upload.argtypes = [I_, I_, I_, I_, PD_, PD_, PD_, PD_, PD_, PD_, PD_]
    lib.mercury_cuda_step.argtypes = [D_, PD_, PD_, D_, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    lib.mercury_cuda_events.argtypes = [D_, D_, D_, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(I_)]
    lib.mercury_cuda_reset.argtypes = [I_]
    lib.mercury_cuda_reset.restype = None
    lib.mercury_cuda_free.restype = None
    arrays = [np.ascontiguousarray(a, dtype=np.float64) for a in (sysw.m, sysw.x, sysw.v, sysw.ngf, sysw.jcen,
                                                                  sysw.rce, sysw.rphys)]
    ptr = [a.ctypes.data_as(PD_) for a in arrays]
    if lib.mercury_cuda_configure(1) != 0 or lib.mercury_cuda_upload(sysw.n, sysw.nbig, 0, sysw.ngflag, *ptr) != 0:
        raise RuntimeError("drop-in upload failed")
    t, t0 = 0.0, None
    for k in range(warm + nsteps):
        if k == warm:
            t0 = time.perf_counter()
        lib.mercury_cuda_reset(0 if k == 0 else 2)
        hh, hd = D_(H), D_(0.0)
        nf, nr = ctypes.c_int64(0), ctypes.c_int64(0)
        if lib.mercury_cuda_step(t, ctypes.byref(hh), ctypes.byref(hd), 0.0, ctypes.byref(nf), ctypes.byref(nr)):
            raise RuntimeError("drop-in step failed")
        evp, cnt = ctypes.c_void_p(), I_(0)
        if lib.mercury_cuda_events(t + H, H, RCEN, ctypes.byref(evp), ctypes.byref(cnt)):
            raise RuntimeError("drop-in events failed")
        t = t + H
    dt = time.perf_counter() - t0
    lib.mercury_cuda_free()
    return (sysw.n - sysw.nbig) * nsteps / dt


DROPIN_METRIC = "MVS drop-in particle-steps/s"


def run_dropin(args, rank, world, dist):
    """The per-step drop-in path on the MVS workload: mercury_cuda_step +
    mercury_cuda_events per step as mal_hcon makes them (synchronous calls,
    wall clock, max over ranks), with the reference's CUDA backend making the
    same calls on this GPU beside it."""
    if args.impl == "reference":
        run_reference(args, rank, DROPIN_METRIC)
        return
    import ctypes
    import torch
    from mercuda_b200.backend import load_library
    lib = load_library()
    ranks = Ranks(dist, device="cuda")
    sysw = workload(args.particles, args.seed, rank=rank)
    ms0, n0 = ctypes.c_double(0.0), ctypes.c_int64(0)
    lib.mercury_b200_dropin_time(ctypes.byref(ms0), ctypes.byref(n0), 1)
    ranks.barrier()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        rate = dropin_steps(lib, sysw, args.steps, warm=max(3, args.warmup))
    ranks.barrier()
    ms, launches = ctypes.c_double(0.0), ctypes.c_int64(0)
    lib.mercury_b200_dropin_time(ctypes.byref(ms), ctypes.byref(launches), 0)
    wall_s = ranks.max(args.particles * args.steps / rate)
    value = world * args.particles * args.steps / wall_s
    ref_gpu = None
    if world == 1 and not args.no_extras:
        ref_lib = load_reference_cuda()
        if ref_lib is not None:
            theirs = dropin_steps(ref_lib, workload(args.particles, args.seed), args.steps, warm=max(3, args.warmup))
            ref_gpu = {"value": theirs, "unit": UNIT, "steps": args.steps, "ratio_vs_reference_cuda": value / theirs,
                       "note": "the reference's CUDA backend through the same calls on this GPU, wall clock"}
    if rank == 0:
        text = (f"MVS per-step drop-in calls (mercury_cuda_step + mercury_cuda_events), {args.particles} massless "
                "particles + 8 planets per GPU, h=8 d, 1% near planets, encounter + central screens every step")
        print(json.dumps({"metric": DROPIN_METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                          "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": wall_s * 1e3 / args.steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": config_of(args, text, h_days=H, l2=MVS_L2),
                          "clocks": clocks.summary(), "gpu_launches": launches.value,
                          "e2e": None, "reference_cuda": ref_gpu}), flush=True)


def load_reference_cuda():
    """The reference's CUDA backend (mercury_cuda.cu built unchanged for
    sm_100a into oracle/_ref by oracle/Makefile's ref target) with the
    argument types of its 16 drop-in entry points; None without a GPU or the
    built library."""
    if not REF_CUDA.exists():
        return None
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except ImportError:
        return None
    import ctypes
    D_, I_ = ctypes.c_double, ctypes.c_int
    PD_, PI_, P64 = ctypes.POINTER(D_), ctypes.POINTER(I_), ctypes.POINTER(ctypes.c_int64)
    L = ctypes.CDLL(str(REF_CUDA))
    L.mercury_cuda_available.restype = I_
    L.mercury_cuda_configure.argtypes = [I_]
    L.mercury_cuda_reset.argtypes = [I_]
    L.mercury_cuda_reset.restype = None
    L.mercury_cuda_limits.argtypes = [PD_]
    L.mercury_cuda_export.argtypes = [D_, I_, PD_, PD_]
    L.mercury_cuda_upload.argtypes = [I_, I_, I_, I_, PD_, PD_, PD_, PD_, PD_, PD_, PD_]
    L.mercury_cuda_step.argtypes = [D_, PD_, PD_, D_, P64, P64]
    L.mercury_cuda_download.argtypes = [PD_, PD_, I_]
    L.mercury_cuda_events.argtypes = [D_, D_, D_, ctypes.POINTER(ctypes.c_void_p), PI_]
    L.mercury_cuda_force.argtypes = [PD_]
    L.mercury_cuda_hybrid_begin.argtypes = [D_, PD_, I_, I_, PI_, PI_, PI_, PI_, PD_, PD_, P64]
    L.mercury_cuda_hybrid_finish.argtypes = [D_, PD_, PD_, PD_, P64]
    L.mercury_cuda_encounter_enter.argtypes = [I_, I_, PD_, PD_, PD_, PD_, PD_, PD_, I_, PI_, PI_]
    L.mercury_cuda_encounter_update.argtypes = [PD_, PD_, PD_]
    L.mercury_cuda_encounter_exit.restype = None
    L.mercury_cuda_free.restype = None
    return L if L.mercury_cuda_available() else None


def adaptive_wall_rate(lib, name, sysw, warmup, steps):
    """Wall-clock particle-steps/s of the drop-in step + events calls as
    mal_hvar makes them (synchronous calls), after `warmup` steps."""
    from mercuda_b200.backend import Backend
    b = Backend(name, lib=lib)
    b.configure()
    b.upload(sysw)
    t, h, dtflag = 0.0, ADAPTIVE_H0, 0
    for k in range(warmup + steps):
        if k == warmup:
            t0 = time.perf_counter()
        hdid, h = b.step(t, h, ADAPTIVE_TOL, dtflag)
        dtflag = 2
        t = t + hdid
        b.events(t, hdid, RCEN)
    dt = time.perf_counter() - t0
    b.free()
    return (sysw.n - sysw.nbig) * steps / dt


def hybrid_wall_rate(lib, sysw, warmup, steps, fused):
    """Wall-clock particle-steps/s of HYBRID steps through the drop-in calls
    (hybrid_begin, the encounter subsystem as mdt_hkce drives it, hybrid_finish,
    the central screen), after `warmup` steps."""
    from mercuda_b200.backend import Backend
    b = Backend("HYBRID", lib=lib)
    b.configure()
    b.upload(sysw)
    state, t = {"dtflag": 0}, 0.0
    for k in range(warmup + steps):
        if k == warmup:
            t0 = time.perf_counter()
        b.hybrid_step(sysw, t, H, 1e-12, state, RCEN, fused=fused)
        t = t + H
        b.events(t, H, RCEN)
    dt = time.perf_counter() - t0
    b.free()
    return (sysw.n - sysw.nbig) * steps / dt


def reference_cuda_rate(args):
    """The reference's own CUDA backend (its mercury_cuda.cu built unchanged
    for sm_100a into oracle/_ref by oracle/Makefile's ref target) stepping the
    same workload on this GPU through its C ABI, one drop-in step and events
    call per step: the existing GPU code this path replaces. None without a
    GPU or without the built library."""
    if not REF_CUDA.exists():
        return None
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except ImportError:
        return None
    import ctypes
    lib = ctypes.CDLL(str(REF_CUDA))
    value = dropin_steps(lib, workload(args.particles, args.seed), DROPIN_STEPS)
    return {"value": value, "unit": UNIT, "steps": DROPIN_STEPS, "particles": args.particles,
            "note": "the reference's CUDA backend on this GPU: mercury_cuda_step + mercury_cuda_events per step, "
                    "wall clock (synchronous calls)"}


ADAPTIVE = {"radau": ("RADAU", 4), "bs": ("BS", 2), "bs2": ("BS2", 3)}
ADAPTIVE_TOL = 1e-12
ADAPTIVE_H0 = 2.0


def adaptive_workload(particles: int, seed: int, rank: int = 0):
    sys_ = workload(particles, seed, 0.0, rank)
    rng = np.random.default_rng(seed + 1000 if rank == 0 else (seed + 1000, rank))
    npart = sys_.n - sys_.nbig
    sys_.ngf[sys_.nbig:, 3] = rng.uniform(0.01, 0.3, npart)
    sys_.ngf[sys_.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
    sys_.pn = 1
    return sys_


def adaptive_cpu(name: str, particles: int, steps: int, seed: int):
    """The oracle's mal_hvar loop (single-threaded, as the Fortran) on a sample."""
    from oracle import oracle as O
    sysc = adaptive_workload(particles, seed)
    t0 = time.perf_counter()
    _, _, _, done, _, _ = O.hvar_run(sysc, ADAPTIVE[name][1], 0.0, 1e9, ADAPTIVE_H0, ADAPTIVE_TOL, RCEN,
                                     max_steps=steps)
    dt = time.perf_counter() - t0
    return particles * done / dt, done, dt


def run_adaptive(args, rank, world, dist):
    name, alg = ADAPTIVE[args.workload]
    metric = f"{name} particle-steps/s"
    workload_text = (f"{name}, {args.particles} massless particles + 8 planets, 1PN, PR beta U[0.01,0.3], "
                     "yar log-U[1e-15,1e-13] random sign, tol 1e-12, encounter + central screens every step")
    if args.impl == "reference":
        if rank != 0:
            return
        particles = min(args.particles, 20_000)
        value, done, dt = adaptive_cpu(args.workload, particles, args.steps, args.seed)
        sample = f"{particles} particles of the same generator x {done} accepted steps ({dt:.1f} s, 1 thread)"
        line = {"impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": done, "warmup": 0, "ms_per_step": dt * 1e3 / max(1, done), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config_of(args, workload_text),
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch
    from mercuda_b200.backend import Backend

    b = Backend(name)
    b.configure()
    sysw = adaptive_workload(args.particles, args.seed, rank)
    b.upload(sysw)

    ranks = Ranks(dist, device="cuda")
    barrier = ranks.barrier

    def run(time0, h, nsteps):
        t, dtflag, nev = time0, 0, 0
        for _ in range(nsteps):
            hdid, h = b.step(t, h, ADAPTIVE_TOL, dtflag)
            dtflag = 2
            t = t + hdid
            nev += len(b.events(t, hdid, RCEN))
        return t, h, nev

    t, h, _ = run(0.0, ADAPTIVE_H0, args.warmup)
    b.dropin_time(reset=True)
    barrier()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        t, h, nev = run(t, h, args.steps)
    barrier()
    ms, launches = b.dropin_time(reset=True)
    ms = ranks.max(ms)
    value = world * args.particles * args.steps / (ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        fresh = pinned_system(adaptive_workload(args.particles, args.seed, rank))
        out = (pinned_like(np.zeros((fresh.n, 3))), pinned_like(np.zeros((fresh.n, 3))))
        flag = fresh.ngflag
        barrier()
        t0 = time.perf_counter()
        b.upload(fresh, flag)
        run(0.0, ADAPTIVE_H0, args.steps)
        x, v = b.download(out=out)
        barrier()
        e2e_s = time.perf_counter() - t0
        e2e_s = ranks.max(e2e_s)
        h2d = h2d_bytes(fresh)
        e2e = {"value": world * args.particles * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": fresh.n * 48 / args.steps,
               "note": "wall clock around upload, the drop-in step + events calls of every step, download"}
    ref_gpu = None
    if world == 1 and not args.no_extras:
        # like for like with the reference's own CUDA backend on this GPU: the
        # same drop-in calls on the same workload, wall clock for both
        ref_lib = load_reference_cuda()
        if ref_lib is not None:
            steps_cmp = min(args.steps, 10)
            ours = adaptive_wall_rate(b.lib, name, adaptive_workload(args.particles, args.seed), 2, steps_cmp)
            theirs = adaptive_wall_rate(ref_lib, name, adaptive_workload(args.particles, args.seed), 2, steps_cmp)
            ref_gpu = {"value": theirs, "unit": UNIT, "steps": steps_cmp, "dropin_wall": ours,
                       "ratio_vs_reference_cuda": ours / theirs,
                       "note": "the reference's CUDA backend and this library through the same drop-in step + "
                               "events calls on this GPU, wall clock"}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        particles = min(args.particles, 20_000)
        v_cpu, done, dt = adaptive_cpu(args.workload, particles, 40, args.seed)
        cpu = {"value": v_cpu, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{particles} particles of the same generator x {done} accepted steps ({dt:.1f} s)"}
    if rank == 0:
        line = {"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config_of(args, workload_text),
                "run": {"h_last": h, "t_end_days": t,
                        "l2": "per step the state, B/E (RA15) or candidates (BS) exceed 126 MB only above "
                              "~300K particles; measured as is"},
                "clocks": clocks.summary(), "gpu_launches": launches, "events": nev, "e2e": e2e,
                "cpu_baseline": cpu}
        if ref_gpu is not None:
            line["reference_cuda"] = ref_gpu
        print(json.dumps(line), flush=True)
    b.free()


def run_hybrid(args, rank, world, dist):
    from mercuda_b200.system import mce_init
    metric = "HYBRID particle-steps/s"
    workload_text = (f"HYBRID, {args.particles} massless particles + 8 planets, h=8 d, "
                     "rcrit = max(3 Hill, 0.4 h vmax), encounter subsystem by BS2, central screen every step")
    tol = 1e-12
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        particles = min(args.particles, 50_000)
        sysc = mce_init(workload(particles, args.seed, HYBRID_NEAR), H, 3.0)
        t0 = time.perf_counter()
        O.hy_run(sysc, 0.0, H, args.steps, tol, RCEN)
        dt = time.perf_counter() - t0
        value = particles * args.steps / dt
        sample = f"{particles} particles of the same generator x {args.steps} steps ({dt:.1f} s, 1 thread)"
        print(json.dumps({"impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": 0, "ms_per_step": dt * 1e3 / args.steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": config_of(args, workload_text),
                          "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                                           "sample": sample},
                          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    from mercuda_b200.backend import Backend

    b = Backend("HYBRID")
    b.configure()
    sysw = mce_init(workload(args.particles, args.seed, HYBRID_NEAR, rank), H, 3.0)
    b.upload(sysw)
    state = {"dtflag": 0}

    ranks = Ranks(dist, device="cuda")
    barrier = ranks.barrier

    def run(t, nsteps):
        nev = pairs = 0
        for _ in range(nsteps):
            ev, npair = b.hybrid_step(sysw, t, H, tol, state, RCEN)
            t = t + H
            nev += len(ev) + len(b.events(t, H, RCEN))
            pairs += npair
        return t, nev, pairs

    t, _, _ = run(0.0, args.warmup)
    b.dropin_time(reset=True)
    barrier()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        w0 = time.perf_counter()
        t, nev, pairs = run(t, args.steps)
        wall = time.perf_counter() - w0
    barrier()
    ms, launches = b.dropin_time(reset=True)
    ms, wall = ranks.max(ms), ranks.max(wall)
    value = world * args.particles * args.steps / (ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        fresh = pinned_system(mce_init(workload(args.particles, args.seed, HYBRID_NEAR, rank), H, 3.0))
        out = (pinned_like(np.zeros((fresh.n, 3))), pinned_like(np.zeros((fresh.n, 3))))
        flag = fresh.ngflag
        barrier()
        t0 = time.perf_counter()
        b.upload(fresh, flag)
        state = {"dtflag": 0}
        sysw = fresh
        run(0.0, args.steps)
        x, v = b.download(out=out)
        barrier()
        e2e_s = time.perf_counter() - t0
        e2e_s = ranks.max(e2e_s)
        h2d = h2d_bytes(fresh) + fresh.n * 8
        e2e = {"value": world * args.particles * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": fresh.n * 48 / args.steps,
               "note": "wall clock around upload, hybrid_begin, the encounter subsystem, hybrid_finish and the "
                       "central screen of every step, download"}
    ref_gpu = None
    if world == 1 and not args.no_extras:
        # like for like with the reference's own CUDA backend on this GPU: the
        # drop-in HYBRID calls driven as mdt_hy / mdt_hkce drive them, wall clock
        ref_lib = load_reference_cuda()
        if ref_lib is not None:
            steps_cmp = min(args.steps, 3)
            fresh = lambda: mce_init(workload(args.particles, args.seed, HYBRID_NEAR), H, 3.0)
            ours = hybrid_wall_rate(b.lib, fresh(), 1, steps_cmp, fused=True)
            theirs = hybrid_wall_rate(ref_lib, fresh(), 1, steps_cmp, fused=False)
            ref_gpu = {"value": theirs, "unit": UNIT, "steps": steps_cmp, "dropin_wall": ours,
                       "ratio_vs_reference_cuda": ours / theirs,
                       "note": "the reference's CUDA backend (its drop-in calls one by one, as its Fortran host "
                               "makes them) and this library on this GPU, wall clock"}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        particles = min(args.particles, 50_000)
        sysc = mce_init(workload(particles, args.seed, HYBRID_NEAR), H, 3.0)
        t0 = time.perf_counter()
        O.hy_run(sysc, 0.0, H, 40, tol, RCEN)
        dt = time.perf_counter() - t0
        cpu = {"value": particles * 40 / dt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{particles} particles of the same generator x 40 steps ({dt:.1f} s)"}
    if rank == 0:
        print(json.dumps({"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": config_of(args, workload_text),
                          "run": {"encounter_pairs": pairs, "wall_ms_per_step": wall * 1e3 / args.steps},
                          "clocks": clocks.summary(), "gpu_launches": launches, "events": nev, "e2e": e2e,
                          "cpu_baseline": cpu, "reference_cuda": ref_gpu}), flush=True)
    b.free()


def plain_loop_ms(systems, hs, steps, sample_every=8):
    """The plain per-system kernel loop the batched launch replaces: every
    sample_every-th system (a uniform sample of the seeded batch) uploaded to
    the single-system path, one warm-up step, then `steps` fused MVS steps,
    whose device time (CUDA events around the launches,
    mercury_b200_timing) is summed; scaled to the whole batch. Uploads,
    downloads and the warm-up are outside the timed sum."""
    from mercuda_b200.backend import Backend
    be = Backend("MVS")
    be.configure()
    total_ms, count = 0.0, 0
    for k in range(0, len(systems), sample_every):
        be.upload(systems[k])
        be.mvs_advance(0.0, float(hs[k]), 1, RCEN)
        be.mvs_advance(float(hs[k]), float(hs[k]), steps, RCEN)
        total_ms += be.timing()["advance_ms"]
        count += 1
    be.free()
    return total_ms * len(systems) / count, count


def batched_summary(seed: int, steps: int, nsys: int = 4096):
    """The batched extension on the 4,096-system workload beside the MVS line:
    device particle-steps/s of one batched advance (after a tuning + warm-up
    advance), the launch shape the tuner chose, and the speed-up over the
    plain per-system kernel loop."""
    from mercuda_b200.backend import Batch
    from mercuda_b200.system import make_batch
    systems, hs = make_batch(seed=seed + 100, nsys=nsys)
    total = sum(s.n - s.nbig for s in systems)
    b = Batch(systems, hs)
    b.advance(0.0, steps, RCEN)
    b.advance(0.0, steps, RCEN)
    tm = b.timing()
    b.free()
    plain_ms, sampled = plain_loop_ms(systems, hs, steps)
    return {"value": total * steps / (tm["ms"] * 1e-3), "unit": UNIT, "systems": nsys, "particles": total,
            "steps": steps, "batched_ms": tm["ms"], "plain_loop_ms": plain_ms,
            "speedup_vs_plain_loop": plain_ms / tm["ms"], "threads_per_cta": tm["threads"],
            "steps_per_launch": tm["steps_per_launch"], "gpu_launches": tm["launches"],
            "plain_loop_sample": f"{sampled} of {nsys} systems (every 8th), device time of each system's "
                                 f"{steps}-step advance, scaled"}


def adjoint_summary(seed: int, particles: int = 100_000, steps: int = 1000, every: int = 50):
    """The adjoint extension (config 4) beside the MVS line: forward and
    backward device time of dL/d(x0, v0, yar), L = sum |x_final|^2, and the
    gradients of 64 random particles for the oracle check (done by the
    caller beside the CPU leg). Returns (summary, gradients, system, picks)."""
    import torch
    from mercuda_b200.adjoint import mvs_trajectory, timing
    s = workload(particles, seed, 0.0)
    rng = np.random.default_rng(seed + 7)
    npart = s.n - s.nbig
    s.ngf[s.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
    nb = s.nbig
    dev = torch.device("cuda")

    def once():
        x0 = torch.tensor(s.x[nb:], device=dev, requires_grad=True)
        v0 = torch.tensor(s.v[nb:], device=dev, requires_grad=True)
        yar = torch.tensor(s.ngf[nb:, 4], device=dev, requires_grad=True)
        xf, _ = mvs_trajectory(x0, v0, yar, (s.m[:nb], s.x[:nb], s.v[:nb]), H, steps, every)
        (xf ** 2).sum().backward()
        return np.concatenate([x0.grad.cpu().numpy(), v0.grad.cpu().numpy(), yar.grad.cpu().numpy()[:, None]],
                              axis=1)

    once()
    g = once()
    fwd, bwd = timing()
    pick = np.sort(rng.choice(npart, 64, replace=False))
    return ({"particles": particles, "steps": steps, "checkpoint_every": every, "forward_ms": fwd,
             "backward_ms": bwd, "backward_over_forward": bwd / fwd,
             "value": particles * steps / ((fwd + bwd) * 1e-3), "unit": UNIT}, g[pick], s, pick)


def adjoint_oracle_error(s, pick, got, steps: int = 1000):
    """Worst relative error of the picked particles' gradients (per block:
    position, velocity, yar) against the oracle's FP64 tangent map, over the
    particles whose trajectories are well conditioned: a relative change of
    1e-15 in the initial positions stays below 1e-9 in the final ones. The
    others (close planetary approaches) amplify rounding by 1e6 and more, so
    two FP64 evaluations in different orders legitimately differ there; they
    are counted, not compared."""
    from oracle import oracle as O
    nb = s.nbig
    sub = s.copy()
    keep = np.concatenate([np.arange(nb), nb + pick])
    for name in ("m", "x", "v", "ngf", "rce", "rphys", "rcrit", "rceh", "rho"):
        setattr(sub, name, getattr(s, name)[keep].copy())
    a, b = sub.copy(), sub.copy()
    b.x[nb:] *= 1.0 + 1e-15
    O.mvs_run(a, 0.0, H, steps, RCEN, central=False, threads=os.cpu_count() or 1)
    O.mvs_run(b, 0.0, H, steps, RCEN, central=False, threads=os.cpu_count() or 1)
    spread = np.abs(a.x[nb:] - b.x[nb:]).max(axis=1) / np.abs(a.x[nb:]).max(axis=1)
    calm = spread < 1e-9
    J = O.mvs_jacobian(sub, H, steps)
    xf = sub.x[nb:]
    want = np.einsum("prk,pr->pk", J, np.concatenate([2 * xf, np.zeros_like(xf)], axis=1))
    worst = 0.0
    for cols in (slice(0, 3), slice(3, 6), slice(6, 7)):
        scale = np.abs(want[calm, cols]).max(axis=1, keepdims=True)
        worst = max(worst, float(np.max(np.abs(got[calm, cols] - want[calm, cols]) / scale)))
    return worst, int((~calm).sum())


def run_batch(args, rank, world, dist):
    from mercuda_b200.system import make_batch
    metric = "batched MVS particle-steps/s"
    systems, hs = make_batch(seed=args.seed + 100 * rank, nsys=args.systems)
    total = sum(s.n - s.nbig for s in systems)
    workload_text = (f"batched MVS, {args.systems} systems per GPU, 1-8 planets, 10-5000 particles log-uniform "
                     f"({total} particles), h U[4,16] d, encounter + central screens every step")
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        sample = systems[:: max(1, len(systems) // 256)]
        t0 = time.perf_counter()
        done = 0
        for sys_, h_ in zip(sample, hs[:: max(1, len(systems) // 256)]):
            O.mvs_run(sys_, 0.0, float(h_), args.steps, RCEN, central=True, threads=cores)
            done += (sys_.n - sys_.nbig) * args.steps
        dt = time.perf_counter() - t0
        value = done / dt
        print(json.dumps({"impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": 0, "ms_per_step": dt * 1e3 / args.steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic",
                          "config": config_of(args, workload_text, systems_per_gpu=args.systems,
                                              particles_per_gpu=total),
                          "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                                           "sample": f"{len(sample)} of the systems x {args.steps} steps"},
                          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    import torch
    from mercuda_b200.backend import Backend, Batch

    ranks = Ranks(dist, device="cuda")
    barrier = ranks.barrier

    b = Batch(systems, hs)
    b.advance(0.0, max(1, args.warmup), RCEN)
    barrier()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        ev, _, _ = b.advance(0.0, args.steps, RCEN)
    barrier()
    tm = b.timing()
    ms = tm["ms"]
    ms = ranks.max(ms)
    value = world * total * args.steps / (ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        barrier()
        t0 = time.perf_counter()
        b2 = Batch(systems, hs)
        b2.advance(0.0, args.steps, RCEN)
        b2.download()
        barrier()
        e2e_s = time.perf_counter() - t0
        e2e_s = ranks.max(e2e_s)
        nb = sum(s.n for s in systems)
        e2e = {"value": world * total * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": nb * (3 + 3 + 1 + 1 + 1) * 8 / args.steps,
               "d2h_bytes_per_step": nb * 48 / args.steps,
               "note": "wall clock around the batched upload, advance (events included) and download"}
    b.free()
    # the plain loop: each system through the single-system path in turn
    barrier()
    plain_ms, sampled = plain_loop_ms(systems, hs, args.steps)
    barrier()
    sample = list(zip(systems[::8], hs[::8]))
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        done = 0
        for sys_, h_ in sample[:32]:
            O.mvs_run(sys_.copy(), 0.0, float(h_), args.steps, RCEN, central=True, threads=cores)
            done += (sys_.n - sys_.nbig) * args.steps
        dt = time.perf_counter() - t0
        cpu = {"value": done / dt, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"32 of the systems x {args.steps} steps ({dt:.1f} s)"}
    if rank == 0:
        print(json.dumps({"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": config_of(args, workload_text, systems_per_gpu=args.systems,
                                              particles_per_gpu=total),
                          "run": {"particles": total, "threads_per_cta": tm["threads"],
                                     "steps_per_launch": tm["steps_per_launch"],
                                     "plain_loop_ms": plain_ms, "batched_ms": ms,
                                     "speedup_vs_plain_loop": plain_ms / ms,
                                     "plain_loop_sample": f"{sampled} of {len(systems)} systems (every 8th), "
                                                          "device time of each system's advance, scaled"},
                          "clocks": clocks.summary(), "gpu_launches": tm["launches"], "events": int(len(ev)),
                          "e2e": e2e, "cpu_baseline": cpu}), flush=True)


def run_adjoint(args, rank, world, dist):
    metric = "adjoint MVS particle-steps/s"

    def make(seed, n, rank=0):
        s_ = workload(n, seed, 0.0, rank)
        rng = np.random.default_rng(seed + 7 if rank == 0 else (seed + 7, rank))
        npart = s_.n - s_.nbig
        s_.ngf[s_.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
        return s_

    workload_text = (f"gradient of sum |x_final|^2 w.r.t. initial x, v and yar of {args.particles} particles, "
                     f"{args.steps} MVS steps of 8 d about 8 planets, checkpoint every {args.checkpoint_every}")

    def cpu_sample(n, steps):
        from oracle import oracle as O
        s_ = make(args.seed, n)
        t0 = time.perf_counter()
        O.mvs_jacobian(s_, H, steps)
        dt = time.perf_counter() - t0
        return n * steps / dt, dt

    if args.impl == "reference":
        if rank != 0:
            return
        n = min(args.particles, 2000)
        value, dt = cpu_sample(n, args.steps)
        print(json.dumps({"impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": 0, "ms_per_step": dt * 1e3 / args.steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": config_of(args, workload_text),
                          "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                                           "sample": f"{n} particles x {args.steps} steps, forward-mode tangents "
                                                     f"of the oracle ({dt:.1f} s)"},
                          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    import torch
    from mercuda_b200.adjoint import mvs_trajectory, timing

    sysw = make(args.seed, args.particles, rank)
    nb = sysw.nbig
    dev = torch.device("cuda")
    big = (sysw.m[:nb], sysw.x[:nb], sysw.v[:nb])

    def once(x0h, v0h, yh):
        x0 = torch.tensor(x0h, device=dev, requires_grad=True)
        v0 = torch.tensor(v0h, device=dev, requires_grad=True)
        yar = torch.tensor(yh, device=dev, requires_grad=True)
        xf, _ = mvs_trajectory(x0, v0, yar, big, H, args.steps, args.checkpoint_every)
        (xf ** 2).sum().backward()
        return x0.grad, v0.grad, yar.grad

    ranks = Ranks(dist, device="cuda")
    for _ in range(max(1, args.warmup)):
        once(sysw.x[nb:], sysw.v[nb:], sysw.ngf[nb:, 4])
    ranks.barrier()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        t0 = time.perf_counter()
        g = once(sysw.x[nb:], sysw.v[nb:], sysw.ngf[nb:, 4])
        gx = g[0].cpu().numpy()
        e2e_s = time.perf_counter() - t0
    fwd, bwd = timing()
    ms = fwd + bwd
    ms, e2e_s = ranks.max(ms), ranks.max(e2e_s)
    value = world * args.particles * args.steps / (ms * 1e-3)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v_cpu, dt = cpu_sample(1000, args.steps)
        cpu = {"value": v_cpu, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"1000 particles x {args.steps} steps, forward-mode tangents of the oracle ({dt:.1f} s)"}
    if rank == 0:
        print(json.dumps({"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                          "warmup": max(1, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": config_of(args, workload_text),
                          "run": {"forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
                                     "checkpoint_every": args.checkpoint_every,
                                     "grad_finite": bool(np.all(np.isfinite(gx)))},
                          "clocks": clocks.summary(), "gpu_launches": 3,
                          "e2e": {"value": world * args.particles * args.steps / e2e_s, "unit": UNIT,
                                  "h2d_bytes_per_step": args.particles * 7 * 8 / args.steps,
                                  "d2h_bytes_per_step": args.particles * 3 * 8 / args.steps,
                                  "note": "wall clock around tensor creation from host arrays, the forward and "
                                          "backward calls and the gradient copy back"},
                          "cpu_baseline": cpu}), flush=True)


def run_hybrid_adjoint(args, rank, world, dist):
    """Gradients through HYBRID: forward through the library's HYBRID path
    (host-driven encounter subsystems), backward on the device."""
    from mercuda_b200.system import mce_init
    metric = "adjoint HYBRID particle-steps/s"

    def make(seed, n, rank=0):
        s_ = mce_init(workload(n, seed, HYBRID_NEAR, rank), H, 3.0)
        rng = np.random.default_rng(seed + 7 if rank == 0 else (seed + 7, rank))
        npart = s_.n - s_.nbig
        s_.ngf[s_.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
        return s_

    tol = 1e-12
    workload_text = (f"gradient of sum |x_final|^2 w.r.t. initial x, v and yar of {args.particles} particles, "
                     f"{args.steps} HYBRID steps of 8 d about 8 planets (encounter subsystem by BS2, tol 1e-12), "
                     f"checkpoint every {args.checkpoint_every}")

    def cpu_sample(n, steps):
        from oracle import oracle as O
        s_ = make(args.seed, n)
        t0 = time.perf_counter()
        O.hy_jacobian(s_, H, steps, tol)
        dt = time.perf_counter() - t0
        return n * steps / dt, dt

    if args.impl == "reference":
        if rank != 0:
            return
        n = min(args.particles, 1000)
        value, dt = cpu_sample(n, args.steps)
        print(json.dumps({"impl": "reference", "metric": metric, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": 0, "ms_per_step": dt * 1e3 / args.steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": config_of(args, workload_text),
                          "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                                           "sample": f"{n} particles x {args.steps} steps, forward-mode tangents "
                                                     f"of the oracle's mdt_hy ({dt:.1f} s)"},
                          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return
    import ctypes

    import torch
    from mercuda_b200.adjoint import hybrid_timing, hybrid_trajectory
    from mercuda_b200.backend import load_library

    sysw = make(args.seed, args.particles, rank)
    nb = sysw.nbig
    dev = torch.device("cuda")
    big = (sysw.m[:nb], sysw.x[:nb], sysw.v[:nb], sysw.rcrit[:nb])

    def once():
        x0 = torch.tensor(sysw.x[nb:], device=dev, requires_grad=True)
        v0 = torch.tensor(sysw.v[nb:], device=dev, requires_grad=True)
        yar = torch.tensor(sysw.ngf[nb:, 4], device=dev, requires_grad=True)
        xf, _ = hybrid_trajectory(x0, v0, yar, big, sysw.rcrit[nb:], H, args.steps, tol, args.checkpoint_every)
        (xf ** 2).sum().backward()
        return x0.grad.cpu().numpy()

    ranks = Ranks(dist, device="cuda")
    lib = load_library()

    def dropin(reset):
        """Kernels the drop-in calls launched since the last reset."""
        launched = ctypes.c_int64(0)
        lib.mercury_b200_dropin_time(None, ctypes.byref(launched), int(reset))
        return launched.value

    for _ in range(max(1, args.warmup)):
        once()
    ranks.barrier()
    dropin(True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        t0 = time.perf_counter()
        gx = once()
        e2e_s = time.perf_counter() - t0
    # forward: the drop-in HYBRID calls' kernels; backward: per segment the
    # recompute and VJP kernels and, where members were recorded, their index
    nseg = (args.steps + args.checkpoint_every - 1) // args.checkpoint_every
    launches = dropin(True) + 3 * nseg
    fwd, bwd, members = hybrid_timing()
    ms = fwd + bwd
    ms, e2e_s = ranks.max(ms), ranks.max(e2e_s)
    value = world * args.particles * args.steps / (ms * 1e-3)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        n_cpu = min(args.particles, 500)
        v_cpu, dt = cpu_sample(n_cpu, args.steps)
        cpu = {"value": v_cpu, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{n_cpu} particles x {args.steps} steps, forward-mode tangents of the oracle's mdt_hy "
                         f"({dt:.1f} s)"}
    if rank == 0:
        print(json.dumps({"metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                          "warmup": max(1, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": config_of(args, workload_text),
                          "run": {"forward_wall_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
                                     "member_steps": members, "checkpoint_every": args.checkpoint_every,
                                     "grad_finite": bool(np.all(np.isfinite(gx)))},
                          "clocks": clocks.summary(), "gpu_launches": launches,
                          "e2e": {"value": world * args.particles * args.steps / e2e_s, "unit": UNIT,
                                  "h2d_bytes_per_step": args.particles * 7 * 8 / args.steps,
                                  "d2h_bytes_per_step": args.particles * 3 * 8 / args.steps,
                                  "note": "wall clock around tensor creation from host arrays, the forward and "
                                          "backward calls and the gradient copy back"},
                          "cpu_baseline": cpu}), flush=True)


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    if args.workload != "mvs":
        if args.impl != "reference":
            import torch
            torch.cuda.set_device(local)
        if args.workload == "hybrid":
            run_hybrid(args, rank, world, dist)
        elif args.workload == "dropin":
            run_dropin(args, rank, world, dist)
        elif args.workload == "batch":
            run_batch(args, rank, world, dist)
        elif args.workload == "adjoint":
            run_adjoint(args, rank, world, dist)
        elif args.workload == "hybrid_adjoint":
            run_hybrid_adjoint(args, rank, world, dist)
        else:
            run_adaptive(args, rank, world, dist)
        if dist:
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, rank)
        if dist:
            dist.destroy_process_group()
        return

    import torch
    from mercuda_b200.backend import Backend

    torch.cuda.set_device(local)
    b = Backend("MVS")
    b.configure()
    if args.threads:
        b.set_launch(threads=args.threads)
    # Weak scaling: every rank integrates its own share of the job's
    # particles about the same planets (no data-path collective).
    sysw = workload(args.particles, args.seed, rank=rank)
    b.upload(sysw)
    e_start, l_start = b.energy(H, physical=True)    # mxx_en of the corrected start state
    peak_tflops = b.fp64_peak()
    # warm-up
    if args.warmup > 0:
        b.mvs_advance(0.0, H, args.warmup, RCEN, args.steps_per_launch)
    t_start = args.warmup * H

    ranks = Ranks(dist, device="cuda")
    barrier = ranks.barrier

    barrier()
    with ClockSampler(local) as clocks:
        events, steps = b.mvs_advance(t_start, H, args.steps, RCEN, args.steps_per_launch)
    barrier()
    tm = b.timing()
    e_end, l_end = b.energy(H, physical=True)
    ms = tm["advance_ms"]
    ms = ranks.max(ms)
    value = world * args.particles * args.steps / (ms * 1e-3)
    # the roofline of the run's longest launch (the first is short so that the
    # next launch's Big-body steps run beside its particles)
    launch_list = b.advance_launches()
    steps_per_launch, kernel_ms = max(launch_list) if launch_list else (args.steps, tm["particle_kernel_ms"])
    flops_per_launch = FLOPS_PER_PARTICLE_STEP * args.particles * steps_per_launch
    achieved = flops_per_launch / (kernel_ms * 1e-3) / 1e12
    clk = clocks.summary()

    e2e = None
    if not args.no_e2e:
        # Through the public C ABI with host buffers: upload (H2D) + the fused
        # multi-step run + event records and final state back (D2H).
        # Through the sharded driver: rank 0 receives the whole job's event
        # records (global ids); each rank reads its own states back.
        fresh = pinned_system(workload(args.particles, args.seed, rank=rank))
        xo, vo = pinned_like(np.zeros((fresh.n, 3))), pinned_like(np.zeros((fresh.n, 3)))
        nbig = fresh.nbig
        ids = np.concatenate([np.arange(nbig), nbig + rank * args.particles + np.arange(args.particles)])
        run = ShardedRun(ranks, b)
        flag = fresh.ngflag   # derived from the input once, as mio_in does
        # one untimed call of the same run first (first-call set-up: events,
        # work counters, the library's scratch for this shape)
        run.run(fresh, ids, nbig + world * args.particles, 0.0, H, args.steps, RCEN, args.steps_per_launch, flag,
                out=(xo, vo))
        barrier()
        t0 = time.perf_counter()
        got, (x, v) = run.run(fresh, ids, nbig + world * args.particles, 0.0, H, args.steps, RCEN,
                              args.steps_per_launch, flag, out=(xo, vo))
        barrier()
        e2e_s = time.perf_counter() - t0
        e2e_s = ranks.max(e2e_s)
        d2h = fresh.n * 6 * 8 + run.local_events * (128 + 4)
        # the one-call run copies no masses of massless particles
        h2d = h2d_bytes(fresh) - (8 * (fresh.n - nbig) if not fresh.m[nbig:].any() else 0)
        e2e = {"value": world * args.particles * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "note": "wall clock around mercury_b200_mvs_run (upload, fused run, download in one C-ABI call; "
                       "the particles' copies overlap their steps) from page-locked host arrays, and the event "
                       "records read back; after one untimed call of the same run"}
    dropin = None
    if world == 1:
        # like for like with the reference's CUDA backend (its arm's
        # reference_cuda): one drop-in step and events call per step
        dropin = {"value": dropin_steps(b.lib, workload(args.particles, args.seed), DROPIN_STEPS), "unit": UNIT,
                  "steps": DROPIN_STEPS, "note": "mercury_cuda_step + mercury_cuda_events per step, wall clock"}

    # the metric's second half on the same GPU: the batched launch against the
    # plain per-system loop, and the adjoint against the forward sweep
    batched = adjoint = None
    if world == 1 and not args.no_extras:
        batched = batched_summary(args.seed, args.steps)
        adjoint, adj_grads, adj_sys, adj_pick = adjoint_summary(args.seed)

    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu_baseline:
        if adjoint is not None:
            # the oracle as the checker of the adjoint's gradients (64 particles)
            err, chaotic = adjoint_oracle_error(adj_sys, adj_pick, adj_grads)
            adjoint["grad_rel_err_vs_oracle"] = err
            adjoint["grad_checked"] = f"{len(adj_pick) - chaotic} of 64 random particles ({chaotic} chaotic left out)"
        sample_particles, sample_steps = 300_000, 457
        v_cpu, cores, dt = cpu_baseline(sample_particles, sample_steps, args.seed)
        cpu = {"value": v_cpu, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{sample_particles} particles of the same generator x {sample_steps} steps ({dt:.1f} s)"}
        # the oracle as the checker of this workload (after every timed region)
        parity = one_step_parity(b.lib, args.particles, args.seed)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(args, MVS_TEXT.format(n=args.particles), h_days=H, l2=MVS_L2),
            "run": {"steps_per_launch": steps_per_launch, "launches": len(launch_list),
                    "launch_steps": compact_steps([k for k, _ in launch_list]),
                    "threads_per_cta": args.threads or 128},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
                         "frac": achieved / peak_tflops,
                         "traffic": (sum(TRAFFIC_MB_PER_LAUNCH[steps_per_launch]) * args.particles
                                     if steps_per_launch in TRAFFIC_MB_PER_LAUNCH else None),
                         "traffic_unit": f"bytes per launch (ncu, {steps_per_launch} steps, scaled from 1M particles)",
                         "peak_source": "measured in this run: fma() chains on every SM (2 FLOP/FMA)",
                         "flops_per_particle_step": FLOPS_PER_PARTICLE_STEP,
                         "kernel_ms_per_launch": kernel_ms,
                         "fp64_pipe": ({"frac": FP64_PIPE_BY_K[steps_per_launch][0],
                                        "inst_per_particle_step": FP64_PIPE_BY_K[steps_per_launch][1],
                                        "issue_active": FP64_PIPE_BY_K[steps_per_launch][2],
                                        "source": f"ncu, one {steps_per_launch}-step launch of this workload"}
                                       if steps_per_launch in FP64_PIPE_BY_K else None)},
            "clocks": clk,
            "gpu_launches": tm["kernel_launches"],
            "events": int(len(events)),
            "energy_error": abs(e_end - e_start) / abs(e_start),
            "angular_momentum_error": abs(l_end - l_start) / abs(l_start),
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        if dropin is not None:
            line["dropin_per_step"] = dropin
        if parity is not None:
            line["parity"] = parity
        if batched is not None:
            line["batched"] = batched
        if adjoint is not None:
            line["adjoint"] = adjoint
        print(json.dumps(line), flush=True)
    b.free()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
