"""Build the in-tree CUDA library ``mercuda_b200/libmercury_cuda.so`` for sm_100a.

Every FP64 statement must round as the Fortran reference does, so the device
code is compiled with ``--fmad=false`` (no contraction into FMA) and IEEE
division and square root (nvcc's defaults), mirroring the reference's
``-ffp-contract=off`` CPU build and ``--fmad=false`` CUDA build.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libmercury_cuda.so"
SOURCES = ["mvs.cu", "abi.cu", "peak.cu", "noalloc.cu", "radau.cu", "bs.cu", "hybrid.cu", "batch.cu", "adjoint.cu", "energy.cu", "hybrid_adjoint.cu",
           "encode.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
         "-cudart", "static", "-Xptxas", "-warn-spills", "-Xlinker", "--no-undefined"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA library cannot be built")
    return path


def _stale() -> bool:
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list((HERE.parent / "include").glob("*.h"))
    return any(p.stat().st_mtime > built for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if any source is newer than it (or if forced): each
    translation unit to an object file in parallel, then one link."""
    if not force and not _stale():
        return LIB
    import concurrent.futures as cf
    import tempfile

    compile_flags = [f for f in FLAGS if f not in ("-shared", "-cudart", "static", "-Xlinker", "--no-undefined")]
    with tempfile.TemporaryDirectory(prefix="mb200_build_") as tmp:
        objs = [str(Path(tmp) / (Path(s).stem + ".o")) for s in SOURCES]
        cmds = [[nvcc(), *ARCH, *compile_flags, "-c", str(CSRC / s), "-o", o] for s, o in zip(SOURCES, objs)]
        if verbose:
            for cmd in cmds:
                print(" ".join(cmd), flush=True)
        workers = max(1, min(len(cmds), os.cpu_count() or 1))
        with cf.ThreadPoolExecutor(workers) as pool:
            results = list(pool.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
        for res in results:
            if res.returncode != 0:
                raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
            if verbose and res.stderr:
                print(res.stderr, file=sys.stderr)
        link = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-Xlinker", "--no-undefined", *objs, "-o",
                str(LIB) + ".tmp"]
        if verbose:
            print(" ".join(link), flush=True)
        res = subprocess.run(link, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
