"""Generate tests/golden/drift_ref.npz: inputs and outputs of the reference's
own drift_one (mercury_cuda_kepler.cuh compiled for the host by
oracle/Makefile's `ref` target into oracle/_ref/libkepler_ref.so).

Run from the repository root on a machine that has the reference tree:
    make -C oracle ref && python tests/golden/make_drift_golden.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

K2 = 2.959122082855911e-4


def cases(seed=2024, count=2000):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        r = rng.uniform(0.05, 40.0)
        x = rng.normal(size=3)
        x *= r / np.linalg.norm(x)
        # speeds from deep elliptic through parabolic to hyperbolic
        vfac = rng.choice([rng.uniform(0.2, 1.0), rng.uniform(1.0, 1.5), np.sqrt(2.0), rng.uniform(1.5, 3.0)])
        vc = np.sqrt(K2 / r) * vfac
        u = rng.normal(size=3)
        u -= u.dot(x) / r / r * x
        u *= vc / np.linalg.norm(u)
        u += rng.normal(size=3) * 0.05 * vc * rng.choice([0.0, 1.0])
        dt = rng.choice([8.0, -8.0, 0.5, 16.0, 365.25, -1000.0, 1e-3]) * rng.uniform(0.5, 1.0)
        mu = K2 * rng.choice([1.0, 1.0000003, 1.001])
        out.append((mu, np.concatenate([x, u]), dt))
    return out


def main():
    mus, inp, dts, outp, flags = [], [], [], [], []
    for mu, xv, dt in cases():
        res, flag = O.ref_drift_one(mu, xv, dt)
        mus.append(mu); inp.append(xv); dts.append(dt); outp.append(res); flags.append(flag)
    np.savez_compressed(ROOT / "tests/golden/drift_ref.npz", mu=np.array(mus), xv=np.array(inp), dt=np.array(dts),
                        out=np.array(outp), flag=np.array(flags, dtype=np.int32))
    print("wrote", len(mus), "reference drift cases")


if __name__ == "__main__":
    main()
