"""The oracle's tangent map, pinned: forward-mode dual numbers pushed through
the oracle's own mdt_mvs statements (oracle.mvs_jacobian) must agree with
central finite differences of the plain oracle run, per test particle, with
respect to its initial position, velocity and Yarkovsky coefficient. This is
the reference for the adjoint's gradients (the reference has no adjoint)."""
import numpy as np

from mercuda_b200.system import make_system


def adjoint_case(seed=21, n=16):
    s = make_system(seed=seed, n_particles=n, nplanets=8, near_fraction=0.0, h=8.0)
    rng = np.random.default_rng(seed + 1)
    npart = s.n - s.nbig
    s.ngf[s.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
    return s


def test_dual_jacobian_matches_finite_differences(oracle):
    s = adjoint_case()
    nsteps, h = 200, 8.0
    a = s.copy()
    J = oracle.mvs_jacobian(a, h, nsteps)
    b = s.copy()
    oracle.mvs_run(b, 0.0, h, nsteps, 0.005)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v)

    def final(sysx):
        c = sysx.copy()
        oracle.mvs_run(c, 0.0, h, nsteps, 0.005)
        return np.concatenate([c.x[c.nbig:], c.v[c.nbig:]], axis=1)

    rx = np.linalg.norm(s.x[s.nbig:], axis=1)
    rv = np.linalg.norm(s.v[s.nbig:], axis=1)
    for k in range(7):
        p, m = s.copy(), s.copy()
        if k < 3:
            step = 1e-8 * rx
            p.x[s.nbig:, k] += step
            m.x[s.nbig:, k] -= step
        elif k < 6:
            step = 1e-8 * rv
            p.v[s.nbig:, k - 3] += step
            m.v[s.nbig:, k - 3] -= step
        else:
            step = np.full(s.n - s.nbig, 1e-13)
            p.ngf[s.nbig:, 4] += step
            m.ngf[s.nbig:, 4] -= step
        fd = (final(p) - final(m)) / (2 * step[:, None])
        # central differences deliver ~1e-6 of each particle's Jacobian block
        # (truncation against rounding at this step size)
        block = slice(0, 3) if k < 3 else slice(3, 6) if k < 6 else slice(6, 7)
        scale = np.abs(J[:, :, block]).max(axis=(1, 2))[:, None]
        assert np.max(np.abs(fd - J[:, :, k]) / scale) < 1e-5, k
