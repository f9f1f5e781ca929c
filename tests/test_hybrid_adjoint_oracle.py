"""The oracle's HYBRID tangent map, pinned: forward-mode dual numbers pushed
through the oracle's own mdt_hy statements (oracle.hy_jacobian: changeover
kicks, solar drifts, the Kepler drift, and mdt_hkce's BS2 substeps for the
steps in which a particle is an encounter member) must reproduce the plain
oracle run's states bit for bit and agree with central finite differences of
that run, per test particle, with respect to its initial position, velocity
and Yarkovsky coefficient. This is the reference for the HYBRID adjoint's
gradients (the reference has no adjoint)."""
import numpy as np

from mercuda_b200.system import make_system


def hybrid_adjoint_case(seed=5, n=24, near=0.3):
    s = make_system(seed=seed, n_particles=n, nplanets=8, near_fraction=near, h=8.0)
    rng = np.random.default_rng(seed + 1)
    npart = s.n - s.nbig
    s.ngf[s.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
    return s


def test_hybrid_dual_jacobian_matches_finite_differences(oracle):
    s = hybrid_adjoint_case()
    nsteps, h = 60, 8.0
    a = s.copy()
    J = oracle.hy_jacobian(a, h, nsteps)
    b = s.copy()
    _, _, _, pairs = oracle.hy_run(b, 0.0, h, nsteps)
    assert pairs > 20                      # encounter members went through BS2
    assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v)

    def final(sysx):
        c = sysx.copy()
        oracle.hy_run(c, 0.0, h, nsteps)
        return np.concatenate([c.x[c.nbig:], c.v[c.nbig:]], axis=1)

    nb, npart = s.nbig, s.n - s.nbig
    rx = np.linalg.norm(s.x[nb:], axis=1)
    rv = np.linalg.norm(s.v[nb:], axis=1)
    errs = []
    for k in range(7):
        p, m = s.copy(), s.copy()
        if k < 3:
            step = 1e-6 * rx
            p.x[nb:, k] += step
            m.x[nb:, k] -= step
        elif k < 6:
            step = 1e-6 * rv
            p.v[nb:, k - 3] += step
            m.v[nb:, k - 3] -= step
        else:
            step = np.full(npart, 1e-11)
            p.ngf[nb:, 4] += step
            m.ngf[nb:, 4] -= step
        fd = (final(p) - final(m)) / (2 * step[:, None])
        block = slice(0, 3) if k < 3 else slice(3, 6) if k < 6 else slice(6, 7)
        scale = np.abs(J[:, :, block]).max(axis=(1, 2))[:, None]
        errs.append(np.max(np.abs(fd - J[:, :, k]) / scale, axis=1))
    err = np.max(errs, axis=0)
    # The difference quotient's own error is rounding / step and, for a few
    # encounter members, the BS2 step control choosing another level under the
    # perturbation; the tangent map is exact for the chosen substeps.
    assert np.median(err) < 1e-6, err
    assert np.mean(err < 2e-6) > 0.8, err
    assert np.max(err) < 1e-4, err
