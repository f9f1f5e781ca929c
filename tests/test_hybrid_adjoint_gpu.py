"""Gradients through the HYBRID test-particle integration on the GPU
(mercury_b200_hybrid_adjoint_*, no reference counterpart) against the oracle's
HYBRID tangent map (forward-mode dual numbers through the oracle's mdt_hy and
mdt_hkce, pinned by central differences in test_hybrid_adjoint_oracle.py):
loss = sum |x_final|^2 + 100 sum |v_final|^2, gradients with respect to every
particle's initial position, velocity and Yarkovsky coefficient, with a
quarter of the particles placed near the planets so that encounter members go
through the BS2 subsystem.

A particle captured deep inside a planet's Hill sphere moves chaotically: its
exact gradient can reach 1e8 and no two trajectories that differ by rounding
share it to 1e-6. The comparison is therefore made on the particles whose
gradient is well conditioned, i.e. where the oracle's own central differences
confirm its tangent map to 1e-4; they must be most of the particles,
including encounter members."""
import numpy as np
import pytest
import torch

from mercuda_b200.adjoint import hybrid_timing, hybrid_trajectory
from test_hybrid_adjoint_oracle import hybrid_adjoint_case

pytestmark = pytest.mark.gpu

H, NSTEPS, TOL = 8.0, 40, 1e-12
VW = 100.0  # weight of the velocity term of the loss


def device_run(s, K, nsteps=NSTEPS, with_yar=True):
    dev = torch.device("cuda")
    nb = s.nbig
    x0 = torch.tensor(s.x[nb:], device=dev, requires_grad=True)
    v0 = torch.tensor(s.v[nb:], device=dev, requires_grad=True)
    yar = torch.tensor(s.ngf[nb:, 4], device=dev, requires_grad=True) if with_yar else None
    big = (s.m[:nb], s.x[:nb], s.v[:nb], s.rcrit[:nb])
    xf, vf = hybrid_trajectory(x0, v0, yar, big, s.rcrit[nb:], H, nsteps, TOL, K)
    loss = (xf ** 2).sum() + VW * (vf ** 2).sum()
    loss.backward()
    g = [x0.grad.cpu().numpy(), v0.grad.cpu().numpy(), yar.grad.cpu().numpy() if with_yar else None]
    return xf.detach().cpu().numpy(), vf.detach().cpu().numpy(), g


def well_conditioned(oracle, s, J, nsteps, gfin, with_yar=True):
    """Particles whose oracle gradient central differences (relative step 1e-6)
    reproduce to 1e-4 of each block."""
    nb, npart = s.nbig, s.n - s.nbig
    want = np.einsum("prk,pr->pk", J, gfin)

    def part_loss(c):
        c = c.copy()
        oracle.hy_run(c, 0.0, H, nsteps, TOL)
        return (c.x[nb:] ** 2).sum(1) + VW * (c.v[nb:] ** 2).sum(1)

    rx = np.linalg.norm(s.x[nb:], axis=1)
    rv = np.linalg.norm(s.v[nb:], axis=1)
    nk = 7 if with_yar else 6
    fd = np.zeros((npart, nk))
    for k in range(nk):
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
        fd[:, k] = (part_loss(p) - part_loss(m)) / (2 * step)
    err = np.zeros(npart)
    blocks = (slice(0, 3), slice(3, 6), slice(6, 7)) if with_yar else (slice(0, 3), slice(3, 6))
    for cols in blocks:
        scale = np.abs(want[:, cols]).max(axis=1)
        err = np.maximum(err, np.abs(fd[:, cols] - want[:, cols]).max(axis=1) / scale)
    return err < 1e-4


def near_planets(s, hills=6.0):
    """Particles that start within `hills` Hill radii of a planet."""
    nb = s.nbig
    hill = np.linalg.norm(s.x[1:nb], axis=1) * np.cbrt(s.m[1:nb] / (3 * s.m[0]))
    d = np.linalg.norm(s.x[nb:, None, :] - s.x[None, 1:nb, :], axis=2) / hill[None, :]
    return d.min(axis=1) < hills


def test_hybrid_gradients_match_oracle(cuda_lib, oracle):
    s = hybrid_adjoint_case(n=64, near=0.25)
    xf, vf, (gx, gv, gy) = device_run(s, 7)
    members = hybrid_timing()[2]
    assert members > 10                     # encounter members took the BS2 path
    ref = s.copy()
    J = oracle.hy_jacobian(ref, H, NSTEPS, TOL)
    nb = s.nbig
    assert np.max(np.abs(xf - ref.x[nb:])) < 1e-9 and np.max(np.abs(vf - ref.v[nb:])) < 1e-9
    gfin = np.concatenate([2 * ref.x[nb:], 2 * VW * ref.v[nb:]], axis=1)
    want = np.einsum("prk,pr->pk", J, gfin)
    got = np.concatenate([gx, gv, gy[:, None]], axis=1)
    well = well_conditioned(oracle, s, J, NSTEPS, gfin)
    near = near_planets(s)
    assert well.mean() > 0.9 and np.count_nonzero(well & near) >= 8, (well.mean(), np.count_nonzero(well & near))
    for cols in (slice(0, 3), slice(3, 6), slice(6, 7)):
        scale = np.abs(want[:, cols]).max(axis=1, keepdims=True)
        err = (np.abs(got[:, cols] - want[:, cols]) / scale).max(axis=1)
        assert np.max(err[well]) < 1e-6, (cols, np.argsort(-err)[:4], np.sort(err)[-4:])


def test_hybrid_checkpoint_interval_changes_nothing(cuda_lib):
    s = hybrid_adjoint_case(seed=9, n=32, near=0.25)
    runs = [device_run(s, K, nsteps=24) for K in (1, 5, 24)]
    for xf, vf, g in runs[1:]:
        assert np.array_equal(xf, runs[0][0]) and np.array_equal(vf, runs[0][1])
        for a, b in zip(g, runs[0][2]):
            assert np.array_equal(a, b)


def test_hybrid_forward_matches_drop_in_path(cuda_lib):
    """The forward sweep is the drop-in HYBRID path: same final states bit for bit."""
    from mercuda_b200.backend import Backend
    s = hybrid_adjoint_case(seed=11, n=48, near=0.25)
    xf, vf, _ = device_run(s, 10, nsteps=20)
    be = Backend("HYBRID", cuda_lib)
    be.configure()
    sys_ = s.copy()
    be.upload(sys_)
    state = {"dtflag": 0}
    t = 0.0
    for _ in range(20):
        be.hybrid_step(sys_, t, H, TOL, state)
        t += H
    x, v = be.download()
    be.free()
    assert np.array_equal(xf, x[s.nbig:]) and np.array_equal(vf, v[s.nbig:])


def test_hybrid_gradients_without_yar(cuda_lib, oracle):
    s = hybrid_adjoint_case(seed=13, n=32, near=0.25)
    s.ngf[:] = 0.0
    xf, vf, (gx, gv, _) = device_run(s, 6, nsteps=18, with_yar=False)
    ref = s.copy()
    J = oracle.hy_jacobian(ref, H, 18, TOL)
    nb = s.nbig
    gfin = np.concatenate([2 * ref.x[nb:], 2 * VW * ref.v[nb:]], axis=1)
    well = well_conditioned(oracle, s, J, 18, gfin, with_yar=False)
    assert well.mean() > 0.9
    want = np.einsum("prk,pr->pk", J, gfin)[:, :6]
    got = np.concatenate([gx, gv], axis=1)
    for cols in (slice(0, 3), slice(3, 6)):
        scale = np.abs(want[:, cols]).max(axis=1, keepdims=True)
        err = (np.abs(got[:, cols] - want[:, cols]) / scale).max(axis=1)
        assert np.max(err[well]) < 1e-6, (cols, np.argsort(-err)[:4], np.sort(err)[-4:])
