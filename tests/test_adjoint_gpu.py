"""Gradients through the MVS test-particle integration on the GPU
(mercury_b200_adjoint_*, no reference counterpart) against the oracle's
tangent map (forward-mode dual numbers through the oracle's mdt_mvs, itself
pinned by finite differences in test_adjoint_oracle.py): loss = sum |x_final|^2,
gradients with respect to every particle's initial position, velocity and
Yarkovsky coefficient, 1,000 steps of 8 days with a checkpoint every 50."""
import numpy as np
import pytest
import torch

from mercuda_b200.adjoint import mvs_trajectory
from mercuda_b200.system import make_system

pytestmark = pytest.mark.gpu

H, NSTEPS = 8.0, 1000


def case(seed=21, n=64, with_yar=True):
    s = make_system(seed=seed, n_particles=n, nplanets=8, near_fraction=0.0, h=H)
    if with_yar:
        rng = np.random.default_rng(seed + 1)
        npart = s.n - s.nbig
        s.ngf[s.nbig:, 4] = np.exp(rng.uniform(np.log(1e-15), np.log(1e-13), npart)) * rng.choice([-1, 1], npart)
    return s


def device_run(s, K, with_yar=True, nsteps=NSTEPS):
    dev = torch.device("cuda")
    nb = s.nbig
    x0 = torch.tensor(s.x[nb:], device=dev, requires_grad=True)
    v0 = torch.tensor(s.v[nb:], device=dev, requires_grad=True)
    yar = torch.tensor(s.ngf[nb:, 4], device=dev, requires_grad=True) if with_yar else None
    xf, vf = mvs_trajectory(x0, v0, yar, (s.m[:nb], s.x[:nb], s.v[:nb]), H, nsteps, K)
    loss = (xf ** 2).sum()
    loss.backward()
    g = [x0.grad.cpu().numpy(), v0.grad.cpu().numpy()]
    g.append(yar.grad.cpu().numpy() if with_yar else None)
    return xf.detach().cpu().numpy(), vf.detach().cpu().numpy(), g


def oracle_grads(oracle, s, nsteps=NSTEPS):
    ref = s.copy()
    J = oracle.mvs_jacobian(ref, H, nsteps)
    xf = ref.x[ref.nbig:]
    gfin = np.concatenate([2 * xf, np.zeros_like(xf)], axis=1)   # dL/d(x_final, v_final)
    grad = np.einsum("prk,pr->pk", J, gfin)                       # J^T g per particle
    return ref, grad


@pytest.mark.parametrize("with_yar", [True, False])
def test_gradients_match_oracle(cuda_lib, oracle, with_yar):
    s = case(with_yar=with_yar)
    xf, vf, (gx, gv, gy) = device_run(s, 50, with_yar)
    ref, grad = oracle_grads(oracle, s)
    nb = s.nbig
    assert np.max(np.abs(xf - ref.x[nb:])) < 1e-9 and np.max(np.abs(vf - ref.v[nb:])) < 1e-11
    got = np.concatenate([gx, gv] + ([gy[:, None]] if with_yar else []), axis=1)
    want = grad[:, :7 if with_yar else 6]
    # relative to each particle's gradient block (position, velocity, yar)
    for cols in (slice(0, 3), slice(3, 6)) + ((slice(6, 7),) if with_yar else ()):
        scale = np.abs(want[:, cols]).max(axis=1, keepdims=True)
        err = np.max(np.abs(got[:, cols] - want[:, cols]) / scale)
        assert err < 1e-6, (cols, err)


def test_checkpoint_interval_changes_nothing(cuda_lib):
    s = case(n=32)
    runs = [device_run(s, K, nsteps=300) for K in (1, 7, 50, 300)]
    for xf, vf, g in runs[1:]:
        assert np.array_equal(xf, runs[0][0]) and np.array_equal(vf, runs[0][1])
        for a, b in zip(g, runs[0][2]):
            assert np.array_equal(a, b)


def test_forward_matches_mvs_path(cuda_lib):
    """The forward sweep steps particles exactly as the drop-in MVS path does."""
    from mercuda_b200.backend import Backend
    s = case(n=40)
    xf, vf, _ = device_run(s, 50, nsteps=100)
    be = Backend("MVS", cuda_lib)
    be.configure()
    be.upload(s.copy())
    be.mvs_advance(0.0, H, 100, 0.005)
    x, v = be.download()
    be.free()
    assert np.array_equal(xf, x[s.nbig:]) and np.array_equal(vf, v[s.nbig:])
