"""Discrete adjoint on the GPU: transposed line operators against the explicit operator matrices,
one-step vector-Jacobian products against finite differences, the full reverse sweep against
torch autograd through the explicit-matrix restatement (32^3), the torch.autograd.Function, and
the 128^3 decaying-turbulence gradient against central differences in 8 seeded directions."""
import math

import numpy as np
import pytest
import torch

import astr_gpu_b200 as ag
import oracle
from adjoint_reference import ExplicitSolver, periodic_matrix
from astr_gpu_b200.adjoint import Adjoint, apply_transpose, final_kinetic_energy, fortran_empty
from astr_gpu_b200.fields import solenoidal_q, solenoidal_velocity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = ag.Context(0)
    yield c
    c.close()


def to_dev(a):
    t = fortran_empty(a.shape)
    t.copy_(torch.from_numpy(np.asarray(a)))
    return t


@pytest.mark.parametrize("kind", ["deriv", "filter"])
@pytest.mark.parametrize("n", [16, 32, 57, 128, 300])
def test_transpose_matches_explicit_matrix(ctx, kind, n):
    if kind == "deriv":
        sch_o, sch_g = oracle.fd_scheme_initiate("643c", 3, n), ag.fd_scheme_initiate(ctx, "643c", 3, n)
    else:
        sch_o = oracle.compact_filter_initiate(3, n, 0.49, 1.11, 1.09)
        sch_g = ag.compact_filter_initiate(ctx, 3, n, 0.49, 1.11, 1.09)
    M = periodic_matrix(sch_o)
    rng = np.random.default_rng(n)
    for direction in range(3):
        shape = [5, 3, 4]
        shape[direction] = n + 1
        g = rng.standard_normal(shape + [2])
        out = apply_transpose(ctx, sch_g, to_dev(g), direction, 0.5).cpu().numpy()
        want = 0.5 * np.moveaxis(np.tensordot(M.T, g, axes=([1], [direction])), 0, direction)
        err = np.abs(out - want).max() / np.abs(want).max()
        assert err <= 1e-13, (kind, n, direction, err)


def perturbed_state(n, mach, seed):
    q = solenoidal_q(n, mach, seed)
    rng = np.random.default_rng(seed + 1)
    x = 2 * np.pi * np.arange(n + 1) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    drho = 0.05 * np.sin(X + 2 * Y) * np.cos(Z)
    q[..., 0] *= 1.0 + drho
    q[..., 1:4] *= (1.0 + drho)[..., None]
    q[..., 4] *= 1.0 + 0.02 * np.cos(2 * X - Z)
    return q


def test_step_vjp_matches_finite_differences(ctx):
    n = 32
    p = ag.FlowParams(mach=0.3, reynolds=500.0)
    s = ag.TGVSolver(ctx, n, params=p)
    q0 = perturbed_state(n, 0.3, 7)
    s.set_q(q0)
    dt = s.cfl_dt(0.5)
    adj = Adjoint(s, 1)
    rng = np.random.default_rng(11)
    lam = rng.standard_normal(q0.shape)
    vjp = adj.step_vjp(dt, lam)
    for trial in range(3):
        d = rng.standard_normal(q0.shape) * np.abs(q0).max(axis=(0, 1, 2))
        eps = 1e-6
        vals = []
        for sgn in (1.0, -1.0):
            s.set_q(q0 + sgn * eps * d)
            s.rk3(dt, 1)
            vals.append(np.sum(lam * s.get_q()))
        fd = (vals[0] - vals[1]) / (2 * eps)
        an = np.sum(vjp * d)
        assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)
    adj.close()
    s.close()


def test_adjoint_matches_autograd_of_explicit_matrices(ctx):
    """32^3, 6 steps with a checkpoint every 4: gradient of J against torch autograd through the
    explicit-matrix restatement (same discrete map, independent transposes)."""
    n, nsteps = 32, 6
    po = oracle.FlowParams(mach=0.3, reynolds=400.0)
    q0 = perturbed_state(n, 0.3, 3)
    s = ag.TGVSolver(ctx, n, params=ag.FlowParams(mach=0.3, reynolds=400.0))
    s.set_q(q0)
    dt = s.cfl_dt(0.5)
    adj = Adjoint(s, 4)
    J = adj.forward(dt, nsteps)
    g = adj.backward()
    es = ExplicitSolver(n, po)
    qt = torch.from_numpy(np.array(q0)).requires_grad_(True)
    q = qt
    for _ in range(nsteps):
        q = es.step(q, dt)
    Jt = es.kinetic_energy(q)
    Jt.backward()
    gt = qt.grad.numpy()
    assert abs(J - Jt.item()) <= 1e-12 * abs(Jt.item())
    for m in range(5):
        scale = np.abs(gt[..., m]).max()
        err = np.abs(g[..., m] - gt[..., m]).max()
        assert err <= 1e-9 * scale, (m, err, scale)
    adj.close()
    s.close()


def test_autograd_function(ctx):
    n = 24
    s = ag.TGVSolver(ctx, n, params=ag.FlowParams(mach=0.2, reynolds=800.0))
    q0 = perturbed_state(n, 0.2, 5)
    s.set_q(q0)
    dt = s.cfl_dt(0.5)
    qt = torch.tensor(q0, device="cuda", requires_grad=True)
    J = final_kinetic_energy(qt, s, dt, 5, 2)
    (2.0 * J).backward()
    s2 = ag.TGVSolver(ctx, n, params=ag.FlowParams(mach=0.2, reynolds=800.0))
    s2.set_q(q0)
    adj = Adjoint(s2, 2)
    J2 = adj.forward(dt, 5)
    g2 = adj.backward()
    assert abs(J.item() - J2) <= 1e-13 * abs(J2)
    np.testing.assert_allclose(qt.grad.cpu().numpy(), 2.0 * g2, rtol=0, atol=1e-13 * np.abs(g2).max())
    adj.close()
    s.close()
    s2.close()


def taylor_reynolds_re(n, seed, target=50.0):
    """Reynolds number giving Re_lambda = target for the solenoidal field (u' and the Taylor
    microscale lambda = u' / <(du_a/dx_a)^2>^(1/2), spectral derivatives, nu = 1/Re)."""
    u = solenoidal_velocity(n, seed)
    k = np.fft.fftfreq(n, 1.0 / n)
    d2 = []
    for a in range(3):
        ka = [k[:, None, None], k[None, :, None], k[None, None, :]][a]
        du = np.fft.ifftn(1j * ka * np.fft.fftn(u[a])).real
        d2.append(np.mean(du ** 2))
    up = np.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2) / 3.0)
    lam = up / np.sqrt(np.mean(d2))
    return target / (up * lam)


def test_decaying_turbulence_128_finite_differences(ctx):
    """128^3 periodic, solenoidal k^4 exp(-2(k/4)^2) field at M_t = 0.3, Re for Re_lambda = 50,
    200 steps with filter, checkpoint every 20: <dJ/dm0, d> against central differences with
    eps = 1e-6 relative (d has the RMS of the initial momentum) in 8 seeded momentum
    directions, to 1e-6."""
    n, nsteps, mach, seed = 128, 200, 0.3, 2024
    re = taylor_reynolds_re(n, seed)
    p = ag.FlowParams(mach=mach, reynolds=re)
    s = ag.TGVSolver(ctx, n, params=p)
    q0 = solenoidal_q(n, mach, seed)
    s.set_q(q0)
    dt = s.cfl_dt(0.5)
    adj = Adjoint(s, 20)
    J0 = adj.forward(dt, nsteps)
    g = adj.backward()
    assert np.isfinite(g).all()
    mrms = np.sqrt(np.mean(q0[..., 1:4] ** 2))
    for trial in range(8):
        # seeded random direction in momentum space: a random field with the same spectrum and
        # RMS as the initial momentum (white-noise directions cancel against the smooth gradient
        # and leave the difference quotient at the level of the forward rounding)
        d = np.zeros_like(q0)
        vel = solenoidal_velocity(n, 9000 + trial)
        for a in range(3):
            d[..., 1 + a] = np.pad(vel[a], [(0, 1)] * 3, mode="wrap")
        d *= mrms / np.sqrt(np.mean(d[..., 1:4] ** 2))
        eps = 1e-6
        vals = []
        for sgn in (1.0, -1.0):
            s.set_q(q0 + sgn * eps * d)
            a2 = Adjoint(s, 20)
            vals.append(a2.forward(dt, nsteps))
            a2.close()
        fd = (vals[0] - vals[1]) / (2 * eps)
        an = float(np.sum(g * d))
        assert abs(fd - an) <= 1e-6 * abs(an), (trial, fd, an)
    adj.close()
    s.close()
