"""Discrete adjoint of the periodic RK3 solver and its ``torch.autograd.Function``.

``final_kinetic_energy(q0, solver, dt, nsteps, checkpoint_every)`` returns
J = sum over nodes 1..N of |rho u|^2 / (2 rho), divided by im*jm*km, of the state reached from
``q0`` after ``nsteps`` steps of ``solver`` (a ``TGVSolver``: compact scheme, filter, SSP-RK3 as
in miniapps/tgv_solver_3d/tgvsolver.F90:994-1082), as a differentiable torch scalar.
``J.backward()`` runs the library's discrete adjoint (transposed compact solves and stencils,
flux vector-Jacobian products, reverse RK3 from checkpoints every ``checkpoint_every`` steps) and
puts dJ/dq0 in ``q0.grad``; the gradient with respect to the initial momentum is
``q0.grad[..., 1:4]``.

Tensors are CUDA float64 of shape (im+1, jm+1, km+1, 5) holding conserved variables on nodes
0..N (any strides; a column-major copy goes to the library).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import ASTR_DEVICE, ASTR_HOST

__all__ = ["Adjoint", "FinalKineticEnergy", "final_kinetic_energy", "apply_transpose", "fortran_empty"]


def _i64(v):
    return (ctypes.c_int64 * 3)(*[int(x) for x in v])


def fortran_empty(shape, device="cuda"):
    """A CUDA float64 tensor of ``shape`` with column-major (Fortran) strides."""
    import torch
    return torch.empty(tuple(reversed(shape)), dtype=torch.float64, device=device).permute(
        *reversed(range(len(shape))))


def _fortran(x):
    y = fortran_empty(tuple(x.shape), x.device)
    y.copy_(x)
    return y


class Adjoint:
    """``astr_adjoint`` on a ``TGVSolver``: ``forward(dt, nsteps)`` advances the solver (from its
    current state) keeping checkpoints and returns J; ``backward()`` returns dJ/dq0."""

    def __init__(self, solver, checkpoint_every: int = 20):
        self.solver = solver
        self.ctx = solver.ctx
        h = ctypes.c_void_p()
        self.ctx.check(self.ctx.L.astr_adjoint_create(solver._h, checkpoint_every, ctypes.byref(h)))
        self._h = h

    def forward(self, dt: float, nsteps: int) -> float:
        J = ctypes.c_double()
        self.ctx.check(self.ctx.L.astr_adjoint_forward(self._h, dt, nsteps, ctypes.byref(J)))
        return J.value

    def backward(self, out=None):
        """dJ/dq at step 0: a Fortran-ordered numpy array, or written into the CUDA tensor ``out``."""
        shape = self.solver.shape
        if out is None:
            g = np.zeros(shape + (5,), order="F")
            self.ctx.check(self.ctx.L.astr_adjoint_backward(self._h, ctypes.c_void_p(g.ctypes.data), _i64(shape),
                                                            _i64((0, 0, 0)), ASTR_HOST))
            return g
        assert out.stride(0) == 1
        self.ctx.check(self.ctx.L.astr_adjoint_backward(self._h, ctypes.c_void_p(out.data_ptr()), _i64(shape),
                                                        _i64((0, 0, 0)), ASTR_DEVICE))
        return out

    def step_vjp(self, dt: float, lam):
        """(d step/d q)^T lam at the solver's current state (numpy, Fortran order)."""
        shape = self.solver.shape
        lam = np.asfortranarray(lam, dtype=np.float64)
        out = np.zeros(shape + (5,), order="F")
        self.ctx.check(self.ctx.L.astr_step_vjp(self._h, dt, ctypes.c_void_p(lam.ctypes.data),
                                                ctypes.c_void_p(out.ctypes.data), _i64(shape), _i64((0, 0, 0)),
                                                ASTR_HOST))
        return out

    def close(self):
        # the adjoint reads its state's context on destruction: skip it once either is gone
        if getattr(self, "_h", None) and self.ctx.alive() and getattr(self.solver, "_h", None):
            self.ctx.L.astr_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _autograd_function():
    import torch

    class FinalKineticEnergy(torch.autograd.Function):
        """J(q0) through the library; backward = the discrete adjoint."""

        @staticmethod
        def forward(ctx, q0, solver, dt, nsteps, checkpoint_every):
            qf = _fortran(q0.detach())
            torch.cuda.current_stream(q0.device).synchronize()
            solver.set_q(qf)
            adj = Adjoint(solver, checkpoint_every)
            J = adj.forward(dt, nsteps)
            ctx.adj = adj
            ctx.shape = tuple(q0.shape)
            return torch.tensor(J, dtype=torch.float64, device=q0.device)

        @staticmethod
        def backward(ctx, gJ):
            g = fortran_empty(ctx.shape, gJ.device)
            torch.cuda.current_stream(gJ.device).synchronize()
            ctx.adj.backward(g)
            ctx.adj.close()
            return g * gJ, None, None, None, None

    return FinalKineticEnergy


_FKE = None


def FinalKineticEnergy():
    global _FKE
    if _FKE is None:
        _FKE = _autograd_function()
    return _FKE


def final_kinetic_energy(q0, solver, dt: float, nsteps: int, checkpoint_every: int = 20):
    """Differentiable J(q0) (see the module docstring)."""
    return FinalKineticEnergy().apply(q0, solver, dt, nsteps, checkpoint_every)


def apply_transpose(ctx, scheme, g, direction: int, scale: float = 1.0):
    """scale * L^T g along ``direction`` for a periodic ``Scheme`` L; ``g`` a CUDA float64 tensor
    of shape (n0, n1, n2[, nfields]) with column-major strides and n[direction] = dim + 1."""
    import torch
    nf = g.shape[3] if g.dim() == 4 else 1
    gf = _fortran(g)
    out = fortran_empty(tuple(g.shape), g.device)
    torch.cuda.current_stream(g.device).synchronize()
    ctx.check(ctx.L.astr_scheme_apply_transpose(ctx._h, scheme._h, direction, ctypes.c_void_p(gf.data_ptr()),
                                                _i64(g.shape[:3]), ctypes.c_void_p(out.data_ptr()), nf, scale))
    return out
