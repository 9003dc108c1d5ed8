"""Explicit-matrix reference of the periodic solver for the adjoint tests (test infrastructure).

Every 1-D operator of the forward step (compact derivative, compact filter; periodic ntype 3) is
assembled as a dense (N+1) x (N+1) matrix by applying the oracle's line routine to periodic unit
vectors (halo copies included), and the whole RK3 step (rhscal, rk3 and filterq of
miniapps/tgv_solver_3d/tgvsolver.F90:539-1082) is restated in torch FP64 on top of those
matrices. torch autograd through this restatement gives the gradient of the same discrete map
that the library's adjoint differentiates, with no hand-written transposes.
"""
from __future__ import annotations

import math

import numpy as np
import torch

import oracle

HM = 5


def _wrap(t, dim):
    return t + dim if t < 0 else (t - dim if t > dim else t)


def periodic_matrix(sch) -> np.ndarray:
    """Columns = the oracle's line operator applied to unit vectors of nodes 0..dim."""
    dim = sch.dim
    n = dim + 1
    M = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        ext = np.array([e[_wrap(t, dim)] for t in range(-HM, dim + HM + 1)])
        M[:, k] = sch.line(ext)
    return M


class ExplicitSolver:
    """The periodic box of ``oracle.TGVOracle`` (same parameters) in torch, cubic n^3."""

    RK = ((1.0, 0.0, 1.0), (0.75, 0.25, 0.25), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0))

    def __init__(self, n: int, params: oracle.FlowParams):
        self.n = n
        p = params
        self.p = p
        dx = 2.0 * math.pi / n
        self.dx = dx
        fd = oracle.fd_scheme_initiate("643c", 3, n)
        flt = oracle.compact_filter_initiate(3, n, p.alfa_filter, p.beta_halo, p.beta_bound)
        self.Dm = torch.from_numpy(periodic_matrix(fd))        # index-space derivative
        self.Fm = torch.from_numpy(periodic_matrix(flt))
        g = p.gamma
        self.const2 = g * p.mach ** 2
        self.const5 = (g - 1.0) * p.mach ** 2
        self.const6 = 1.0 / (g - 1.0)
        self.tc = p.sutherland / p.ref_tem
        self.tc1 = 1.0 + self.tc

    @staticmethod
    def along(M, f, axis):
        return torch.movedim(torch.tensordot(M, f, dims=([1], [axis])), 0, axis)

    def deriv(self, f, axis):
        return self.along(self.Dm, f, axis) / self.dx

    def rhs(self, q):
        rho = q[..., 0]
        m = [q[..., 1 + a] for a in range(3)]
        u = [m[a] / rho for a in range(3)]
        q4 = q[..., 4]
        p = (q4 - 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2])) / self.const6
        T = p / rho * self.const2
        G = [[self.deriv(u[a], b) for b in range(3)] for a in range(3)]
        GT = [self.deriv(T, b) for b in range(3)]
        qn = [rho, m[0], m[1], m[2], q4]
        R = [torch.zeros_like(rho) for _ in range(5)]
        for d in range(3):
            for n in range(5):
                if n == 4:
                    F = (q4 + p) * u[d]
                else:
                    F = qn[n] * u[d] + (p if n == d + 1 else 0.0)
                R[n] = R[n] + self.deriv(F, d)
        R = [-r for r in R]
        S = [[0.5 * (G[a][b] + G[b][a]) for b in range(3)] for a in range(3)]
        skk = (S[0][0] + S[1][1] + S[2][2]) / 3.0
        miu = T * torch.sqrt(T) * self.tc1 / (T + self.tc) / self.p.reynolds
        hcc = (miu / self.p.prandtl) / self.const5
        sig = [[2.0 * miu * (S[a][b] - (skk if a == b else 0.0)) for b in range(3)] for a in range(3)]
        Q = [hcc * GT[d] + sig[d][0] * u[0] + sig[d][1] * u[1] + sig[d][2] * u[2] for d in range(3)]
        for d in range(3):
            for j in range(3):
                R[j + 1] = R[j + 1] + self.deriv(sig[d][j], d)
            R[4] = R[4] + self.deriv(Q[d], d)
        return torch.stack(R, dim=-1)

    def filt(self, q):
        if not self.p.filter_on:
            return q
        for axis in range(3):
            q = self.along(self.Fm, q, axis)
        return q

    def step(self, q, dt):
        qsave = q
        for c1, c2, c3 in self.RK:
            q = self.filt(c1 * qsave + c2 * q + c3 * dt * self.rhs(q))
        return q

    def kinetic_energy(self, q):
        n = self.n
        s = q[1:, 1:, 1:]
        return 0.5 * ((s[..., 1] ** 2 + s[..., 2] ** 2 + s[..., 3] ** 2) / s[..., 0]).sum() / n ** 3
