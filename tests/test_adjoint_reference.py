"""The explicit-matrix restatement used as the adjoint's reference reproduces the oracle's RK3
steps, and its periodic operator matrices are the oracle's line operators."""
import numpy as np
import torch

import oracle
from adjoint_reference import ExplicitSolver, periodic_matrix
from astr_gpu_b200.fields import solenoidal_q


def test_matrices_match_line_operators():
    n = 24
    rng = np.random.default_rng(3)
    for sch in (oracle.fd_scheme_initiate("643c", 3, n), oracle.compact_filter_initiate(3, n, 0.49, 1.11, 1.09)):
        M = periodic_matrix(sch)
        f = rng.standard_normal(n + 1)
        ext = np.array([f[t + n if t < 0 else (t - n if t > n else t)] for t in range(-5, n + 6)])
        np.testing.assert_allclose(M @ f, sch.line(ext), rtol=0, atol=1e-14 * np.abs(f).max() * 10)


def test_explicit_steps_match_oracle():
    n = 20
    p = oracle.FlowParams(mach=0.3, reynolds=500.0)
    q0 = solenoidal_q(n, 0.3, 5)
    o = oracle.TGVOracle(n, params=p)
    o.set_q(q0)
    dt = o.cfl_dt(0.5)
    o.set_dt(dt)
    es = ExplicitSolver(n, p)
    q = torch.from_numpy(np.array(q0))
    for _ in range(2):
        q = es.step(q, dt)
    o.steps(2)
    qo = o.get_q()
    assert np.abs(q.numpy() - qo).max() <= 1e-12 * np.abs(qo).max()
