"""The oracle against the reference's own golden data.

miniapps/tgv_solver_3d/state.ref_128 (tests/golden/state_ref_128.txt) is the Taylor-Green
history the reference miniapp wrote (tgvsolver.F90:938) at 128^3, dt=1e-3, Mach 0.1, Re 1600,
'643c', alpha_f = 0.49, filter after every stage. The oracle must reproduce it to 1e-12
relative; in practice it is bit-identical.
"""
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden", "state_ref_128.txt")
TOL = 1e-12


def _golden():
    return np.loadtxt(GOLD)


def _run(nsteps):
    t = oracle.TGVOracle(128)
    t.init_tgv()
    t.set_dt(1e-3)
    t.steps(nsteps)
    return t.history()


def _check(h, g):
    assert h.shape[0] == g.shape[0]
    np.testing.assert_array_equal(h[:, 0], g[:, 0])
    np.testing.assert_allclose(h[:, 1], g[:, 1], rtol=1e-15, atol=0)
    rel_ke = np.abs(h[:, 2] - g[:, 2]) / np.abs(g[:, 2])
    rel_en = np.abs(h[:, 3] - g[:, 3]) / np.abs(g[:, 3])
    assert rel_ke.max() <= TOL, rel_ke.max()
    assert rel_en.max() <= TOL, rel_en.max()


def test_golden_first_steps():
    g = _golden()[:4]
    _check(_run(4), g)


@pytest.mark.slow
def test_golden_full_history():
    g = _golden()
    _check(_run(100), g)
