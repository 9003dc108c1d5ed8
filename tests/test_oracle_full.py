"""The oracle's full-solver mode (TGV::rk3_full, a restatement of the full solver's
time_integration_rk on a periodic box) checked on the CPU where an exact relation holds. Its
parity against the reference itself is unpinned: no full-solver output exists here."""
import numpy as np

import oracle


def test_full_rhs_is_jacobian_times_miniapp_rhs_without_filter():
    """Filter off, a state with node N equal to node 0 and primitives consistent with q: qswap's
    averaging changes nothing, so the metric-form rhscal (convrsdcal6 / diffrsdcal6 with jacob and
    dxi) equals jacob times the miniapp's rhscal (divided by dx) to rounding."""
    n = 24
    p = oracle.FlowParams(filter_on=False)
    a = oracle.TGVOracle(n, params=p)
    a.init_tgv()
    mini = a.rhs()
    b = oracle.TGVOracle(n, params=p)
    b.init_tgv()
    full = b.rhs_full()
    h = 2 * np.pi / n
    jac, p0 = h ** 3, 1.0 / (1.4 * 0.1 ** 2)
    for m in range(5):
        scale = max(np.abs(jac * mini[..., m]).max(), jac * p0 / h)
        assert np.abs(full[..., m] - jac * mini[..., m]).max() <= 1e-13 * scale


def test_full_step_averages_duplicate_nodes_each_stage():
    """After a full-solver rhscal (filterq + qswap), nodes 0 and N hold the same conserved state
    on every axis; after the miniapp's steps they do not."""
    n = 24
    a = oracle.TGVOracle(n)
    a.init_tgv()
    a.set_dt(2e-3)
    a.steps_full(2)
    a.rhs_full()
    q = a.get_q()
    assert np.array_equal(q[0], q[-1]) and np.array_equal(q[:, 0], q[:, -1]) and np.array_equal(q[:, :, 0], q[:, :, -1])
    b = oracle.TGVOracle(n)
    b.init_tgv()
    b.set_dt(2e-3)
    b.steps(2)
    qb = b.get_q()
    assert not np.array_equal(qb[0], qb[-1])


def test_full_and_miniapp_steps_agree_to_the_averaging_level():
    """The two drivers advance the same equations: after 3 steps of the Taylor-Green box they
    differ by the duplicate-node averaging and the filter placement, a few 1e-8 of each field's
    scale (the momenta sharing theirs), not more."""
    n = 24
    for filt in (False, True):
        p = oracle.FlowParams(filter_on=filt)
        a = oracle.TGVOracle(n, params=p)
        a.init_tgv()
        a.set_dt(2e-3)
        a.steps(3)
        b = oracle.TGVOracle(n, params=p)
        b.init_tgv()
        b.set_dt(2e-3)
        b.steps_full(3)
        qa, qb = a.get_q(), b.get_q()
        mom = max(np.abs(qa[..., m]).max() for m in (1, 2, 3))
        scale = [np.abs(qa[..., 0]).max(), mom, mom, mom, np.abs(qa[..., 4]).max()]
        d = max(np.abs(qa[..., m] - qb[..., m]).max() / scale[m] for m in range(5))
        assert 1e-12 < d < 1e-6, (filt, d)


def test_walls_hold_the_wall_state_after_boucon():
    """Isothermal no-slip walls at the two ends along y: after a stage's filter and boucon the
    wall nodes carry zero momentum and the wall temperature's density p/T gamma M^2."""
    dims = (16, 20, 12)
    p = oracle.FlowParams(mach=0.2, reynolds=500.0, sutherland=110.3, beta_bound=0.98, ntype=(3, 4, 3), twall=1.3)
    o = oracle.TGVOracle(*dims, params=p)
    x = [2 * np.pi * np.arange(n + 1) / n for n in dims]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    q = np.zeros(tuple(n + 1 for n in dims) + (5,), order="F")
    q[..., 0] = 1.0 + 0.02 * np.cos(X)
    q[..., 1] = q[..., 0] * np.sin(Y / 2) ** 2
    q[..., 4] = 1.0 / (1.4 * 0.04) / 0.4 + 0.5 * q[..., 1] ** 2 / q[..., 0]
    o.set_q(q)
    o.rhs_full()
    qs = o.get_q()
    for j in (0, -1):
        assert np.all(qs[:, j, :, 1:4] == 0.0)
        pr = qs[:, j, :, 4] * 0.4
        np.testing.assert_allclose(qs[:, j, :, 0], pr / 1.3 * (1.4 * 0.04), rtol=1e-14)
