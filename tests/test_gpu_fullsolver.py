"""The full solver's time integration (astr_full_*, src/mainloop.F90:298-476) against the oracle's
full-solver mode on the same inputs: filterq before rhscal at every stage, qswap's averaging of
nodes 0 and N with primitives recomputed on the boundary planes and halos only, rhscal in its
metric form, the update of q*jacob, Sutherland 110.3.

Tolerances: one stage's RHS within 1e-12 of max(|R_m|_inf, jacob p0/dx) per field (the rounding
floor of differentiating the O(p0) pressure, p0 = 1/(gamma M^2)); the state after one stage's
filter and averaging within 1e-13 of each field's largest value; conserved variables after the
steps within 1e-10 of each field's largest value; diagnostics rows within 1e-12 relative.

The upwind convection (conschm 543, convrsdcmp, src/solver.F90:1272-1938: Steger-Warming split,
compact interface flux, MP limiter, optionally in characteristic variables with the Ducros
sensor) is checked the same way; its RHS tolerance carries a factor 1/M for the split fluxes'
acoustic parts (see test_full_upwind_rhs_matches_oracle)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import astr_gpu_b200 as ag
    return ag.Context(0)


def _state(dims, seed, mach):
    rng = np.random.default_rng(seed)
    x = [2 * np.pi * np.arange(n + 1) / n for n in dims]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    rho = 1.0 + 0.05 * np.sin(X + Y) * np.cos(Z)
    u = np.sin(X) * np.cos(Y) * np.cos(Z) + 0.1 * np.cos(2 * Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z) + 0.1 * rng.standard_normal() * np.sin(X)
    w = 0.2 * np.sin(Y + Z)
    p = 1.0 / (1.4 * mach ** 2) + 0.1 * np.cos(2 * X)
    q = np.zeros(tuple(n + 1 for n in dims) + (5,), order="F")
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 3] = rho * w
    q[..., 4] = p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)
    # make node N differ from node 0 slightly, so that qswap's averaging matters
    q[-1, :, :, :] *= 1.0 + 1e-6
    q[:, -1, :, :] *= 1.0 - 1e-6
    return q


def _rel_fields(a, b):
    return max(float(np.abs(a[..., m] - b[..., m]).max() / np.abs(b[..., m]).max()) for m in range(5))


def _pair(dims, mach, reynolds, filter_on=True):
    import astr_gpu_b200 as ag
    op = oracle.FlowParams(mach=mach, reynolds=reynolds, sutherland=110.3, beta_bound=0.98, filter_on=filter_on)
    gp = ag.FlowParams(mach=mach, reynolds=reynolds, sutherland=110.3, beta_bound=0.98, filter_on=filter_on)
    return op, gp


@pytest.mark.parametrize("dims", [(48, 48, 48), (40, 56, 36)])
def test_full_rhs_matches_oracle(ctx, dims):
    import astr_gpu_b200 as ag
    mach = 0.2
    q = _state(dims, 7, mach)
    op, gp = _pair(dims, mach, 800.0)
    o = oracle.TGVOracle(*dims, params=op)
    o.set_q(q)
    ref = o.rhs_full()
    s = ag.FullSolver(ctx, *dims, params=gp)
    s.set_q(q)
    got = s.rhs()
    h = [2 * np.pi / n for n in dims]
    jac, p0 = h[0] * h[1] * h[2], 1.0 / (1.4 * mach ** 2)
    for m in range(5):
        scale = max(np.abs(ref[..., m]).max(), jac * p0 / min(h))
        assert np.abs(got[..., m] - ref[..., m]).max() <= 1e-12 * scale, m
    # the state after the stage's filter and qswap
    assert _rel_fields(s.get_q(), o.get_q()) <= 1e-13
    s.close()


@pytest.mark.parametrize("filter_on", [True, False])
def test_full_tgv64_steps_match_oracle(ctx, filter_on):
    """Taylor-Green 64^3 at Mach 0.1, Re 1600: 20 full-solver steps, dt from CFL 0.5."""
    import astr_gpu_b200 as ag
    n, steps = 64, 20
    op, gp = _pair((n,) * 3, 0.1, 1600.0, filter_on)
    o = oracle.TGVOracle(n, params=op)
    o.init_tgv()
    dt = o.cfl_dt(0.5)
    q0 = o.get_q()
    o.set_dt(dt)
    o.steps_full(steps)
    s = ag.FullSolver(ctx, n, params=gp)
    s.set_q(q0)
    s.step(dt, steps)
    assert _rel_fields(s.get_q(), o.get_q()) <= 1e-10
    h, hc = s.history(), o.history(compensated=True)
    assert h.shape == hc.shape
    np.testing.assert_array_equal(h[:, 0], hc[:, 0])
    for c in (2, 3, 4):
        assert np.abs(h[:, c] - hc[:, c]).max() / np.abs(hc[:, c]).max() <= 1e-12
    s.close()


def test_full_noncubic_steps_match_oracle(ctx):
    import astr_gpu_b200 as ag
    dims = (40, 56, 36)
    mach = 0.2
    q = _state(dims, 11, mach)
    op, gp = _pair(dims, mach, 800.0)
    o = oracle.TGVOracle(*dims, params=op)
    o.set_q(q)
    dt = o.cfl_dt(0.5)
    o.set_dt(dt)
    o.steps_full(10)
    s = ag.FullSolver(ctx, *dims, params=gp)
    s.set_q(q)
    s.step(dt, 10)
    assert _rel_fields(s.get_q(), o.get_q()) <= 1e-10
    s.close()


def test_full_and_miniapp_modes_differ_as_expected(ctx):
    """The two drivers are different time integrations of the same equations (filter placement,
    duplicate-node averaging): after 10 steps of the same Taylor-Green box they differ far above
    rounding and far below the solution's scale, while each matches its own oracle mode."""
    import astr_gpu_b200 as ag
    n = 32
    op, gp = _pair((n,) * 3, 0.1, 1600.0)
    s1 = ag.FullSolver(ctx, n, params=gp)
    s2 = ag.TGVSolver(ctx, n, params=gp)
    s2.init_tgv()
    s1.set_q(s2.get_q())
    s1.step(2e-3, 10)
    s2.rk3(2e-3, 10)
    a, b = s1.get_q(), s2.get_q()
    mom = max(np.abs(b[..., m]).max() for m in (1, 2, 3))
    scale = [np.abs(b[..., 0]).max(), mom, mom, mom, np.abs(b[..., 4]).max()]
    d = max(np.abs(a[..., m] - b[..., m]).max() / scale[m] for m in range(5))
    assert 1e-12 < d < 1e-5


def _channel_state(dims, mach, seed):
    """A wall-bounded state: x and z periodic, walls at y = 0 and y = L with zero velocity."""
    rng = np.random.default_rng(seed)
    x = [2 * np.pi * np.arange(n + 1) / n for n in dims]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    rho = 1.0 + 0.02 * np.cos(X) * np.sin(Y / 2)
    u = np.sin(Y / 2) ** 2 * (1.0 + 0.1 * np.cos(X) * np.sin(Z))
    v = 0.05 * np.sin(Y) * np.sin(X) * (1.0 + 0.1 * rng.standard_normal())
    w = 0.05 * np.sin(Y) * np.cos(Z)
    p = 1.0 / (1.4 * mach ** 2) + 0.05 * np.cos(X)
    q = np.zeros(tuple(n + 1 for n in dims) + (5,), order="F")
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 3] = rho * w
    q[..., 4] = p / 0.4 + 0.5 * rho * (u * u + v * v + w * w)
    return q


@pytest.mark.parametrize("ntype", [(3, 4, 3), (4, 3, 3)])
def test_full_walls_match_oracle(ctx, ntype):
    """Non-periodic closures end to end with isothermal no-slip walls (bctype 41, boucon's noslip,
    src/bc.F90:6281-6595) at the physical ends of one direction: the compact boundary closures of the
    derivative and the filter (beta_bound 0.98, the filter's boundary reset), the wall state set
    after the filter at every stage, no exchange along the walled direction. One stage's RHS and 10
    steps against the oracle's full-solver mode with the same boundaries."""
    import astr_gpu_b200 as ag
    dims = (40, 48, 36) if ntype[1] == 4 else (48, 40, 36)
    mach = 0.2
    q = _channel_state(dims, mach, 5)
    if ntype[0] == 4:   # walls at x = 0 and x = L: rotate the velocity pattern
        q = np.asfortranarray(np.transpose(_channel_state((dims[1], dims[0], dims[2]), mach, 5), (1, 0, 2, 3))[..., [0, 2, 1, 3, 4]])
    kw = dict(mach=mach, reynolds=500.0, sutherland=110.3, beta_bound=0.98, ntype=ntype, twall=1.0)
    o = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o.set_q(q)
    ref = o.rhs_full()
    s = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s.set_q(q)
    got = s.rhs()
    h = [2 * np.pi / n for n in dims]
    jac, p0 = h[0] * h[1] * h[2], 1.0 / (1.4 * mach ** 2)
    for m in range(5):
        scale = max(np.abs(ref[..., m]).max(), jac * p0 / min(h))
        assert np.abs(got[..., m] - ref[..., m]).max() <= 1e-12 * scale, m
    o2 = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o2.set_q(q)
    o2.set_dt(1e-3)
    o2.steps_full(10)
    s2 = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s2.set_q(q)
    s2.step(1e-3, 10)
    qo, qg = o2.get_q(), s2.get_q()
    mom = max(np.abs(qo[..., m]).max() for m in (1, 2, 3))
    scale = [np.abs(qo[..., 0]).max(), mom, mom, mom, np.abs(qo[..., 4]).max()]
    assert max(np.abs(qg[..., m] - qo[..., m]).max() / scale[m] for m in range(5)) <= 1e-10
    s.close()
    s2.close()


def test_full_box_with_walls_on_every_side_matches_oracle(ctx):
    """ntype 4 in all three directions (a closed box, as the lid-driven cavity's layout without the
    lid): every face gets the isothermal no-slip state in boucon's order, so the edges and corners
    are set by the last face that owns them. One stage's RHS and 5 steps against the oracle."""
    import astr_gpu_b200 as ag
    dims = (40, 48, 36)
    mach = 0.2
    q = _channel_state(dims, mach, 5)
    kw = dict(mach=mach, reynolds=500.0, sutherland=110.3, beta_bound=0.98, ntype=(4, 4, 4), twall=1.0)
    o = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o.set_q(q)
    ref = o.rhs_full()
    s = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s.set_q(q)
    got = s.rhs()
    h = [2 * np.pi / n for n in dims]
    jac, p0 = h[0] * h[1] * h[2], 1.0 / (1.4 * mach ** 2)
    for m in range(5):
        scale = max(np.abs(ref[..., m]).max(), jac * p0 / min(h))
        assert np.abs(got[..., m] - ref[..., m]).max() <= 1e-12 * scale, m
    s.close()
    o2 = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o2.set_q(q)
    o2.set_dt(1e-3)
    o2.steps_full(5)
    s2 = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s2.set_q(q)
    s2.step(1e-3, 5)
    qo, qg = o2.get_q(), s2.get_q()
    mom = max(np.abs(qo[..., m]).max() for m in (1, 2, 3))
    scale = [np.abs(qo[..., 0]).max(), mom, mom, mom, np.abs(qo[..., 4]).max()]
    assert max(np.abs(qg[..., m] - qo[..., m]).max() / scale[m] for m in range(5)) <= 1e-10
    s2.close()


def test_miniapp_step_rejects_walls(ctx):
    import astr_gpu_b200 as ag
    with pytest.raises(ag.AstrError) as e:
        ag.TGVSolver(ctx, 32, params=ag.FlowParams(ntype=(3, 4, 3)))
    assert e.value.code == -4


@pytest.mark.parametrize("bfac", [0.0, 0.5, 1.0])
def test_full_upwind_rhs_matches_oracle(ctx, bfac):
    """conschm 543: convrsdcmp without the characteristic decomposition (Steger-Warming splitting,
    the compact interface flux of each part, the MP limiter at every interface, the flux
    difference; src/solver.F90:1272-1938) in one full-solver stage, against the oracle.

    Tolerance: 1e-12 of the field's scale times 1/M. The split fluxes f+ and f- carry the acoustic
    parts, larger than the net flux by about c/|u| = 1/M, and cancel in Fh(i) - Fh(i-1); their
    rounding, not the net flux's, sets the floor (measured 1.1e-12 relative at M = 0.2, b = 0)."""
    import astr_gpu_b200 as ag
    dims = (40, 48, 36)
    mach = 0.2
    q = _state(dims, 13, mach)
    kw = dict(mach=mach, reynolds=800.0, sutherland=110.3, beta_bound=0.98, conschm=543, bfacmpld=bfac)
    o = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o.set_q(q)
    ref = o.rhs_full()
    s = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s.set_q(q)
    got = s.rhs()
    h = [2 * np.pi / n for n in dims]
    jac, p0 = h[0] * h[1] * h[2], 1.0 / (1.4 * mach ** 2)
    for m in range(5):
        scale = max(np.abs(ref[..., m]).max(), jac * p0 / min(h))
        assert np.abs(got[..., m] - ref[..., m]).max() <= 1e-12 / mach * scale, m
    s.close()


@pytest.mark.parametrize("ntype", [(3, 3, 3), (3, 4, 3)])
def test_full_upwind_steps_match_oracle(ctx, ntype):
    """10 full-solver steps with the upwind compact flux (b = 0.3), periodic and with no-slip walls
    at the ends of y, against the oracle."""
    import astr_gpu_b200 as ag
    dims = (40, 48, 36)
    mach = 0.2
    q = _state(dims, 17, mach) if ntype == (3, 3, 3) else _channel_state(dims, mach, 9)
    kw = dict(mach=mach, reynolds=800.0, sutherland=110.3, beta_bound=0.98, conschm=543, bfacmpld=0.3,
              ntype=ntype, twall=1.0)
    o = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o.set_q(q)
    o.set_dt(1e-3)
    o.steps_full(10)
    s = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s.set_q(q)
    s.step(1e-3, 10)
    qo, qg = o.get_q(), s.get_q()
    mom = max(np.abs(qo[..., m]).max() for m in (1, 2, 3))
    scale = [np.abs(qo[..., 0]).max(), mom, mom, mom, np.abs(qo[..., 4]).max()]
    assert max(np.abs(qg[..., m] - qo[..., m]).max() / scale[m] for m in range(5)) <= 1e-10
    s.close()


@pytest.mark.parametrize("shkcrt", [1e-5, 0.01])
def test_full_upwind_characteristic_rhs_matches_oracle(ctx, shkcrt):
    """lchardecomp: the Ducros sensor (ducrossensor, commcal.F90:196-353) flags the nodes, and
    convrsdcmp limits in characteristic variables (chardecomp's Roe-averaged eigenvectors,
    solver.F90:1959-2163) with each interface's flag. shkcrt 1e-5 flags about 60 % of the nodes
    of this state, 0.01 none (the limiter then never acts)."""
    import astr_gpu_b200 as ag
    dims = (40, 48, 36)
    mach = 0.2
    q = _state(dims, 19, mach)
    kw = dict(mach=mach, reynolds=800.0, sutherland=110.3, beta_bound=0.98, conschm=543, bfacmpld=0.3,
              lchardecomp=True, shkcrt=shkcrt)
    o = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o.set_q(q)
    ref = o.rhs_full()
    flags = o.shock_flags()
    assert (0.3 < flags.mean() < 0.9) if shkcrt < 1e-3 else not flags.any()
    s = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s.set_q(q)
    got = s.rhs()
    h = [2 * np.pi / n for n in dims]
    jac, p0 = h[0] * h[1] * h[2], 1.0 / (1.4 * mach ** 2)
    for m in range(5):
        scale = max(np.abs(ref[..., m]).max(), jac * p0 / min(h))
        assert np.abs(got[..., m] - ref[..., m]).max() <= 1e-12 / mach * scale, m   # as the upwind test above
    s.close()


def test_full_upwind_characteristic_steps_match_oracle(ctx):
    import astr_gpu_b200 as ag
    dims = (40, 48, 36)
    mach = 0.2
    q = _state(dims, 23, mach)
    kw = dict(mach=mach, reynolds=800.0, sutherland=110.3, beta_bound=0.98, conschm=543, bfacmpld=0.1,
              lchardecomp=True, shkcrt=1e-5)
    o = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o.set_q(q)
    o.set_dt(1e-3)
    o.steps_full(10)
    s = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s.set_q(q)
    s.step(1e-3, 10)
    assert _rel_fields(s.get_q(), o.get_q()) <= 1e-10
    s.close()


def test_full_solver_rejects_bad_parameters(ctx):
    import astr_gpu_b200 as ag
    for kw in (dict(conschm=543, bfacmpld=float("nan")), dict(conschm=543, lchardecomp=True, shkcrt=float("inf")),
               dict(mach=0.0), dict(gamma=1.0), dict(conschm=642)):
        with pytest.raises(ag.AstrError) as e:
            ag.FullSolver(ctx, 32, params=ag.FlowParams(**kw))
        assert e.value.code == -1, kw


def test_characteristic_mode_rejects_walls(ctx):
    import astr_gpu_b200 as ag
    with pytest.raises(ag.AstrError) as e:
        ag.FullSolver(ctx, 32, params=ag.FlowParams(conschm=543, lchardecomp=True, ntype=(3, 4, 3)))
    assert e.value.code == -4


def test_upwind_and_central_differ_as_expected(ctx):
    """The two convection schemes are different discretisations: on a smooth Taylor-Green box the
    upwind flux with b = 1 (a symmetric 6th-order interface scheme) keeps the momentum RHS within
    1e-3 of the central compact one and the energy RHS within 5e-2 (the MP limiter clips the
    split energy fluxes where the split's eigenvalue uu crosses zero), all far above rounding."""
    import astr_gpu_b200 as ag
    n = 32
    out = {}
    for cs in (643, 543):
        p = ag.FlowParams(mach=0.1, reynolds=1600.0, sutherland=110.3, beta_bound=0.98, filter_on=False, conschm=cs,
                          bfacmpld=1.0)
        t = ag.TGVSolver(ctx, n, params=ag.FlowParams())
        t.init_tgv()
        s = ag.FullSolver(ctx, n, params=p)
        s.set_q(t.get_q())
        out[cs] = s.rhs()
        s.close()
    for m, bound in ((1, 1e-3), (2, 1e-3), (4, 5e-2)):
        d = np.abs(out[543][..., m] - out[643][..., m]).max() / np.abs(out[643][..., m]).max()
        assert 1e-12 < d < bound, (m, d)


def test_miniapp_step_rejects_upwind(ctx):
    import astr_gpu_b200 as ag
    with pytest.raises(ag.AstrError) as e:
        ag.TGVSolver(ctx, 32, params=ag.FlowParams(conschm=543))
    assert e.value.code == -4
    with pytest.raises(ag.AstrError):
        ag.FullSolver(ctx, 32, params=ag.FlowParams(conschm=553))
