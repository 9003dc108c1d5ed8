"""Batched ensemble of uneven periodic boxes: stepping them together must give, box by box, the
state of stepping each box alone with the same solve layout, and the same history. The batched
pass kernels are separate compilations of the same code, so the compiler may contract a few
multiply-adds differently: states agree to rounding (<= 1e-12 of each field's largest value after
10 steps), not bitwise."""
import numpy as np
import pytest

import astr_gpu_b200 as ag
from astr_gpu_b200.fields import solenoidal_q

pytestmark = pytest.mark.gpu

PASSES = ["A", "B", "C", "A'", "B'", "F_C", "F_A"]


def group_layout(n):
    """Solve layout the library picks for a periodic box of n intervals (filter rows -3..n+3)."""
    rows = n + 7
    for lim, lay in ((96, (3, 1)), (160, (5, 1)), (288, (9, 1)), (576, (9, 2)), (1152, (9, 4))):
        if rows <= lim:
            return lay
    raise ValueError(n)


def make_box(ctx, spec, pin=False):
    p = ag.FlowParams(mach=spec.mach, reynolds=spec.reynolds)
    s = ag.TGVSolver(ctx, spec.n, params=p)
    if spec.kind == "tgv":
        s.init_tgv()
    else:
        s.set_q(solenoidal_q(spec.n, spec.mach, spec.seed))
    if pin:
        S, W = group_layout(spec.n)
        for nm in PASSES:
            s.set_launch_shape(nm, S, W, 4 if W == 1 else 2)
    return s


def assert_close_fields(qe, qr, what, tol=1e-12):
    for m in range(5):
        # momentum components share one scale (a component may stay near zero by symmetry)
        scale = np.abs(qr[..., 1:4]).max() if 1 <= m <= 3 else np.abs(qr[..., m]).max()
        err = np.abs(qe[..., m] - qr[..., m]).max()
        assert err <= tol * scale, (what, m, err, scale)


@pytest.fixture(scope="module")
def ctx():
    c = ag.Context(0)
    yield c
    c.close()


SPECS = [ag.fields.BoxSpec(32, 0.2, 800.0, "tgv", 0), ag.fields.BoxSpec(48, 0.45, 3000.0, "solenoidal", 11),
         ag.fields.BoxSpec(96, 0.1, 1600.0, "tgv", 0), ag.fields.BoxSpec(32, 0.3, 400.0, "solenoidal", 12),
         ag.fields.BoxSpec(64, 0.35, 2200.0, "solenoidal", 13)]


def test_ensemble_equals_boxes_alone(ctx):
    ens_boxes = [make_box(ctx, sp) for sp in SPECS]
    ref_boxes = [make_box(ctx, sp, pin=True) for sp in SPECS]
    dts = [b.cfl_dt(0.5) for b in ens_boxes]
    ens = ag.Ensemble(ctx, ens_boxes)
    ens.step(dts, 4)
    ens.step(dts, 6)       # second call: every box owes its last filter along A
    for b, r, dt in zip(ens_boxes, ref_boxes, dts):
        r.rk3(dt, 10)
    for sp, b, r in zip(SPECS, ens_boxes, ref_boxes):
        qe, qr = b.get_q(), r.get_q()
        assert_close_fields(qe, qr, sp)
        he, hr = b.history(), r.history()
        assert he.shape == hr.shape == (10, 5)
        np.testing.assert_array_equal(he[:, :2], hr[:, :2])
        np.testing.assert_allclose(he[:, 2:], hr[:, 2:], rtol=1e-12, atol=0)
    ens.close()


def test_ensemble_mixed_pending_and_dt_change(ctx):
    """A box that owes its filter while another does not, and a dt change between calls."""
    specs = SPECS[:3]
    ens_boxes = [make_box(ctx, sp) for sp in specs]
    ref_boxes = [make_box(ctx, sp, pin=True) for sp in specs]
    dts = np.array([b.cfl_dt(0.5) for b in ens_boxes])
    ens_boxes[0].rk3(dts[0], 1)          # box 0 owes its filter, the others do not
    ref_boxes[0].rk3(dts[0], 1)
    ens = ag.Ensemble(ctx, ens_boxes)
    ens.step(dts, 3)
    ens.step(dts * 0.5, 2)
    for i, (r, dt) in enumerate(zip(ref_boxes, dts)):
        r.rk3(dt, 3)
        r.rk3(dt * 0.5, 2)
    for sp, b, r in zip(specs, ens_boxes, ref_boxes):
        assert_close_fields(b.get_q(), r.get_q(), sp)
    ens.close()


def test_ensemble_tgv_box_matches_oracle(ctx):
    """A 32^3 box stepped inside an ensemble against the CPU oracle (<= 1e-10 after 5 steps)."""
    from oracle import TGVOracle, FlowParams as OFP
    sp = ag.fields.BoxSpec(32, 0.25, 1000.0, "solenoidal", 5)
    boxes = [make_box(ctx, sp), make_box(ctx, SPECS[2])]
    dt = boxes[0].cfl_dt(0.5)
    ens = ag.Ensemble(ctx, boxes)
    ens.step([dt, boxes[1].cfl_dt(0.5)], 5)
    o = TGVOracle(32, 32, 32, OFP(mach=sp.mach, reynolds=sp.reynolds))
    o.set_q(solenoidal_q(sp.n, sp.mach, sp.seed))
    o.set_dt(dt)
    o.steps(5)
    qo, qg = o.get_q(), boxes[0].get_q()
    err = np.abs(qg - qo).max() / np.abs(qo).max()
    assert err <= 1e-10, err
    ens.close()


def test_ensemble_rejects_bad_input(ctx):
    b = make_box(ctx, SPECS[0])
    ens = ag.Ensemble(ctx, [b])
    with pytest.raises(ag.AstrError):
        ens.step([-1.0], 1)
    ens.close()

