"""Line-level parity of the compact interface flux: astr_flux_lines (the drop-in for
flux_compact, flux.F90:125-150) and astr_flux_diff_lines (fh(i) - fh(i-1), solver.F90:1509-1513)
against the oracle on identical seeded inputs: every ntype, both winds, b factors 0 and 1 and
one in between, every direction, lines from 32 to 1148 interfaces (the longest system, 1152
rows, of the largest solve layout). Tolerance: relative
L-infinity <= 1e-12 per call (relative to max |oracle output|).

The reference's own flux test (test.F90:675-870: 128^3, x and z periodic, y one block with
both ends physical on [0, 2], bfacmpld = 1, the test function sin x sin(pi y / 2) sin z) runs
through the same calls, checked against the oracle and against the analytic gradient."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
HM = 5
TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    import astr_gpu_b200 as ag
    return ag.Context(0)


def _field(shape, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal(shape))


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("ntype", [1, 2, 3, 4])
@pytest.mark.parametrize("wind", ["+", "-"])
@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("dim,bfac", [(32, 0.0), (100, 1.0), (256, 0.37), (512, 1.0), (1000, 0.0), (1148, 0.5)])
def test_flux_lines(ctx, ntype, wind, direction, dim, bfac):
    import astr_gpu_b200 as ag
    shape = [6, 5, 7]
    shape[direction] = dim + 1 + 2 * HM
    lb = [0, 0, 0]
    lb[direction] = -HM
    f = _field(shape + [2], 7 * ntype + direction + dim)
    ref = oracle.compact_flux_initiate(ntype, dim, wind, bfac).apply3d(f, direction, lbound=lb)
    s = ag.compact_flux_initiate(ctx, ntype, dim, wind, bfac)
    got = ag.flux_compact(ctx, s, f, direction, lbound=lb)
    assert got.shape == ref.shape
    assert _rel(got, ref) <= TOL


@pytest.mark.parametrize("ntype", [1, 2, 3, 4])
@pytest.mark.parametrize("wind", ["+", "-"])
def test_flux_difference_lines(ctx, ntype, wind):
    import astr_gpu_b200 as ag
    dim, direction = 130, 1
    f = _field((9, dim + 1 + 2 * HM, 4), 50 + ntype)
    lb = (0, -HM, 0)
    fh = oracle.compact_flux_initiate(ntype, dim, wind, 1.0).apply3d(f, direction, lbound=lb)
    ref = 3.0 * (fh[:, 1:, :] - fh[:, :-1, :])
    got = ag.flux_difference(ctx, ag.compact_flux_initiate(ctx, ntype, dim, wind, 1.0), f, direction, lbound=lb,
                             scale=3.0)
    assert got.shape == ref.shape
    assert _rel(got, ref) <= TOL


def test_flux_lines_on_device_tensors(ctx):
    """The device path (torch tensors in HBM, Fortran strides) gives the host path's result."""
    import torch
    import astr_gpu_b200 as ag
    dim = 64
    f = _field((dim + 1 + 2 * HM, 8, 8), 3)
    lb = (-HM, 0, 0)
    s = ag.compact_flux_initiate(ctx, 3, dim, "-", 1.0)
    host = ag.flux_compact(ctx, s, f, 0, lbound=lb)
    ft = torch.from_numpy(np.ascontiguousarray(f.T)).cuda().T
    dev = ag.flux_compact(ctx, s, ft, 0, lbound=lb)
    np.testing.assert_array_equal(dev.cpu().numpy(), host)


def test_flux_rejects_bad_arguments(ctx):
    import astr_gpu_b200 as ag
    with pytest.raises(ValueError):
        ag.compact_flux_initiate(ctx, 3, 64, "x", 0.0)
    with pytest.raises(ag.AstrError):
        ag.compact_flux_initiate(ctx, 3, 64, "+", 0.0, scheme=553)
    with pytest.raises(ag.AstrError):
        ag.compact_flux_initiate(ctx, 5, 64, "+", 0.0)
    s = ag.compact_flux_initiate(ctx, 3, 32, "+", 0.0)
    f = _field((32 + 1 + 2 * HM, 3, 3), 1)
    with pytest.raises(ag.AstrError):   # output must cover interfaces -1..dim
        ag.flux_compact(ctx, s, f, 0, lbound=(-HM, 0, 0), out_lbound=(0, 0, 0), out_shape=(33, 3, 3))
    with pytest.raises(ag.AstrError):   # a derivative scheme is not a flux
        ag.flux_compact(ctx, ag.fd_scheme_initiate(ctx, "643c", 3, 32), f, 0, lbound=(-HM, 0, 0))


def test_reference_flux_test_configuration(ctx):
    """fluxtest (test.F90:675-870): 128^3, x and z periodic (ntype 3), y one block with both ends
    physical (ntype 4) on [0, 2], bfacmpld = 1, f = sin x sin(pi y / 2) sin z. The flux-form
    gradient (fh(i) - fh(i-1)) / dx per direction matches the oracle per call, and its L2 error
    against the analytic gradient is that of a high-order scheme (the reference prints it)."""
    import astr_gpu_b200 as ag
    n = 128
    x = 2 * np.pi * np.arange(-HM, n + HM + 1) / n
    y = 2.0 * np.arange(-HM, n + HM + 1) / n
    z = x
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    v = np.asfortranarray(np.sin(X) * np.sin(0.5 * np.pi * Y) * np.sin(Z))
    inner = (slice(HM, HM + n + 1),) * 3
    exact = [np.cos(X) * np.sin(0.5 * np.pi * Y) * np.sin(Z),
             0.5 * np.pi * np.sin(X) * np.cos(0.5 * np.pi * Y) * np.sin(Z),
             np.sin(X) * np.sin(0.5 * np.pi * Y) * np.cos(Z)]
    h = (2 * np.pi / n, 2.0 / n, 2 * np.pi / n)
    ntypes = (3, 4, 3)
    errs = []
    for d in range(3):
        # the line array of the test: halos along d only, nodes 0..n on the other axes
        sl = [slice(HM, HM + n + 1)] * 3
        sl[d] = slice(0, n + 1 + 2 * HM)
        f = np.asfortranarray(v[tuple(sl)])
        lb = [0, 0, 0]
        lb[d] = -HM
        fh = oracle.compact_flux_initiate(ntypes[d], n, "+", 1.0).apply3d(f, d, lbound=lb)
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[d] = slice(1, None)
        b[d] = slice(None, -1)
        ref = (fh[tuple(a)] - fh[tuple(b)]) / h[d]
        got = ag.flux_difference(ctx, ag.compact_flux_initiate(ctx, ntypes[d], n, "+", 1.0), f, d, lbound=lb,
                                 scale=1.0 / h[d])
        assert _rel(got, ref) <= TOL
        e = got[1:, 1:, 1:] - exact[d][inner][1:, 1:, 1:]
        errs.append(np.sqrt((e ** 2).sum() / n ** 3))
    assert max(errs[0], errs[2]) < 1e-10    # periodic: 6th order at b = 1 (4.4e-12 in the oracle)
    assert errs[1] < 5e-5                   # the 3rd-order physical closures dominate (1.1e-5)
