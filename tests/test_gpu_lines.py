"""Line-level parity: astr_deriv_lines / astr_filter_lines (the drop-in for fds%central and
compact_filter) against the oracle on identical seeded inputs, every ntype, every direction.
Tolerance: relative L-infinity <= 1e-12 per call (relative to max |oracle output|)."""
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
@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("dim", [32, 64, 128, 256])
def test_deriv_lines(ctx, ntype, direction, dim):
    import astr_gpu_b200 as ag
    n_other = 9
    shape = [n_other, n_other + 2, n_other + 1]
    shape[direction] = dim + 1 + 2 * HM
    lb = [0, 0, 0]
    lb[direction] = -HM
    f = _field(shape + [2], 10 * ntype + direction)
    ref = oracle.fd_scheme_initiate("643c", ntype, dim).apply3d(f, direction, lbound=lb)
    got = ag.central(ctx, ag.fd_scheme_initiate(ctx, "643c", ntype, dim), f, direction, lbound=lb)
    assert got.shape == ref.shape
    assert _rel(got, ref) <= TOL


@pytest.mark.parametrize("ntype", [1, 2, 3, 4])
@pytest.mark.parametrize("direction", [0, 1, 2])
@pytest.mark.parametrize("dim", [32, 100, 256, 512])
def test_filter_lines(ctx, ntype, direction, dim):
    import astr_gpu_b200 as ag
    shape = [7, 6, 5]
    shape[direction] = dim + 1 + 2 * HM
    lb = [0, 0, 0]
    lb[direction] = -HM
    f = _field(shape, 100 + ntype)
    ref = oracle.compact_filter_initiate(ntype, dim, 0.49, 1.11, 0.98).apply3d(f, direction, lbound=lb)
    got = ag.compact_filter(ctx, ag.compact_filter_initiate(ctx, ntype, dim, 0.49, 1.11, 0.98), f, direction, lbound=lb)
    assert _rel(got, ref) <= TOL


@pytest.mark.parametrize("ntype", [3, 4])
def test_filter_note_boundary_no_filter(ctx, ntype):
    import astr_gpu_b200 as ag
    dim = 64
    f = _field((dim + 1 + 2 * HM, 4, 3), 7)
    lb = (-HM, 0, 0)
    ref = oracle.compact_filter_initiate(ntype, dim, 0.49, 1.11, 0.98, boundary_no_filter=True).apply3d(f, 0, lbound=lb)
    got = ag.compact_filter(ctx, ag.compact_filter_initiate(ctx, ntype, dim, 0.49, 1.11, 0.98,
                                                            note="boundary_no_filter"), f, 0, lbound=lb)
    assert _rel(got, ref) <= TOL


@pytest.mark.parametrize("ntype", [1, 2, 3, 4])
def test_explicit_lines(ctx, ntype):
    import astr_gpu_b200 as ag
    dim = 48
    f = _field((5, dim + 1 + 2 * HM, 4), 3)
    lb = (0, -HM, 0)
    ref = oracle.fd_scheme_initiate("643e", ntype, dim).apply3d(f, 1, lbound=lb)
    got = ag.central(ctx, ag.fd_scheme_initiate(ctx, "643e", ntype, dim), f, 1, lbound=lb)
    assert _rel(got, ref) <= TOL


def test_scheme_tables_match_oracle(ctx):
    import astr_gpu_b200 as ag
    for ntype in (1, 2, 3, 4):
        a = ag.fd_scheme_initiate(ctx, "643c", ntype, 64).ac()
        f0, l0, a1, a2, a3 = oracle.fd_scheme_initiate("643c", ntype, 64).ac()
        assert (a[0], a[1]) == (f0, l0)
        np.testing.assert_array_equal(a[2][0], a1)
        np.testing.assert_array_equal(a[2][1][1:], a2[1:])
        b = ag.compact_filter_initiate(ctx, ntype, 64, 0.49, 1.11, 0.98).ac()
        f0, l0, b1, b2, b3 = oracle.compact_filter_initiate(ntype, 64, 0.49, 1.11, 0.98).ac()
        np.testing.assert_array_equal(b[2][0], b1)


def test_device_tensors_and_mixed_bc_gradient(ctx):
    """Config-1 shape in miniature: x,z periodic (ntype 3), y non-periodic (ntype 4), device
    arrays, derivative along each axis then the filter along each axis."""
    import torch
    import astr_gpu_b200 as ag
    n = 64
    rng = np.random.default_rng(5)
    f = np.asfortranarray(rng.standard_normal((n + 1 + 2 * HM, n + 1, n + 1 + 2 * HM)))
    lb = (-HM, 0, -HM)
    ft = torch.from_numpy(np.ascontiguousarray(f.T)).cuda().T  # Fortran-ordered view on device
    for d, nt in ((0, 3), (1, 4), (2, 3)):
        ref = oracle.fd_scheme_initiate("643c", nt, n).apply3d(f, d, lbound=lb)
        oshape = [n + 1, n + 1, n + 1]
        got = ag.central(ctx, ag.fd_scheme_initiate(ctx, "643c", nt, n), ft, d, lbound=lb,
                         out_lbound=(0, 0, 0), out_shape=oshape)
        sl = [slice(HM, HM + n + 1), slice(0, n + 1), slice(HM, HM + n + 1)]
        sl[d] = slice(None)
        assert _rel(got.cpu().numpy(), ref[tuple(sl)]) <= TOL


@pytest.mark.parametrize("direction", [0, 2])
def test_host_output_entries_outside_the_written_range_stay(ctx, direction):
    """A host output array whose range along the line reaches past nodes 0..dim (here the same
    halo'd layout as the input) gets nodes 0..dim from the call and keeps its other entries."""
    import ctypes
    import astr_gpu_b200 as ag
    from astr_gpu_b200 import _lib
    dim = 64
    shape = [7, 6, 5]
    shape[direction] = dim + 1 + 2 * HM
    lb = [0, 0, 0]
    lb[direction] = -HM
    f = _field(shape + [2], 77 + direction)
    ref = oracle.fd_scheme_initiate("643c", 3, dim).apply3d(f, direction, lbound=lb)
    out = np.full(f.shape, 5.5, order="F")
    s = ag.fd_scheme_initiate(ctx, "643c", 3, dim)
    i64 = lambda v: (ctypes.c_int64 * 3)(*v)
    ctx.check(ctx.L.astr_deriv_lines(ctx._h, s._h, direction, ctypes.c_void_p(f.ctypes.data), i64(shape), i64(lb),
                                     ctypes.c_void_p(out.ctypes.data), i64(shape), i64(lb), 2, 1.0, _lib.ASTR_HOST))
    inner = [slice(None)] * 4
    inner[direction] = slice(HM, HM + dim + 1)
    assert _rel(out[tuple(inner)], ref) <= TOL
    keep = np.ones(f.shape, dtype=bool)
    keep[tuple(inner)] = False
    assert np.all(out[keep] == 5.5)
