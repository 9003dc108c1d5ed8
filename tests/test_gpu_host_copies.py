"""Host arrays in ordinary (pageable) memory: above 32 MB the state's upload and download move them
through pinned staging slots with several host threads instead of the driver's own staging. The
results must be bit for bit those of the same calls on pinned memory, for the miniapp state
(astr_state_upload / _download / astr_rk3_step_host) and the full solver (astr_full_upload /
_download), in both directions, at sizes that exercise whole and partial staging chunks; arrays
with halos go whole to the device and come back node rows only."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import astr_gpu_b200 as ag
    return ag.Context(0)


def _pinned_like(a):
    import torch
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    t.numpy()[:] = a.ravel(order="F")
    return t


def _i64(v):
    return (ctypes.c_int64 * 3)(*v)


@pytest.mark.parametrize("n", [128, 161])
def test_state_copies_and_host_step_agree_with_pinned(ctx, n):
    import astr_gpu_b200 as ag
    from astr_gpu_b200 import _lib
    s = ag.TGVSolver(ctx, n)
    s.autotune(False)
    s.init_tgv()
    q0 = s.get_q()                         # a pageable download (> 32 MB for both sizes)
    assert q0.nbytes >= 32 << 20
    pinned = _pinned_like(q0)
    got = np.asfortranarray(pinned.numpy().reshape(q0.shape, order="F"))
    assert np.array_equal(got, q0)         # pinned and pageable downloads agree
    # an upload of a perturbed field from pageable memory equals the one from pinned memory
    rng = np.random.default_rng(n)
    q1 = np.asfortranarray(q0 * (1.0 + 1e-3 * rng.standard_normal(q0.shape)))
    s.set_q(q1)
    assert np.array_equal(s.get_q(), q1)
    p1 = _pinned_like(q1)
    shape, lb = _i64(q1.shape[:3]), _i64((0, 0, 0))
    ctx.check(ctx.L.astr_state_upload(s._h, ctypes.c_void_p(p1.data_ptr()), shape, lb, _lib.ASTR_HOST))
    assert np.array_equal(s.get_q(), q1)
    # two host steps from each kind of memory
    dt = s.cfl_dt(0.5)
    qa = q1.copy(order="F")
    for _ in range(2):
        ctx.check(ctx.L.astr_rk3_step_host(s._h, ctypes.c_void_p(qa.ctypes.data), shape, lb, dt, 1, None))
    for _ in range(2):
        ctx.check(ctx.L.astr_rk3_step_host(s._h, ctypes.c_void_p(p1.data_ptr()), shape, lb, dt, 1, None))
    qb = np.asfortranarray(p1.numpy().reshape(q1.shape, order="F"))
    assert np.array_equal(qa, qb)
    s.close()


def test_full_solver_copies_agree_with_pinned(ctx):
    import astr_gpu_b200 as ag
    from astr_gpu_b200 import _lib
    from astr_gpu_b200.fields import tgv_q
    n = 136
    s = ag.FullSolver(ctx, n)
    q = tgv_q(n, 0.1)
    assert q.nbytes >= 32 << 20
    s.set_q(q)                             # pageable
    a = s.get_q()                          # pageable
    assert np.array_equal(a, q)
    p = _pinned_like(q)
    shape, lb = _i64(q.shape[:3]), _i64((0, 0, 0))
    ctx.check(ctx.L.astr_full_upload(s._h, ctypes.c_void_p(p.data_ptr()), shape, lb, _lib.ASTR_HOST))
    s.step(1e-3, 1)
    b = s.get_q()
    ctx.check(ctx.L.astr_full_download(s._h, ctypes.c_void_p(p.data_ptr()), shape, lb, _lib.ASTR_HOST))
    assert np.array_equal(b, np.asfortranarray(p.numpy().reshape(q.shape, order="F")))
    s.close()


def test_state_halo_arrays_agree_with_pinned_and_keep_their_halos(ctx):
    """Arrays with halos (the reference's q(-hm:im+hm, ...)): from pageable memory they go whole to
    the device and come back node rows only; the results equal the pinned path's (pitched copies)
    and the caller's halo entries are left as they were."""
    import astr_gpu_b200 as ag
    from astr_gpu_b200 import _lib
    n, hm = 128, 5
    s = ag.TGVSolver(ctx, n)
    s.autotune(False)
    s.init_tgv()
    q0 = s.get_q()
    full = (n + 1 + 2 * hm,) * 3 + (5,)
    assert np.prod(full) * 8 >= 32 << 20
    shape, lb = _i64(full[:3]), _i64((-hm, -hm, -hm))
    inner = (slice(hm, hm + n + 1),) * 3
    # pageable halo array: interior = q0, halos = a sentinel that must survive the download
    qa = np.full(full, 7.0, order="F")
    qa[inner] = q0
    ctx.check(ctx.L.astr_state_upload(s._h, ctypes.c_void_p(qa.ctypes.data), shape, lb, _lib.ASTR_HOST))
    assert np.array_equal(s.get_q(), q0)
    dt = s.cfl_dt(0.5)
    ctx.check(ctx.L.astr_rk3_step_host(s._h, ctypes.c_void_p(qa.ctypes.data), shape, lb, dt, 1, None))
    halo = np.ones(full[:3], dtype=bool)
    halo[inner] = False
    assert np.all(qa[halo] == 7.0)
    # the same step from a pinned halo array (pitched copies)
    s.set_q(q0)
    qp = _pinned_like(np.full(full, 7.0, order="F"))
    qpv = qp.numpy().reshape(full, order="F")
    qpv[inner] = q0
    ctx.check(ctx.L.astr_rk3_step_host(s._h, ctypes.c_void_p(qp.data_ptr()), shape, lb, dt, 1, None))
    assert np.array_equal(qa, qpv)
    # a download into a pageable halo array leaves its halos alone
    qd = np.full(full, -3.0, order="F")
    ctx.check(ctx.L.astr_state_download(s._h, ctypes.c_void_p(qd.ctypes.data), shape, lb, _lib.ASTR_HOST))
    assert np.array_equal(qd[inner], qpv[inner]) and np.all(qd[halo] == -3.0)
    s.close()


@pytest.mark.parametrize("n", [40, 128])
def test_full_solver_halo_downloads_keep_the_halos(ctx, n):
    """The full solver's download into an array with halos (the reference's own q layout) writes
    nodes 0..N only, from pageable (small and staged) and pinned memory alike."""
    import astr_gpu_b200 as ag
    from astr_gpu_b200 import _lib
    from astr_gpu_b200.fields import tgv_q
    hm = 5
    s = ag.FullSolver(ctx, n)
    q = tgv_q(n, 0.1)
    full = (n + 1 + 2 * hm,) * 3 + (5,)
    inner = (slice(hm, hm + n + 1),) * 3
    shape, lb = _i64(full[:3]), _i64((-hm, -hm, -hm))
    halo = np.ones(full[:3], dtype=bool)
    halo[inner] = False
    qa = np.full(full, 9.0, order="F")
    qa[inner] = q
    ctx.check(ctx.L.astr_full_upload(s._h, ctypes.c_void_p(qa.ctypes.data), shape, lb, _lib.ASTR_HOST))
    assert np.array_equal(s.get_q(), q)
    s.step(1e-3, 1)
    ref = s.get_q()
    qd = np.full(full, -2.0, order="F")
    ctx.check(ctx.L.astr_full_download(s._h, ctypes.c_void_p(qd.ctypes.data), shape, lb, _lib.ASTR_HOST))
    assert np.array_equal(qd[inner], ref) and np.all(qd[halo] == -2.0)
    qp = _pinned_like(np.full(full, -4.0, order="F"))
    ctx.check(ctx.L.astr_full_download(s._h, ctypes.c_void_p(qp.data_ptr()), shape, lb, _lib.ASTR_HOST))
    qpv = qp.numpy().reshape(full, order="F")
    assert np.array_equal(qpv[inner], ref) and np.all(qpv[halo] == -4.0)
    s.close()


def test_line_calls_on_large_pageable_arrays_agree_with_pinned(ctx):
    """astr_deriv_lines / astr_filter_lines on a host field of more than 32 MB: the staged copies
    of a pageable array give the pinned array's result bit for bit."""
    import torch
    import astr_gpu_b200 as ag
    from astr_gpu_b200 import _lib
    dim, hm = 256, 5
    shape = (dim + 1, dim + 1 + 2 * hm, 70)
    lb = (0, -hm, 0)
    f = np.asfortranarray(np.random.default_rng(3).standard_normal(shape))
    assert f.nbytes >= 32 << 20
    i64 = lambda v: (ctypes.c_int64 * 3)(*v)
    oshape = (dim + 1, dim + 1, 70)
    for make, call in ((lambda: ag.fd_scheme_initiate(ctx, "643c", 4, dim), ctx.L.astr_deriv_lines),
                       (lambda: ag.compact_filter_initiate(ctx, 4, dim), ctx.L.astr_filter_lines)):
        sch = make()
        a = np.zeros(oshape, order="F")
        args = (ctx._h, sch._h, 1, ctypes.c_void_p(f.ctypes.data), i64(shape), i64(lb), ctypes.c_void_p(a.ctypes.data),
                i64(oshape), i64((0, 0, 0)), 1)
        ctx.check(call(*args, 1.0, _lib.ASTR_HOST) if call is ctx.L.astr_deriv_lines else call(*args, _lib.ASTR_HOST))
        fp = torch.from_numpy(f.ravel(order="F")).pin_memory()
        bp = torch.zeros(int(np.prod(oshape)), dtype=torch.float64).pin_memory()
        args = (ctx._h, sch._h, 1, ctypes.c_void_p(fp.data_ptr()), i64(shape), i64(lb), ctypes.c_void_p(bp.data_ptr()),
                i64(oshape), i64((0, 0, 0)), 1)
        ctx.check(call(*args, 1.0, _lib.ASTR_HOST) if call is ctx.L.astr_deriv_lines else call(*args, _lib.ASTR_HOST))
        assert np.array_equal(a, bp.numpy().reshape(oshape, order="F"))
