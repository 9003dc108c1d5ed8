"""astr_cfl_dt_noalloc: the CFL time step for callers that cannot let the library allocate
device memory (a solver running inside one fixed device pool or a capped allocator, where a
cudaMalloc fails or synchronises the device mid-step). Its scratch is a static device array;
its result must equal that of astr_cfl_dt on the same field, call after call.

This file is collected last so that a run stopping at the first failure has run every other
test before it."""
import ctypes

import numpy as np
import pytest

from astr_gpu_b200 import _lib


def _i64(v):
    return (ctypes.c_int64 * 3)(*[int(x) for x in v])


def test_rejects_sizes_beyond_its_scratch_without_touching_the_gpu():
    L = _lib.load()
    dt = ctypes.c_double()
    big = 1000   # (1001)^2 x lines > 524288
    rc = L.astr_cfl_dt_noalloc(None, ctypes.c_void_p(8), _i64((big + 1,) * 3), _i64((0, 0, 0)), big, big, big,
                               0.1, 1.4, 0.5, ctypes.byref(dt))
    assert rc == _lib.ASTR_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_noalloc_cfl_matches_astr_cfl_dt_twice():
    import torch
    import astr_gpu_b200 as ag
    ctx = ag.Context(0)
    L = ctx.L
    for n, seed in ((48, 0), (96, 1)):
        s = ag.TGVSolver(ctx, n)
        s.init_tgv()
        q = s.get_q()
        # perturb the velocity so the two calls see different fields
        q[..., 1] *= 1.0 + 0.1 * seed
        s.set_q(q)
        ref = s.cfl_dt(0.5)
        # the same field as a Fortran-ordered device array with a halo of 2 nodes
        qh = np.zeros((n + 5, n + 5, n + 5, 5), order="F")
        qh[2:n + 3, 2:n + 3, 2:n + 3, :] = q
        qd = torch.from_numpy(np.ascontiguousarray(qh.transpose(3, 2, 1, 0))).cuda()
        torch.cuda.synchronize()
        dt = ctypes.c_double()
        rc = L.astr_cfl_dt_noalloc(ctx._h, ctypes.c_void_p(qd.data_ptr()), _i64(qh.shape[:3]), _i64((-2, -2, -2)),
                                   n, n, n, 0.1, 1.4, 0.5, ctypes.byref(dt))
        assert rc == 0, L.astr_last_error(ctx._h)
        assert abs(dt.value - ref) <= 1e-15 * ref
        s.close()
