"""Device selection of the C ABI: every call on a context runs on that context's device and
leaves the caller's current device as it found it. On a one-GPU machine the second half (a
context on another device than the current one) cannot run and is skipped."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _current_device():
    from cuda.bindings import runtime as rt   # the CUDA runtime's own view, not torch's cache
    err, dev = rt.cudaGetDevice()
    assert err == rt.cudaError_t.cudaSuccess
    return dev


def _exercise(ctx, n=24):
    import astr_gpu_b200 as ag
    s = ag.TGVSolver(ctx, n)
    s.init_tgv()
    dt = s.cfl_dt(0.5)
    s.rk3(dt, 2)
    q = s.get_q()
    s.close()
    return q


def test_calls_keep_the_callers_device():
    import torch
    import astr_gpu_b200 as ag
    torch.cuda.set_device(0)
    before = _current_device()
    ctx = ag.Context(0)
    assert _current_device() == before
    q = _exercise(ctx)
    assert np.isfinite(q).all()
    assert _current_device() == before
    ctx.close()


@pytest.mark.skipif("__import__('torch').cuda.device_count() < 2", reason="needs two GPUs")
def test_context_on_another_device():
    import torch
    import astr_gpu_b200 as ag
    torch.cuda.set_device(0)
    ref = _exercise(ag.Context(0))
    ctx1 = ag.Context(1)
    assert _current_device() == 0
    q = _exercise(ctx1)
    assert _current_device() == 0
    np.testing.assert_array_equal(q, ref)
