"""Flow-field checkpoints of the solver states against the oracle: writeflfed's flow field
(src/readwrite.F90:1720-1979) and readcheckpoint + updateq (src/readwrite.F90:1378-1528,
src/fludyna.F90:254-300), through astr_state_* / astr_full_* {write,read}_flowfield.

Files are checked with the oracle's HDF5 reader and made by the oracle's HDF5 writer
(oracle/h5format.py). Bars: the written primitives equal the oracle's q2fvar of the state's q bit
for bit (miniapp state; the conversion is evaluated without contraction), or within 4e-15 of each
field's largest value (full solver, whose primitive arrays come from its own updatefvar kernel);
q after a read equals the oracle's fvar2q of the file's fields bit for bit; steps after a restart
match the oracle's restart (the same file, the same steps) within the step tests' 1e-10."""
import numpy as np
import pytest

import oracle
from oracle import h5format

pytestmark = pytest.mark.gpu
NAMES = ("ro", "u1", "u2", "u3", "p", "t")


@pytest.fixture(scope="module")
def ctx():
    import astr_gpu_b200 as ag
    return ag.Context(0)


def _prims(shape, mach, seed):
    """A smooth compressible field (ro, u1, u2, u3, p, t) with t = p / ro * gamma M^2."""
    rng = np.random.default_rng(seed)
    x = [2 * np.pi * np.arange(n) / (n - 1) for n in shape]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    ro = 1.0 + 0.05 * np.sin(X + Y) * np.cos(Z) + 0.01 * rng.random()
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z) + 0.1 * np.sin(Z)
    w = 0.2 * np.sin(Y + Z)
    p = 1.0 / (1.4 * mach ** 2) + 0.1 * np.cos(2 * X) * np.cos(Y)
    return np.asfortranarray(np.stack([ro, u, v, w, p, p / ro * 1.4 * mach ** 2], axis=-1))


def _write_oracle_file(fn, prims, nstep, time, stream=False):
    if stream:
        items = [(n, prims[..., m].ravel(order="F")) for m, n in enumerate(NAMES)]
    else:
        items = [(n, np.ascontiguousarray(prims[..., m].T)) for m, n in enumerate(NAMES)]
    items += [("nstep", np.array([nstep], dtype=np.int32)), ("time", np.array([time]))]
    h5format.write(fn, items)


def _file_prims(fn):
    info = h5format.read(fn)
    prims = np.asfortranarray(np.stack([info.entries[n].data.T for n in NAMES], axis=-1))
    return prims, int(info.entries["nstep"].data[0]), float(info.entries["time"].data[0])


def _rel(a, b):
    return max(float(np.abs(a[..., m] - b[..., m]).max() / np.abs(b[..., m]).max()) for m in range(a.shape[-1]))


def _rel_q(a, b):
    """Per conserved field, relative to its largest value; the momentum components share the
    largest momentum (a Taylor-Green box's z-momentum is rounding-sized)."""
    mom = max(np.abs(b[..., m]).max() for m in (1, 2, 3))
    scale = [np.abs(b[..., 0]).max(), mom, mom, mom, np.abs(b[..., 4]).max()]
    return max(float(np.abs(a[..., m] - b[..., m]).max() / scale[m]) for m in range(5))


def test_state_writes_q2fvar_of_its_q(ctx, tmp_path):
    import astr_gpu_b200 as ag
    s = ag.TGVSolver(ctx, 24, 20, 16)
    s.init_tgv()
    dt = s.cfl_dt(0.5)
    s.rk3(dt, 3)
    fn = tmp_path / "flowfield.h5"
    s.write_flowfield(fn)
    prims, nstep, time = _file_prims(fn)
    assert prims.shape == (25, 21, 17, 6)
    ref = oracle.q2fvar(s.get_q(), s.params.mach, s.params.gamma)
    assert np.array_equal(prims, ref)
    t = 0.0
    for _ in range(3):
        t = t + dt
    assert (nstep, time) == (3, t)
    s.close()


@pytest.mark.parametrize("stream", [False, True])
def test_state_reads_an_oracle_written_flowfield(ctx, tmp_path, stream):
    import astr_gpu_b200 as ag
    dims = (24, 20, 16)
    p = ag.FlowParams(mach=0.2)
    prims = _prims(tuple(n + 1 for n in dims), 0.2, 3)
    fn = tmp_path / "flowfield.h5"
    _write_oracle_file(fn, prims, 1200, 12.5, stream)
    s = ag.TGVSolver(ctx, *dims, params=p)
    assert s.read_flowfield(fn, "s" if stream else "h") == (1200, 12.5)
    assert np.array_equal(s.get_q(), oracle.fvar2q_temperature(prims, 0.2, 1.4))
    s.rk3(1e-3, 2)
    h = s.history()
    assert h[:, 0].tolist() == [1200.0, 1201.0] and h[:, 1].tolist() == [12.5, 12.5 + 1e-3]
    s.close()


def test_state_reads_fields_stored_otherwise(ctx, tmp_path):
    """Fields the chunked transfers cannot take directly (big-endian float32 in a file with a user
    block and version-2 layout messages) go through the converting reader: q is the oracle's
    fvar2q of the widened values."""
    import astr_gpu_b200 as ag
    dims = (24, 20, 16)
    prims = _prims(tuple(n + 1 for n in dims), 0.1, 4).astype(np.float32)
    items = [(n, np.ascontiguousarray(prims[..., m].T)) for m, n in enumerate(NAMES)]
    items += [("nstep", np.array([3], dtype=np.int64)), ("time", np.array([0.125], dtype=np.float32))]
    fn = tmp_path / "f32.h5"
    h5format.write(fn, items, user_block=512, layout_version=2, byte_order=">")
    s = ag.TGVSolver(ctx, *dims)
    assert s.read_flowfield(fn) == (3, 0.125)
    assert np.array_equal(s.get_q(), oracle.fvar2q_temperature(prims.astype(np.float64), 0.1, 1.4))
    s.close()


def test_state_reads_a_version2_file(ctx, tmp_path):
    """A flow field in the format's version-2 layout (checksummed headers, compact links)."""
    import astr_gpu_b200 as ag
    dims = (24, 20, 16)
    prims = _prims(tuple(n + 1 for n in dims), 0.1, 8)
    items = [(n, np.ascontiguousarray(prims[..., m].T)) for m, n in enumerate(NAMES)]
    h5format.write_v2(tmp_path / "v2.h5", items + [("nstep", np.array([11], np.int32)), ("time", np.array([0.5]))])
    s = ag.TGVSolver(ctx, *dims)
    assert s.read_flowfield(tmp_path / "v2.h5") == (11, 0.5)
    assert np.array_equal(s.get_q(), oracle.fvar2q_temperature(prims, 0.1, 1.4))
    s.close()


def test_state_restart_continues_the_run(ctx, tmp_path):
    """Four steps, checkpoint, four more steps; a second state restarted from the checkpoint takes
    the same four steps. Both agree with the oracle restarted from the same file."""
    import astr_gpu_b200 as ag
    n = 32
    a = ag.TGVSolver(ctx, n)
    a.init_tgv()
    dt = a.cfl_dt(0.5)
    a.rk3(dt, 4)
    fn = tmp_path / "flowfield.h5"
    a.write_flowfield(fn)
    a.rk3(dt, 4)
    b = ag.TGVSolver(ctx, n)
    nstep, time = b.read_flowfield(fn)
    assert nstep == 4
    b.rk3(dt, 4)
    prims, _, _ = _file_prims(fn)
    o = oracle.TGVOracle(n)
    o.set_q(oracle.fvar2q_temperature(prims, a.params.mach, a.params.gamma))
    o.set_dt(dt)
    o.steps(4)
    assert _rel_q(b.get_q(), o.get_q()) <= 1e-10
    assert _rel_q(b.get_q(), a.get_q()) <= 1e-12
    assert b.history()[:, 0].tolist() == [4.0, 5.0, 6.0, 7.0]
    a.close()
    b.close()


@pytest.mark.parametrize("ntype", [(3, 3, 3), (3, 4, 3)])
def test_full_solver_checkpoint_and_restart(ctx, tmp_path, ntype):
    """The full solver writes its primitive arrays; a restart from the file (q by fvar2q, the
    interior primitives as read) continues like the oracle's full-solver mode restarted from the
    same file, walls included."""
    import astr_gpu_b200 as ag
    dims, mach = (32, 40, 28), 0.2
    kw = dict(mach=mach, reynolds=500.0, sutherland=110.3, beta_bound=0.98, ntype=ntype, twall=1.0)
    shape = tuple(n + 1 for n in dims)
    q = oracle.fvar2q_temperature(_prims(shape, mach, 5), mach, 1.4)
    if ntype[1] == 4:      # no-slip wall values at y = 0 and y = L, as the walled tests start
        q[:, 0, :, 1:4] = 0.0
        q[:, -1, :, 1:4] = 0.0
    s = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    s.set_q(q)
    s.step(1e-3, 3)
    fn = tmp_path / "flowfield.h5"
    s.write_flowfield(fn)
    prims, nstep, time = _file_prims(fn)
    assert nstep == 3 and abs(time - 3e-3) < 1e-15
    assert _rel(prims, oracle.q2fvar(s.get_q(), mach, 1.4)) <= 4e-15
    s2 = ag.FullSolver(ctx, *dims, params=ag.FlowParams(**kw))
    assert s2.read_flowfield(fn) == (3, time)
    assert np.array_equal(s2.get_q(), oracle.fvar2q_temperature(prims, mach, 1.4))
    s2.step(1e-3, 3)
    o = oracle.TGVOracle(*dims, params=oracle.FlowParams(**kw))
    o.set_flowfield(prims)
    o.set_dt(1e-3)
    o.steps_full(3)
    assert _rel_q(s2.get_q(), o.get_q()) <= 1e-10
    assert s2.history()[:, 0].tolist() == [3.0, 4.0, 5.0]
    s.close()
    s2.close()


def test_full_solver_reads_a_stream_file(ctx, tmp_path):
    """readcheckpoint's mode 's' (h5ra3d_r8_stream): 1-D datasets of the block's nodes."""
    import astr_gpu_b200 as ag
    dims, mach = (20, 24, 16), 0.2
    prims = _prims(tuple(n + 1 for n in dims), mach, 6)
    fn = tmp_path / "stream.h5"
    _write_oracle_file(fn, prims, 40, 2.0, stream=True)
    s = ag.FullSolver(ctx, *dims, params=ag.FlowParams(mach=mach, sutherland=110.3))
    assert s.read_flowfield(fn, "s") == (40, 2.0)
    assert np.array_equal(s.get_q(), oracle.fvar2q_temperature(prims, mach, 1.4))
    s.write_flowfield(tmp_path / "back.h5")
    back, nstep, time = _file_prims(tmp_path / "back.h5")
    assert (nstep, time) == (40, 2.0)
    assert np.array_equal(back, prims)       # the primitives as read, written back unchanged
    s.close()


def test_flowfield_refusals_leave_the_state_unchanged(ctx, tmp_path):
    import astr_gpu_b200 as ag
    s = ag.TGVSolver(ctx, 24, 20, 16)
    s.init_tgv()
    q0 = s.get_q()
    other = ag.TGVSolver(ctx, 20, 20, 16)
    other.init_tgv()
    other.write_flowfield(tmp_path / "other.h5")
    prims = _prims((25, 21, 17), 0.1, 1)
    _write_oracle_file(tmp_path / "h.h5", prims, 1, 0.5)
    h5format.write(tmp_path / "nop.h5", [(n, np.ascontiguousarray(prims[..., m].T)) for m, n in enumerate(NAMES)
                                         if n != "p"] + [("nstep", np.array([1], np.int32)), ("time", np.array([0.5]))])
    for fn, mode in [("other.h5", "h"), ("nop.h5", "h"), ("h.h5", "s"), ("h.h5", "x"), ("missing.h5", "h")]:
        with pytest.raises(ag.AstrError):
            s.read_flowfield(tmp_path / fn, mode)
        assert np.array_equal(s.get_q(), q0)
    with pytest.raises(ag.AstrError):
        s.write_flowfield(tmp_path / "no_such_dir" / "f.h5")
    s.close()
    other.close()
