"""B200-native (sm_100a) implementation of ASTR's per-step RHS hot path.

Host-side mirror of the reference's interface (Perrbit/astr_gpu), over the C ABI of
``include/astr_b200.h``:

* ``fd_scheme_initiate`` / ``compact_filter_initiate``  (src/derivative.F90:63, src/filter.F90:31)
* ``central`` — ``fds%central`` over every line of an array (src/derivative.F90:22-41)
* ``compact_filter`` — every line of an array (src/filter.F90:112)
* ``TGVSolver`` — the Taylor-Green miniapp driver: ``flowfield_init``, ``rhscal``, ``rk3``,
  ``stacal`` (miniapps/tgv_solver_3d/tgvsolver.F90)
* ``FullSolver`` — the full solver's ``time_integration_rk`` / ``rhscal`` on a periodic box
  (src/mainloop.F90:298-476, src/solver.F90:184-283)
* ``h5io_init`` / ``H5File`` — the HDF5 file interface of the reference's checkpoints
  (src/hdf5io.F90: h5io_init, h5write, h5read, h5io_end), without the HDF5 library; the solvers'
  ``write_flowfield`` / ``read_flowfield`` are writeflfed's flow field and readcheckpoint + updateq
  (src/readwrite.F90:1378-1528, 1720-1979)

Arrays are Fortran-ordered numpy arrays (host) or CUDA torch tensors laid out the same way
(device). All compute runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, fields

import numpy as np

from . import _lib
from ._lib import ASTR_DEVICE, ASTR_HOST, AstrParams

__all__ = ["AstrError", "Context", "Scheme", "fd_scheme_initiate", "compact_filter_initiate", "central",
           "compact_filter", "compact_flux_initiate", "flux_compact", "flux_difference", "FlowParams",
           "TGVSolver", "FullSolver", "Ensemble", "H5File", "h5io_init"]


class AstrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"astr error {code}: {msg}")
        self.code = code


def _i64(v):
    return (ctypes.c_int64 * 3)(*[int(x) for x in v])


class Context:
    """One device and one CUDA stream (``astr_init``). ``stream`` may be a ``torch.cuda.Stream``
    or a raw ``cudaStream_t`` integer; by default the library owns a non-blocking stream.
    ``strict`` runs everything made from this context through the strict-parity build of the
    library (no multiply-add contraction)."""

    def __init__(self, device: int = 0, stream=None, strict: bool = False):
        self.L = _lib.load(strict)
        h = ctypes.c_void_p()
        rc = self.L.astr_init(device, ctypes.byref(h))
        if rc != 0:
            raise AstrError(rc, "astr_init failed (no CUDA device?)")
        self._h = h
        self.device = device
        if stream is not None:
            raw = getattr(stream, "cuda_stream", stream)
            self.check(self.L.astr_set_stream(self._h, ctypes.c_void_p(int(raw))))

    def check(self, rc):
        if rc != 0:
            raise AstrError(rc, self.L.astr_last_error(self._h).decode())
        return rc

    def synchronize(self):
        self.check(self.L.astr_synchronize(self._h))

    def alive(self) -> bool:
        """False once the context is destroyed: the objects made on it then drop their handles
        without calling into the library (their device memory goes with the process)."""
        return bool(getattr(self, "_h", None))

    def close(self):
        if getattr(self, "_h", None):
            self.L.astr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scheme:
    """A ``compact_scheme`` living on the device (derivative, filter or interface flux)."""

    def __init__(self, ctx: Context, h, dim: int, ntype: int, is_filter: bool, wind: str | None = None):
        self.ctx, self._h, self.dim, self.ntype, self.is_filter = ctx, h, dim, ntype, is_filter
        self.wind = wind   # '+' or '-' for an interface-flux scheme, else None

    def ac(self):
        """(first_node, last_node, ac(3,n)) — the pre-factored Thomas table."""
        n = 0
        f, l = ctypes.c_int(), ctypes.c_int()
        buf = np.zeros(3 * (self.dim + 7))
        self.ctx.check(self.ctx.L.astr_scheme_ac(self._h, buf.ctypes.data_as(_lib._dp), ctypes.byref(f), ctypes.byref(l)))
        n = l.value - f.value + 1
        return f.value, l.value, buf[: 3 * n].reshape(n, 3).T.copy()

    def __del__(self):
        try:
            if getattr(self, "_h", None) and self.ctx.alive():
                self.ctx.L.astr_scheme_destroy(self._h)
                self._h = None
        except Exception:
            pass


def fd_scheme_initiate(ctx: Context, scheme: str, ntype: int, dim: int) -> Scheme:
    """derivative.F90:63 — '643c' (compact 6th order) or '643e' (explicit 6th order)."""
    h = ctypes.c_void_p()
    ctx.check(ctx.L.astr_fd_scheme_create(ctx._h, scheme.encode()[:4], ntype, dim, ctypes.byref(h)))
    return Scheme(ctx, h, dim, ntype, False)


def compact_filter_initiate(ctx: Context, ntype: int, dim: int, alfa: float = 0.49, beta_halo: float = 1.11,
                            beta_bound: float = 0.98, note: str | None = None) -> Scheme:
    """filter.F90:31 with filter_coefficient_cal(alfa, beta_halo, beta_bound) (filter.F90:299)."""
    h = ctypes.c_void_p()
    ctx.check(ctx.L.astr_filter_create(ctx._h, ntype, dim, alfa, beta_halo, beta_bound,
                                       int(note == "boundary_no_filter"), ctypes.byref(h)))
    return Scheme(ctx, h, dim, ntype, True)


def compact_flux_initiate(ctx: Context, ntype: int, dim: int, wind: str = "+", bfac: float = 0.0,
                          scheme: int = 543) -> Scheme:
    """flux.F90:32 — the '543' compact interface-flux scheme, ``wind`` '+' (upwind-biased,
    ``flux_uw_*``) or '-' (downwind-biased, ``flux_dw_*``), ``bfac`` the MP-LD b factor."""
    if wind not in ("+", "-"):
        raise ValueError("wind must be '+' or '-'")
    h = ctypes.c_void_p()
    ctx.check(ctx.L.astr_flux_create(ctx._h, scheme, ntype, dim, wind.encode(), float(bfac), ctypes.byref(h)))
    return Scheme(ctx, h, dim, ntype, False, wind)


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _apply(ctx, scheme, f, direction, lbound, out_lbound, out_shape, scale, kind):
    dim = scheme.dim
    nf = f.shape[3] if f.ndim == 4 else 1
    fshape = list(f.shape[:3])
    lb = list(lbound)
    # the interface flux spans interfaces -1..dim along the direction, everything else nodes 0..dim
    n_dir, lb_dir = (dim + 2, -1) if kind == "flux" else (dim + 1, 0)
    oshape = list(out_shape) if out_shape is not None else [fshape[d] if d != direction else n_dir for d in range(3)]
    olb = list(out_lbound) if out_lbound is not None else [lb[d] if d != direction else lb_dir for d in range(3)]
    if _is_torch(f):
        import torch
        assert f.is_cuda and f.dtype == torch.float64
        # Fortran order <=> the tensor's strides are column-major
        fp = f
        out = torch.empty(tuple(oshape) + ((nf,) if f.ndim == 4 else ()), dtype=torch.float64, device=f.device)
        out = out.permute(*reversed(range(out.ndim))).contiguous().permute(*reversed(range(out.ndim)))
        assert fp.stride(0) == 1 and out.stride(0) == 1, "device arrays must be Fortran-ordered"
        torch.cuda.current_stream(f.device).synchronize()
        fptr, optr, where = fp.data_ptr(), out.data_ptr(), ASTR_DEVICE
    else:
        fp = np.asfortranarray(f, dtype=np.float64)
        out = np.zeros(tuple(oshape) + ((nf,) if f.ndim == 4 else ()), order="F")
        fptr, optr, where = fp.ctypes.data, out.ctypes.data, ASTR_HOST
    L = ctx.L
    args = (ctx._h, scheme._h, direction, ctypes.c_void_p(fptr), _i64(fshape), _i64(lb), ctypes.c_void_p(optr),
            _i64(oshape), _i64(olb), nf)
    if kind == "filter":
        ctx.check(L.astr_filter_lines(*args, where))
    elif kind == "flux":
        ctx.check(L.astr_flux_lines(*args, where))
    elif kind == "fluxdiff":
        ctx.check(L.astr_flux_diff_lines(*args, float(scale), 0, where))
    else:
        ctx.check(L.astr_deriv_lines(ctx._h, scheme._h, direction, ctypes.c_void_p(fptr), _i64(fshape), _i64(lb),
                                     ctypes.c_void_p(optr), _i64(oshape), _i64(olb), nf, float(scale), where))
    if where == ASTR_DEVICE:
        ctx.synchronize()
    return out


def central(ctx: Context, scheme: Scheme, f, direction: int, lbound=(0, 0, 0), scale: float = 1.0,
            out_lbound=None, out_shape=None):
    """``df = fds%central(asolver, f, dim)`` for every line of ``f`` along ``direction``.
    ``f(lbound...)`` must carry nodes -5..dim+5 along ``direction`` when the scheme reads halos.
    The result spans nodes 0..dim along ``direction`` (index-space derivative times ``scale``)."""
    return _apply(ctx, scheme, f, direction, lbound, out_lbound, out_shape, scale, "deriv")


def compact_filter(ctx: Context, scheme: Scheme, f, direction: int, lbound=(0, 0, 0), out_lbound=None,
                   out_shape=None):
    """``ff = compact_filter(afilter, f, dim)`` for every line of ``f`` along ``direction``."""
    return _apply(ctx, scheme, f, direction, lbound, out_lbound, out_shape, 1.0, "filter")


def flux_compact(ctx: Context, scheme: Scheme, f, direction: int, lbound=(0, 0, 0), out_lbound=None,
                 out_shape=None):
    """``fh = flux_compact(asolver, f, dim)`` (flux.F90:125) for every line of ``f`` along
    ``direction``; the result spans interfaces -1..dim along ``direction`` (lower bound -1)."""
    return _apply(ctx, scheme, f, direction, lbound, out_lbound, out_shape, 1.0, "flux")


def flux_difference(ctx: Context, scheme: Scheme, f, direction: int, lbound=(0, 0, 0), scale: float = 1.0,
                    out_lbound=None, out_shape=None):
    """``scale * (fh(i) - fh(i-1))`` at nodes 0..dim of every line (the flux-form derivative of
    convrsdcmp, solver.F90:1509-1513, and of the reference's flux test, test.F90:755-765)."""
    return _apply(ctx, scheme, f, direction, lbound, out_lbound, out_shape, scale, "fluxdiff")


@dataclass
class FlowParams:
    """commvar of the miniapp (tgvsolver.F90:152-195, :253)."""
    mach: float = 0.1
    reynolds: float = 1600.0
    prandtl: float = 0.72
    gamma: float = 1.4
    ref_tem: float = 273.15
    sutherland: float = 110.4
    alfa_filter: float = 0.49
    beta_halo: float = 1.11
    beta_bound: float = 1.09
    filter_on: bool = True
    ntype: tuple = (3, 3, 3)   # per direction: 3 periodic; 1, 2, 4 physical ends (FullSolver only)
    twall: float = 1.0         # isothermal no-slip walls at the physical ends (bctype 41)
    conschm: int = 643         # convection: 643 central compact, 543 upwind compact flux (FullSolver only)
    bfacmpld: float = 0.0      # b factor of the upwind compact flux
    lchardecomp: bool = False  # upwind flux in characteristic variables with the Ducros sensor
    shkcrt: float = 0.01       # the Ducros sensor's threshold

    def c_params(self, im, jm, km):
        return AstrParams(im, jm, km, self.mach, self.reynolds, self.prandtl, self.gamma, self.ref_tem,
                          self.sutherland, self.alfa_filter, self.beta_halo, self.beta_bound, int(self.filter_on),
                          (ctypes.c_int * 3)(*[int(t) for t in self.ntype]), float(self.twall), int(self.conschm),
                          float(self.bfacmpld), int(self.lchardecomp), float(self.shkcrt))


class H5File:
    """One HDF5 file opened by ``h5io_init`` (src/hdf5io.F90:86-135): mode "read", "write"
    (create or truncate) or "rdwr" (add datasets to an existing file, as h5srite does). Arrays are
    Fortran-ordered: a dataset's HDF5 dataspace is the reversed shape, as the reference's Fortran
    HDF5 calls store it. Host memory only; needs no GPU."""

    def __init__(self, filename: str, mode: str = "read"):
        self.L = _lib.load()
        h = ctypes.c_void_p()
        rc = self.L.astr_h5io_init(str(filename).encode(), mode.encode(), ctypes.byref(h))
        if rc != 0:
            raise AstrError(rc, self.L.astr_h5_last_error(None).decode())
        self._h = h
        self.filename, self.mode = str(filename), mode

    def _check(self, rc):
        if rc != 0:
            raise AstrError(rc, self.L.astr_h5_last_error(self._h).decode())

    def names(self) -> list[str]:
        n = ctypes.c_int()
        self._check(self.L.astr_h5_count(self._h, ctypes.byref(n)))
        out = []
        for i in range(n.value):
            buf = ctypes.create_string_buffer(4096)
            self._check(self.L.astr_h5_name(self._h, i, buf, len(buf)))
            out.append(buf.value.decode())
        return out

    def info(self, varname: str):
        """(Fortran shape, type class 0 integer / 1 float / -1 other, element size)."""
        rank, cls, size = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        dims = (ctypes.c_int64 * 32)()
        self._check(self.L.astr_h5_dataset_info(self._h, varname.encode(), ctypes.byref(rank), dims,
                                                ctypes.byref(cls), ctypes.byref(size)))
        return tuple(dims[i] for i in range(rank.value)), cls.value, size.value

    def write(self, varname: str, var):
        """h5write: a real(8) or integer(4) dataset from a numpy array (float64 or int32)."""
        a = np.asfortranarray(var)
        dims = (ctypes.c_int64 * max(a.ndim, 1))(*(a.shape or (1,)))
        if a.dtype == np.int32:
            fn = self.L.astr_h5write_i4
        else:
            a = np.asfortranarray(a, dtype=np.float64)
            fn = self.L.astr_h5write_r8
        self._check(fn(self._h, varname.encode(), max(a.ndim, 1), dims, ctypes.c_void_p(a.ctypes.data)))

    def read(self, varname: str, shape=None, offset=None, mode: str = "h", dtype=np.float64) -> np.ndarray:
        """h5read: the block of Fortran `shape` at `offset` of the dataset (mode 'h'; default the
        whole dataset), or prod(shape) elements from element offset[0] of a 1-D dataset (mode 's',
        the stream layout); float64, or int32 for integer datasets."""
        if shape is None:
            shape = self.info(varname)[0]
        shape = tuple(int(x) for x in shape)
        scalar = len(shape) == 0           # a scalar dataspace: read as one element
        out = np.zeros(shape or (1,), dtype=np.int32 if np.dtype(dtype) == np.int32 else np.float64, order="F")
        shape = shape or (1,)
        dims = (ctypes.c_int64 * len(shape))(*shape)
        off = None if offset is None else (ctypes.c_int64 * len(offset))(*[int(x) for x in offset])
        fn = self.L.astr_h5read_i4 if out.dtype == np.int32 else self.L.astr_h5read_r8
        self._check(fn(self._h, varname.encode(), len(shape), dims, off, mode.encode(), ctypes.c_void_p(out.ctypes.data)))
        return out.reshape(()) if scalar else out

    def close(self):
        """h5io_end (src/hdf5io.F90:149-163)."""
        if getattr(self, "_h", None):
            h, self._h = self._h, None
            rc = self.L.astr_h5io_end(h)
            if rc != 0:
                raise AstrError(rc, self.L.astr_h5_last_error(None).decode())

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def h5io_init(filename: str, mode: str = "read") -> H5File:
    return H5File(filename, mode)


def _read_flowfield(ctx, fn, h, filename, mode):
    ns, t = ctypes.c_int(), ctypes.c_double()
    ctx.check(fn(h, str(filename).encode(), mode.encode(), ctypes.byref(ns), ctypes.byref(t)))
    return ns.value, t.value


class TGVSolver:
    """The miniapp ``boxsolver`` on the GPU: a periodic im x jm x km box advanced by SSP-RK3 with
    the compact scheme and the compact filter (tgvsolver.F90:994-1082)."""

    def __init__(self, ctx: Context, im: int, jm: int | None = None, km: int | None = None,
                 params: FlowParams | None = None):
        self.ctx = ctx
        self.im, self.jm, self.km = im, jm or im, km or im
        p = params or FlowParams()
        self.params = p
        cp = p.c_params(self.im, self.jm, self.km)
        h = ctypes.c_void_p()
        ctx.check(ctx.L.astr_state_create(ctx._h, ctypes.byref(cp), ctypes.byref(h)))
        self._h = h

    @property
    def shape(self):
        return (self.im + 1, self.jm + 1, self.km + 1)

    def close(self):
        if getattr(self, "_h", None) and self.ctx.alive():
            self.ctx.L.astr_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_tgv(self):
        """flowfield_init (tgvsolver.F90:172-234)."""
        self.ctx.check(self.ctx.L.astr_state_init_tgv(self._h))

    def set_q(self, q, lbound=(0, 0, 0)):
        L = self.ctx.L
        if _is_torch(q):
            assert q.stride(0) == 1
            self.ctx.check(L.astr_state_upload(self._h, ctypes.c_void_p(q.data_ptr()), _i64(q.shape[:3]), _i64(lbound),
                                               ASTR_DEVICE))
        else:
            qf = np.asfortranarray(q, dtype=np.float64)
            self.ctx.check(L.astr_state_upload(self._h, ctypes.c_void_p(qf.ctypes.data), _i64(qf.shape[:3]),
                                               _i64(lbound), ASTR_HOST))

    def get_q(self) -> np.ndarray:
        out = np.zeros(self.shape + (5,), order="F")
        self.ctx.check(self.ctx.L.astr_state_download(self._h, ctypes.c_void_p(out.ctypes.data), _i64(self.shape),
                                                      _i64((0, 0, 0)), ASTR_HOST))
        return out

    def cfl_dt(self, cfl: float) -> float:
        dt = ctypes.c_double()
        self.ctx.check(self.ctx.L.astr_cfl_dt(self._h, cfl, ctypes.byref(dt)))
        return dt.value

    def rhs(self) -> np.ndarray:
        out = np.zeros(self.shape + (5,), order="F")
        self.ctx.check(self.ctx.L.astr_rhs(self._h, ctypes.c_void_p(out.ctypes.data), _i64(self.shape),
                                           _i64((0, 0, 0)), ASTR_HOST))
        return out

    def rk3(self, dt: float, nsteps: int = 1):
        self.ctx.check(self.ctx.L.astr_rk3_step(self._h, dt, nsteps))

    def write_flowfield(self, filename: str):
        """writeflfed's flow field: ro, u1, u2, u3, p, t (q2fvar of the state), nstep, time."""
        self.ctx.check(self.ctx.L.astr_state_write_flowfield(self._h, str(filename).encode()))

    def read_flowfield(self, filename: str, mode: str = "h"):
        """readcheckpoint's flow field + updateq; returns (nstep, time), which the state takes."""
        return _read_flowfield(self.ctx, self.ctx.L.astr_state_read_flowfield, self._h, filename, mode)

    def rk3_host(self, q: np.ndarray, dt: float, nsteps: int = 1) -> np.ndarray:
        """One call with the state in host memory (uploaded, advanced, downloaded in place)."""
        assert q.flags["F_CONTIGUOUS"] and q.dtype == np.float64
        diag = np.zeros(3)
        self.ctx.check(self.ctx.L.astr_rk3_step_host(self._h, ctypes.c_void_p(q.ctypes.data), _i64(q.shape[:3]),
                                                     _i64((0, 0, 0)), dt, nsteps, diag.ctypes.data_as(_lib._dp)))
        return diag

    def history(self) -> np.ndarray:
        """stacal rows (nstep, time, tke, enstrophy, dissipation)."""
        n = ctypes.c_int()
        self.ctx.check(self.ctx.L.astr_history(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1) * 5)
        self.ctx.check(self.ctx.L.astr_history(self._h, out.ctypes.data_as(_lib._dp), n.value, ctypes.byref(n)))
        return out[: 5 * n.value].reshape(n.value, 5)

    def diagnostics(self) -> np.ndarray:
        out = np.zeros(3)
        self.ctx.check(self.ctx.L.astr_diagnostics(self._h, out.ctypes.data_as(_lib._dp)))
        return out

    def use_graph(self, on: bool):
        self.ctx.check(self.ctx.L.astr_state_use_graph(self._h, int(on)))

    def split_filter(self, on: bool):
        """Run the filter along y owed by each stage as its own pass (True) or fused into the
        first gradient pass (False); turns autotuning off."""
        self.ctx.check(self.ctx.L.astr_state_split_filter(self._h, int(on)))

    def autotune(self, on: bool):
        """Per-pass launch-shape autotuning at the first RK3 step (default on above 100^3)."""
        self.ctx.check(self.ctx.L.astr_state_autotune(self._h, int(on)))

    def set_launch_shape(self, pass_name: str, S: int, WPL: int, TI: int, LPW: int = 1, FPS: int = 5):
        """Pin one pass's launch shape (disables autotuning)."""
        names = ["A", "B", "C", "A'", "B'", "F_C", "F_A"]
        self.ctx.check(self.ctx.L.astr_state_set_launch_shape(self._h, names.index(pass_name), S, WPL, TI, LPW, FPS))

    def launch_shapes(self) -> dict:
        """{pass: (rows per lane, warps per line, lines per CTA, tile pitch, lines per warp group,
        fields per step)}."""
        buf = (ctypes.c_int * 42)()
        self.ctx.check(self.ctx.L.astr_state_launch_shapes(self._h, buf))
        names = ["A", "B", "C", "A'", "B'", "F_C", "F_A"]
        return {nm: tuple(buf[6 * i:6 * i + 6]) for i, nm in enumerate(names)}


class FullSolver:
    """The full solver's time integration on a periodic box (``time_integration_rk`` with rk3,
    src/mainloop.F90:298-476), on the reference's array layout with stored halos: the filter before
    every stage's rhscal, qswap's averaging of nodes 0 and N with primitives recomputed on the
    boundary planes only, rhscal in its metric form, the update of q*jacob. The default Sutherland
    constant is the full solver's 110.3 (src/solver.F90:121-122)."""

    def __init__(self, ctx: Context, im: int, jm: int | None = None, km: int | None = None,
                 params: FlowParams | None = None):
        self.ctx = ctx
        self.im, self.jm, self.km = im, jm or im, km or im
        p = params or FlowParams(sutherland=110.3)
        self.params = p
        cp = p.c_params(self.im, self.jm, self.km)
        h = ctypes.c_void_p()
        ctx.check(ctx.L.astr_full_create(ctx._h, ctypes.byref(cp), ctypes.byref(h)))
        self._h = h

    @property
    def shape(self):
        return (self.im + 1, self.jm + 1, self.km + 1)

    def close(self):
        if getattr(self, "_h", None) and self.ctx.alive():
            self.ctx.L.astr_full_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_q(self, q, lbound=(0, 0, 0)):
        qf = np.asfortranarray(q, dtype=np.float64)
        self.ctx.check(self.ctx.L.astr_full_upload(self._h, ctypes.c_void_p(qf.ctypes.data), _i64(qf.shape[:3]),
                                                   _i64(lbound), ASTR_HOST))

    def get_q(self) -> np.ndarray:
        out = np.zeros(self.shape + (5,), order="F")
        self.ctx.check(self.ctx.L.astr_full_download(self._h, ctypes.c_void_p(out.ctypes.data), _i64(self.shape),
                                                     _i64((0, 0, 0)), ASTR_HOST))
        return out

    def step(self, dt: float, nsteps: int = 1):
        self.ctx.check(self.ctx.L.astr_full_step(self._h, dt, nsteps))

    def write_flowfield(self, filename: str):
        """writeflfed's flow field: the primitive arrays ro, u1, u2, u3, p, t, nstep, time."""
        self.ctx.check(self.ctx.L.astr_full_write_flowfield(self._h, str(filename).encode()))

    def read_flowfield(self, filename: str, mode: str = "h"):
        """readcheckpoint + updateq: q from the file's (ro, u, t), interior primitives as read;
        returns (nstep, time), which the solver takes."""
        return _read_flowfield(self.ctx, self.ctx.L.astr_full_read_flowfield, self._h, filename, mode)

    def rhs(self) -> np.ndarray:
        """One stage's filterq + qswap + rhscal (the state keeps the filtered, averaged q)."""
        out = np.zeros(self.shape + (5,), order="F")
        self.ctx.check(self.ctx.L.astr_full_rhs(self._h, ctypes.c_void_p(out.ctypes.data), _i64(self.shape),
                                                _i64((0, 0, 0)), ASTR_HOST))
        return out

    def history(self) -> np.ndarray:
        n = ctypes.c_int()
        self.ctx.check(self.ctx.L.astr_full_history(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1) * 5)
        self.ctx.check(self.ctx.L.astr_full_history(self._h, out.ctypes.data_as(_lib._dp), n.value, ctypes.byref(n)))
        return out[: 5 * n.value].reshape(n.value, 5)


class Ensemble:
    """Independent periodic boxes (``TGVSolver`` objects of one context, sizes may differ)
    advanced together: each pass of an RK3 stage is one launch over every box sharing a solve
    layout, and each step is one CUDA graph. Per-box results equal ``TGVSolver.rk3``."""

    def __init__(self, ctx: Context, boxes: list[TGVSolver]):
        self.ctx = ctx
        self.boxes = list(boxes)
        arr = (ctypes.c_void_p * len(self.boxes))(*[b._h.value for b in self.boxes])
        h = ctypes.c_void_p()
        ctx.check(ctx.L.astr_ensemble_create(ctx._h, arr, len(self.boxes), ctypes.byref(h)))
        self._h = h

    def step(self, dt, nsteps: int = 1):
        """``nsteps`` RK3 steps of every box; ``dt`` is one time step per box (or one for all)."""
        d = np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(self.boxes),)).copy()
        self.ctx.check(self.ctx.L.astr_ensemble_step(self._h, d.ctypes.data_as(_lib._dp), nsteps))

    def close(self):
        if getattr(self, "_h", None) and self.ctx.alive():
            self.ctx.L.astr_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
