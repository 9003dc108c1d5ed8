"""ORACLE — test infrastructure only.

ctypes binding of ``oracle/astr_oracle.cpp``, a CPU restatement of the reference ASTR
(Perrbit/astr_gpu) hot path: compact derivatives (derivative.F90), compact filter (filter.F90),
Thomas solver (commfunc.F90:752-813) and the Taylor-Green miniapp driver
(miniapps/tgv_solver_3d/tgvsolver.F90). Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg / ``--impl reference`` arm of ``bench.py`` may import this module, and only
as the checker or the timed CPU reference — never as part of the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libastr_oracle.so")
_lib = None

HM = 5  # halo width, commvar.F90:190


def build(force: bool = False) -> str:
    """Compile the oracle shared library in-tree (``make -C oracle``)."""
    src = os.path.join(_HERE, "astr_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "-s"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, dp, ip, i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), \
            ctypes.POINTER(ctypes.c_int64)
        d, i = ctypes.c_double, ctypes.c_int
        sig = {
            "orc_fd_scheme_create": (vp, [ctypes.c_char_p, i, i]),
            "orc_filter_create": (vp, [i, i, d, d, d, i]),
            "orc_scheme_free": (None, [vp]),
            "orc_scheme_info": (i, [vp, ip, ip]),
            "orc_scheme_ac": (None, [vp, dp, dp, dp]),
            "orc_deriv_line": (None, [vp, dp, dp]),
            "orc_filter_line": (None, [vp, dp, dp]),
            "orc_deriv3d": (None, [vp, i, dp, i64p, i64p, i, dp]),
            "orc_filter3d": (None, [vp, i, dp, i64p, i64p, i, dp]),
            "orc_flux_create": (vp, [i, i, i, i, d]),
            "orc_flux_line": (None, [vp, dp, dp]),
            "orc_flux3d": (None, [vp, i, dp, i64p, i64p, i, dp]),
            "orc_tgv_create": (vp, [i, i, i, d, d, d, d, d, d, d, d, d, i]),
            "orc_tgv_free": (None, [vp]),
            "orc_tgv_init_tgv": (None, [vp]),
            "orc_tgv_set_q": (None, [vp, dp]),
            "orc_tgv_get_q": (None, [vp, dp]),
            "orc_tgv_set_flowfield": (None, [vp, dp]),
            "orc_tgv_get_flowfield": (None, [vp, dp]),
            "orc_tgv_set_dt": (None, [vp, d]),
            "orc_tgv_cfl_dt": (d, [vp, d]),
            "orc_tgv_steps": (None, [vp, i]),
            "orc_tgv_steps_full": (None, [vp, i]),
            "orc_tgv_set_boundaries": (None, [vp, i, i, i, d]),
            "orc_tgv_set_convection": (i, [vp, i, d, i, d]),
            "orc_tgv_shock_flags": (i, [vp, ctypes.c_void_p]),
            "orc_chardecomp": (None, [d, d, d, d, dp, d, d, d, dp, dp, dp, dp]),
            "orc_sw_split": (None, [d, d, d, dp, d, d, dp, dp, d, dp, dp]),
            "orc_mp5": (d, [dp, d, i]),
            "orc_tgv_rhs_full": (None, [vp, dp]),
            "orc_tgv_history": (i, [vp, dp, i]),
            "orc_tgv_history_compensated": (i, [vp, dp, i]),
            "orc_tgv_rhs": (None, [vp, dp]),
            "orc_tgv_diagnostics": (None, [vp, dp]),
            "orc_num_threads": (i, []),
            "orc_set_num_threads": (None, [i]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"] or a.ndim == 1
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Scheme:
    """A ``compact_scheme`` (commtype.F90:13-23): derivative (``fd_scheme_initiate``) or filter
    (``compact_filter_initiate`` + ``filter_coefficient_cal``)."""

    def __init__(self, handle, dim, ntype, is_filter):
        self._h = handle
        self.dim = dim
        self.ntype = ntype
        self.is_filter = is_filter

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_scheme_free(self._h)
            self._h = None

    def ac(self):
        L = lib()
        f, l = ctypes.c_int(), ctypes.c_int()
        n = L.orc_scheme_info(self._h, ctypes.byref(f), ctypes.byref(l))
        a1, a2, a3 = (np.zeros(n) for _ in range(3))
        L.orc_scheme_ac(self._h, _dp(a1), _dp(a2), _dp(a3))
        return f.value, l.value, a1, a2, a3

    def line(self, f: np.ndarray) -> np.ndarray:
        """f holds f(-5..dim+5); returns the dim+1 outputs (df_compact / compact_filter)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        assert f.shape == (self.dim + 1 + 2 * HM,)
        out = np.zeros(self.dim + 1)
        (lib().orc_filter_line if self.is_filter else lib().orc_deriv_line)(self._h, _dp(f), _dp(out))
        return out

    def apply3d(self, f: np.ndarray, direction: int, lbound=(0, 0, 0)) -> np.ndarray:
        """Apply along ``direction`` (0,1,2) to every line of a Fortran-ordered array
        f(l0:, l1:, l2:[, nfields]); the output spans 0..dim along that direction."""
        f = np.asfortranarray(f, dtype=np.float64)
        nf = f.shape[3] if f.ndim == 4 else 1
        shape = np.array(f.shape[:3], dtype=np.int64)
        lb = np.array(lbound, dtype=np.int64)
        oshape = list(f.shape)
        oshape[direction] = self.dim + 1
        out = np.zeros(oshape, order="F")
        fn = lib().orc_filter3d if self.is_filter else lib().orc_deriv3d
        fn(self._h, direction, _dp(f), shape.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
           lb.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), nf, _dp(out))
        return out


def fd_scheme_initiate(scheme: str, ntype: int, dim: int) -> Scheme:
    """derivative.F90:63-158."""
    h = lib().orc_fd_scheme_create(scheme.encode(), ntype, dim)
    if not h:
        raise ValueError(f"scheme not defined: {scheme}")
    return Scheme(h, dim, ntype, False)


def compact_filter_initiate(ntype: int, dim: int, alfa: float = 0.49, beta_halo: float = 1.11,
                            beta_bound: float = 0.98, boundary_no_filter: bool = False) -> Scheme:
    """filter.F90:31-100 with the coefficients of filter_coefficient_cal (filter.F90:299-432)."""
    h = lib().orc_filter_create(ntype, dim, alfa, beta_halo, beta_bound, int(boundary_no_filter))
    return Scheme(h, dim, ntype, True)


class FluxScheme(Scheme):
    """A compact interface-flux scheme (``compact_flux_initiate``, flux.F90:32-112): the
    tridiagonal '543' scheme with wind-biased interior coefficients blended by ``bfac``; its
    outputs are the interface values fh(-1..dim) of ``flux_compact`` (flux.F90:125-150)."""

    def __init__(self, handle, dim, ntype, wind, bfac):
        super().__init__(handle, dim, ntype, False)
        self.wind = wind
        self.bfac = bfac

    def line(self, f: np.ndarray) -> np.ndarray:
        """f holds f(-5..dim+5); returns the dim+2 interface values fh(-1..dim)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        assert f.shape == (self.dim + 1 + 2 * HM,)
        out = np.zeros(self.dim + 2)
        lib().orc_flux_line(self._h, _dp(f), _dp(out))
        return out

    def apply3d(self, f: np.ndarray, direction: int, lbound=(0, 0, 0)) -> np.ndarray:
        """Every line of a Fortran-ordered f(l0:, l1:, l2:[, nfields]) along ``direction``; the output
        spans -1..dim along that direction (dim+2 planes), the input's extents elsewhere."""
        f = np.asfortranarray(f, dtype=np.float64)
        nf = f.shape[3] if f.ndim == 4 else 1
        shape = np.array(f.shape[:3], dtype=np.int64)
        lb = np.array(lbound, dtype=np.int64)
        oshape = list(f.shape)
        oshape[direction] = self.dim + 2
        out = np.zeros(oshape, order="F")
        lib().orc_flux3d(self._h, direction, _dp(f), shape.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                         lb.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), nf, _dp(out))
        return out


def compact_flux_initiate(ntype: int, dim: int, wind: str = "+", bfac: float = 0.0, scheme: int = 543) -> FluxScheme:
    """flux.F90:32-112; ``wind`` is '+' (upwind-biased) or '-' (downwind-biased)."""
    w = {"+": 1, "-": -1}[wind]
    h = lib().orc_flux_create(scheme, ntype, dim, w, bfac)
    if not h:
        raise ValueError(f"flux scheme not defined: {scheme}, ntype {ntype}")
    return FluxScheme(h, dim, ntype, w, bfac)


def chardecomp(gamma, left, right, ddi):
    """chardecomp (solver.F90:1959-2163): left/right = (rho, p, rhoE, (u, v, w)); returns (R, L)."""
    R, L = np.zeros(25), np.zeros(25)
    arr = lambda v: np.ascontiguousarray(v, dtype=np.float64)
    vl, vr, dd = arr(left[3]), arr(right[3]), arr(ddi)
    lib().orc_chardecomp(gamma, left[0], left[1], left[2], _dp(vl), right[0], right[1], right[2], _dp(vr), _dp(dd),
                         _dp(R), _dp(L))
    return R.reshape(5, 5), L.reshape(5, 5)


def sw_split(gamma, mach, rho, u, p, metric, jacob=1.0):
    """flux_steger_warming (riemann.F90:23-161) of one node: returns (f+, f-)."""
    arr = lambda v: np.ascontiguousarray(v, dtype=np.float64)
    u = arr(u)
    t = p / rho * gamma * mach ** 2
    qq = arr([rho, rho * u[0], rho * u[1], rho * u[2], p / (gamma - 1) + 0.5 * rho * (u @ u)])
    fp, fm = np.zeros(5), np.zeros(5)
    m = arr(metric)
    lib().orc_sw_split(gamma, mach, rho, _dp(u), p, t, _dp(qq), _dp(m), jacob, _dp(fp), _dp(fm))
    return fp, fm


def mp5(u, ul, discont=True):
    """MP5 (flux.F90:434-496) of the stencil u[0..4] with the linear value ul."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    return lib().orc_mp5(_dp(u), float(ul), int(discont))


@dataclass
class FlowParams:
    mach: float = 0.1
    reynolds: float = 1600.0
    prandtl: float = 0.72
    gamma: float = 1.4
    ref_tem: float = 273.15
    sutherland: float = 110.4     # tgvsolver.F90:133 (the full solver uses 110.3)
    alfa_filter: float = 0.49
    beta_halo: float = 1.11
    beta_bound: float = 1.09      # tgvsolver.F90:253
    filter_on: bool = True
    ntype: tuple = (3, 3, 3)      # per direction: 3 periodic; 1, 2, 4 physical ends (full-solver mode)
    twall: float = 1.0            # isothermal no-slip walls at the physical ends (bctype 41)
    conschm: int = 643            # full-solver convection: 643 central compact, 543 upwind compact flux
    bfacmpld: float = 0.0         # b factor of the upwind compact flux (bfacmpld of the input)
    lchardecomp: bool = False     # upwind flux in characteristic variables, with the Ducros sensor
    shkcrt: float = 0.01          # the Ducros sensor's threshold


def thermo_constants(mach: float, gamma: float):
    """const1, const2, const6 of a nondimensional run (tgvsolver.F90:189-195)."""
    return 1.0 / (gamma * (gamma - 1.0) * (mach * mach)), gamma * (mach * mach), 1.0 / (gamma - 1.0)


def q2fvar(q: np.ndarray, mach: float, gamma: float) -> np.ndarray:
    """q2fvar_3da (src/fludyna.F90:545-634) with thermal_3d (:136-153): (ro, u1, u2, u3, p, t)
    from q(..., 0:5), every operation in the reference's order (numpy rounds each one)."""
    _c1, c2, c6 = thermo_constants(mach, gamma)
    r = q[..., 0]
    u, v, w = q[..., 1] / r, q[..., 2] / r, q[..., 3] / r
    p = (q[..., 4] - 0.5 * r * (u * u + v * v + w * w)) / c6
    return np.stack([r, u, v, w, p, p / r * c2], axis=-1)


def fvar2q_temperature(f: np.ndarray, mach: float, gamma: float) -> np.ndarray:
    """fvar2q_3da's temperature branch (src/fludyna.F90:449-533), which updateq takes after
    readcheckpoint (src/fludyna.F90:254-300): q from (ro, u1, u2, u3, p, t) = f(..., 0:6)."""
    c1, _c2, _c6 = thermo_constants(mach, gamma)
    r, u, v, w, t = f[..., 0], f[..., 1], f[..., 2], f[..., 3], f[..., 5]
    return np.stack([r, r * u, r * v, r * w, r * (t * c1 + 0.5 * (u * u + v * v + w * w))], axis=-1)


class TGVOracle:
    """The miniapp ``boxsolver`` (tgvsolver.F90:1086-1116) on an im x jm x km periodic box."""

    def __init__(self, im: int, jm: int | None = None, km: int | None = None, params: FlowParams | None = None):
        self.im, self.jm, self.km = im, jm or im, km or im
        p = params or FlowParams()
        self.params = p
        self._h = lib().orc_tgv_create(self.im, self.jm, self.km, p.mach, p.reynolds, p.prandtl, p.gamma,
                                       p.ref_tem, p.sutherland, p.alfa_filter, p.beta_halo, p.beta_bound,
                                       int(p.filter_on))
        if tuple(p.ntype) != (3, 3, 3):
            lib().orc_tgv_set_boundaries(self._h, *[int(t) for t in p.ntype], float(p.twall))
        if p.conschm != 643:
            if lib().orc_tgv_set_convection(self._h, int(p.conschm), float(p.bfacmpld), int(p.lchardecomp),
                                            float(p.shkcrt)) != 0:
                raise ValueError(f"convection scheme not defined: {p.conschm}")

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_tgv_free(self._h)
            self._h = None

    @property
    def shape(self):
        return (self.im + 1, self.jm + 1, self.km + 1)

    def init_tgv(self):
        lib().orc_tgv_init_tgv(self._h)

    def set_q(self, q: np.ndarray):
        q = np.asfortranarray(q, dtype=np.float64)
        assert q.shape == self.shape + (5,)
        lib().orc_tgv_set_q(self._h, _dp(q))

    def get_q(self) -> np.ndarray:
        out = np.zeros(self.shape + (5,), order="F")
        lib().orc_tgv_get_q(self._h, _dp(out))
        return out

    def set_dt(self, dt: float):
        lib().orc_tgv_set_dt(self._h, dt)

    def set_flowfield(self, prims: np.ndarray):
        """readcheckpoint + updateq: the primitive arrays take the file's (ro, u1, u2, u3, p, t),
        prims[..., 0:6] on nodes 0..N, and q = fvar2q(ro, u, t) (src/fludyna.F90:449-533)."""
        f = np.asfortranarray(prims, dtype=np.float64)
        assert f.shape == self.shape + (6,)
        lib().orc_tgv_set_flowfield(self._h, _dp(f))

    def get_flowfield(self) -> np.ndarray:
        """The primitive arrays (ro, u1, u2, u3, p, t) on nodes 0..N, as writeflfed writes them."""
        out = np.zeros(self.shape + (6,), order="F")
        lib().orc_tgv_get_flowfield(self._h, _dp(out))
        return out

    def cfl_dt(self, cfl: float) -> float:
        return lib().orc_tgv_cfl_dt(self._h, cfl)

    def steps(self, n: int):
        lib().orc_tgv_steps(self._h, n)

    def steps_full(self, n: int):
        """n steps of the full solver's time_integration_rk (src/mainloop.F90:392-476) on this
        periodic box: filterq before rhscal at every stage, qswap's averaging of nodes 0 and N,
        interior primitives of the unfiltered state, the metric form of rhscal, q*jacob update."""
        lib().orc_tgv_steps_full(self._h, n)

    def rhs_full(self) -> np.ndarray:
        """One full-solver stage's qrhs (after its filterq and qswap, which change the state's q)."""
        out = np.zeros(self.shape + (5,), order="F")
        lib().orc_tgv_rhs_full(self._h, _dp(out))
        return out

    def shock_flags(self) -> np.ndarray:
        """The Ducros sensor's shock flags of the last full-solver rhscal (characteristic mode)."""
        out = np.zeros(self.shape, dtype=np.uint8, order="F")
        if lib().orc_tgv_shock_flags(self._h, out.ctypes.data) != 0:
            raise ValueError("no shock flags: the characteristic decomposition is off")
        return out.astype(bool)
    def history(self, compensated: bool = False) -> np.ndarray:
        """Rows of (nstep, time, tke, enstrophy, dissipation), one per step (stacal). The sums run
        over the nodes in the reference's sequential order; with ``compensated`` the same per-node
        terms are summed with Neumaier's compensation instead (rounding independent of the node
        count, the reference value for sums taken in another order)."""
        L = lib()
        fn = L.orc_tgv_history_compensated if compensated else L.orc_tgv_history
        n = fn(self._h, _dp(np.zeros(5)), 0)
        out = np.zeros(5 * max(n, 1))
        fn(self._h, _dp(out), n)
        return out[: 5 * n].reshape(n, 5)

    def rhs(self) -> np.ndarray:
        out = np.zeros(self.shape + (5,), order="F")
        lib().orc_tgv_rhs(self._h, _dp(out))
        return out

    def diagnostics(self) -> np.ndarray:
        out = np.zeros(3)
        lib().orc_tgv_diagnostics(self._h, _dp(out))
        return out


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int):
    lib().orc_set_num_threads(n)
