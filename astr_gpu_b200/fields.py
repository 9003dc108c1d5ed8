"""Initial fields and box sets for the periodic solver (host side, numpy).

* ``tgv_q`` -- the Taylor-Green state of the miniapp's ``flowfield_init``
  (miniapps/tgv_solver_3d/tgvsolver.F90:172-234), for boxes that do not use the device initialiser.
* ``solenoidal_q`` -- a random divergence-free velocity whose shell spectrum follows the
  reference's ``IniEnergDis`` (src/pp.F90:2849-2859), E(k) = A k^4 exp(-2 (k/k0)^2) with k0 = 4
  (src/pp.F90:2656), on uniform density and pressure. Phases come from a seeded numpy generator,
  not from the reference's Fortran ``random_number`` stream, so fields match the reference's
  statistics, not its samples.
* ``ensemble_specs`` -- the seeded set of uneven boxes (sizes, Mach, Reynolds, initial kind) of a
  batched ensemble run.
* ``spectral_field`` / ``gradient_input`` -- the scalar test field of the gradient-kernel workload
  (the reference's ``gradtest`` grid, src/test.F90:440-650: x and z periodic on [0, 2 pi), y
  non-periodic on [0, 2]): a seeded sum of Fourier modes 0 < |k| <= 16 with amplitudes |k|^(-5/3),
  and the halo-extended array the line operators read.

Arrays are (im+1, jm+1, km+1, 5) Fortran-ordered conserved variables (rho, rho u, rho v, rho w,
rho E) on nodes 0..N with node N equal to node 0, the layout ``TGVSolver.set_q`` takes.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["tgv_q", "solenoidal_velocity", "solenoidal_q", "BoxSpec", "ensemble_specs", "spectral_field",
           "gradient_input", "write_field", "read_field"]


def _conserved(rho, u, v, w, p, gamma):
    q = np.empty(rho.shape + (5,), order="F")
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 3] = rho * w
    q[..., 4] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return q


def _periodic_nodes(f):
    """N^3 samples on nodes 0..N-1 -> (N+1)^3 with the periodic image at node N."""
    return np.pad(f, [(0, 1)] * 3, mode="wrap")


def tgv_q(n: int, mach: float, gamma: float = 1.4) -> np.ndarray:
    """flowfield_init of the miniapp: rho = 1, u = sin x cos y cos z, v = -cos x sin y cos z, w = 0,
    p = 1/(gamma M^2) + (cos 2x + cos 2y)(cos 2z + 2)/16 on x_i = 2 pi i / n."""
    x = 2.0 * np.pi * np.arange(n + 1) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    p = 1.0 / (gamma * mach * mach) + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    return _conserved(np.ones_like(u), u, v, w, p, gamma)


U_RMS = 1.0 / np.sqrt(3.0)   # <|u|^2> = 1: the box's Mach number is its turbulent Mach number


def solenoidal_velocity(n: int, seed: int, k0: float = 4.0, urms: float = U_RMS):
    """Random divergence-free (u, v, w) on an n^3 periodic grid with shell spectrum
    E(k) ~ k^4 exp(-2 (k/k0)^2), scaled to <|u|^2>/3 = urms^2. Returns three (n, n, n) arrays.
    The default makes <|u|^2> = 1, so with p = 1/(gamma M^2) the turbulent Mach number
    sqrt(<|u|^2>)/c equals M (at M = 0.5 with u_rms = 1 the boxes form shocks the central scheme
    does not survive).

    Each Fourier mode gets a complex Gaussian amplitude, is projected onto the plane normal to its
    wavevector (which makes the spectral divergence zero) and rescaled so that the energy of the
    shell |k| in [k-1/2, k+1/2) equals E(k)."""
    rng = np.random.default_rng(seed)
    k1 = np.fft.fftfreq(n, 1.0 / n)
    kz = np.fft.rfftfreq(n, 1.0 / n)
    KX, KY, KZ = np.meshgrid(k1, k1, kz, indexing="ij")
    kk = np.sqrt(KX * KX + KY * KY + KZ * KZ)
    shape = KX.shape
    uh = [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in range(3)]
    with np.errstate(invalid="ignore", divide="ignore"):
        kdotu = (KX * uh[0] + KY * uh[1] + KZ * uh[2]) / np.where(kk > 0, kk * kk, 1.0)
    uh = [uh[0] - KX * kdotu, uh[1] - KY * kdotu, uh[2] - KZ * kdotu]
    for c in range(3):
        uh[c][kk == 0] = 0.0
        # the Nyquist planes have no partner mode: drop them so the real field is exact
        uh[c][np.abs(KX) == n // 2] = 0.0
        uh[c][np.abs(KY) == n // 2] = 0.0
        uh[c][KZ == n // 2] = 0.0
    # rfft half-space weights: modes with 0 < kz < n/2 stand for themselves and their conjugates
    wgt = np.where((KZ > 0) & (KZ < n / 2), 2.0, 1.0)
    e_mode = 0.5 * wgt * sum(np.abs(c) ** 2 for c in uh)
    shell = np.rint(kk).astype(np.int64)
    nshell = int(shell.max()) + 1
    e_have = np.bincount(shell.ravel(), weights=e_mode.ravel(), minlength=nshell)
    ks = np.arange(nshell, dtype=np.float64)
    e_want = ks ** 4 * np.exp(-2.0 * (ks / k0) ** 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        scale = np.where(e_have > 0, np.sqrt(e_want / np.where(e_have > 0, e_have, 1.0)), 0.0)
    fac = scale[shell]
    vel = [np.fft.irfftn(c * fac, s=(n, n, n), axes=(0, 1, 2)) for c in uh]
    r = np.sqrt(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2) / 3.0)
    return [v * (urms / r) for v in vel]


def solenoidal_q(n: int, mach: float, seed: int, gamma: float = 1.4, k0: float = 4.0, urms: float = U_RMS):
    """Uniform rho = 1 and p = 1/(gamma M^2) with the random solenoidal velocity above."""
    u, v, w = (_periodic_nodes(c) for c in solenoidal_velocity(n, seed, k0, urms))
    rho = np.ones_like(u)
    p = np.full_like(u, 1.0 / (gamma * mach * mach))
    return _conserved(rho, u, v, w, p, gamma)


@dataclass(frozen=True)
class BoxSpec:
    n: int              # nodes 0..n per axis, periodic
    mach: float
    reynolds: float
    kind: str           # "tgv" or "solenoidal"
    seed: int           # phase seed of a solenoidal box


def ensemble_specs(nbox: int = 48, seed: int = 48, sizes=(32, 48, 64, 96, 128), mach=(0.1, 0.5),
                   reynolds=(400.0, 3200.0)) -> list[BoxSpec]:
    """Seeded uneven box set: size uniform over ``sizes``, Mach and Reynolds uniform in their
    ranges; the first half Taylor-Green, the second half random solenoidal."""
    rng = np.random.default_rng(seed)
    ns = rng.choice(np.asarray(sizes), size=nbox)
    ms = rng.uniform(mach[0], mach[1], size=nbox)
    rs = rng.uniform(reynolds[0], reynolds[1], size=nbox)
    return [BoxSpec(int(ns[b]), float(ms[b]), float(rs[b]), "tgv" if b < nbox // 2 else "solenoidal",
                    int(seed * 1000 + b)) for b in range(nbox)]


SPECTRAL_SEED = 20251203
HM = 5   # halo width of the reference's arrays (commvar.F90:190)


def spectral_field(im: int, jm: int | None = None, km: int | None = None, kmax: int = 16,
                   seed: int = SPECTRAL_SEED) -> np.ndarray:
    """f(x, y, z) = sum over integer wavevectors 0 < |k| <= kmax of |k|^(-5/3) cos(k_x x + (pi/2) k_y y
    + k_z z + phi_k) on nodes x_i = 2 pi i/im, y_j = 2 j/jm, z_k = 2 pi k/km (i = 0..im etc.), the
    phases phi_k uniform on [0, 2 pi) from numpy's PCG64 seeded with `seed`, drawn in lexicographic
    order of (k_x, k_y, k_z) from -kmax to kmax. Returns an (im+1, jm+1, km+1) Fortran-ordered
    array. The mode sum is evaluated axis by axis (a separable complex contraction)."""
    jm = jm or im
    km = km or im
    r = np.arange(-kmax, kmax + 1)
    KX, KY, KZ = np.meshgrid(r, r, r, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    keep = (k2 > 0) & (k2 <= kmax * kmax)
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0.0, 2.0 * np.pi, size=int(keep.sum()))
    coef = np.zeros(KX.shape, dtype=np.complex128)
    coef[keep] = np.power(np.sqrt(k2[keep].astype(np.float64)), -5.0 / 3.0) * np.exp(1j * phi)
    x = 2.0 * np.pi * np.arange(im + 1) / im
    y = 2.0 * np.arange(jm + 1) / jm
    z = 2.0 * np.pi * np.arange(km + 1) / km
    ex = np.exp(1j * np.outer(r, x))                  # (nk, im+1)
    ey = np.exp(1j * np.outer(r, 0.5 * np.pi * y))    # (nk, jm+1)
    ez = np.exp(1j * np.outer(r, z))                  # (nk, km+1)
    a1 = np.tensordot(coef, ez, axes=([2], [0]))      # (kx, ky, z)
    a2 = np.einsum("abk,bj->ajk", a1, ey)             # (kx, y, z)
    f = np.tensordot(ex.T, a2, axes=([1], [0]))       # (x, y, z)
    return np.asfortranarray(f.real)


def gradient_input(f: np.ndarray, periodic=(True, False, True)) -> tuple[np.ndarray, tuple]:
    """The array the line operators read: f on nodes 0..N of each axis, extended by the
    reference's periodic halo copy f(-k) = f(N-k), f(N+k) = f(k), k = 1..5, along the periodic
    axes (dataswap of gradtest). Returns the Fortran-ordered array and its lower bounds."""
    pads = [(HM, HM) if p else (0, 0) for p in periodic]
    g = f
    for ax, p in enumerate(periodic):
        if not p:
            continue
        n = f.shape[ax] - 1
        lo = np.take(g, np.arange(n - HM, n), axis=ax)
        hi = np.take(g, np.arange(1, HM + 1), axis=ax)
        g = np.concatenate([lo, g, hi], axis=ax)
    return np.asfortranarray(g), tuple(-a for a, _ in pads)


def write_field(path: str, f: np.ndarray) -> None:
    """Raw little-endian float64 in Fortran order, preceded by the three extents as int64."""
    with open(path, "wb") as fh:
        np.asarray(f.shape[:3], dtype="<i8").tofile(fh)
        np.asfortranarray(f, dtype="<f8").ravel(order="F").tofile(fh)


def read_field(path: str) -> np.ndarray:
    with open(path, "rb") as fh:
        shape = tuple(int(v) for v in np.fromfile(fh, dtype="<i8", count=3))
        data = np.fromfile(fh, dtype="<f8")
    return data.reshape(shape, order="F")
