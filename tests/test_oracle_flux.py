"""The oracle's compact interface flux (compact_flux_initiate / flux_compact, flux.F90:32-256)
against an independent numpy restatement that assembles the same tridiagonal system densely
(row i: a_i x_{i-1} + x_i + c_i x_{i+1} = d_i, the convention of tridiagonal_thomas_proprocess,
commfunc.F90:752-813) and solves it with LAPACK; plus the scheme's own accuracy properties.

The reference carries no golden vectors for this path; its flux test (test.F90:675-870) prints
an L2 error only, so the pin here is the second restatement and the order of accuracy."""
import numpy as np
import pytest

import oracle

HM = 5


def _dense_flux(f, ntype, dim, wind, b):
    """fh(-1..dim) of one line, f = f(-5..dim+5)."""
    F = lambda j: f[j + HM]
    i0 = -1 if ntype in (1, 4) else -2
    im = dim if ntype in (2, 4) else dim + 1
    n = im - i0 + 1
    if wind == "+":
        a = np.full(n, 0.5 - b / 6.0)
        c = np.full(n, 1.0 / 6.0 + b / 6.0)
    else:
        a = np.full(n, 1.0 / 6.0 + b / 6.0)
        c = np.full(n, 0.5 - b / 6.0)
    a[0] = c[0] = a[-1] = c[-1] = 0.0
    if ntype in (1, 4):
        a[0] = c[0] = 2.0
        a[1] = c[1] = 0.25
    if ntype in (2, 4):
        a[-1] = c[-1] = 2.0
        a[-2] = c[-2] = 0.25
    d = np.zeros(n)

    def central(j):
        return 37 / 60 * (F(j) + F(j + 1)) - 2 / 15 * (F(j - 1) + F(j + 2)) + 1 / 60 * (F(j - 2) + F(j + 3))

    for r in range(n):
        j = i0 + r
        if wind == "+":
            d[r] = (1 / 18 - b / 36) * F(j - 1) + (19 / 18 - 9 * b / 36) * F(j) + (5 / 9 + 9 * b / 36) * F(j + 1) \
                + b / 36 * F(j + 2)
        else:
            d[r] = (1 / 18 - b / 36) * F(j + 2) + (19 / 18 - 9 * b / 36) * F(j + 1) + (5 / 9 + 9 * b / 36) * F(j) \
                + b / 36 * F(j - 1)
    if ntype in (1, 4):
        d[0] = 2.5 * F(i0 + 1) + 0.5 * F(i0 + 2)
        d[1] = 0.75 * F(i0 + 1) + 0.75 * F(i0 + 2)
    else:
        d[0] = central(i0)
    if ntype in (2, 4):
        d[-2] = 0.75 * F(im) + 0.75 * F(im - 1)
        d[-1] = 2.5 * F(im) + 0.5 * F(im - 1)
    else:
        d[-1] = central(im)
    A = np.eye(n)
    for r in range(n):
        if r > 0:
            A[r, r - 1] = a[r]
        if r < n - 1:
            A[r, r + 1] = c[r]
    x = np.linalg.solve(A, d)
    return x[-1 - i0: -1 - i0 + dim + 2]


@pytest.mark.parametrize("ntype", [1, 2, 3, 4])
@pytest.mark.parametrize("wind", ["+", "-"])
@pytest.mark.parametrize("bfac", [0.0, 1.0, 0.37])
def test_oracle_flux_matches_dense_restatement(ntype, wind, bfac):
    dim = 40
    rng = np.random.default_rng(100 * ntype + int(10 * bfac) + (wind == "-"))
    f = rng.standard_normal(dim + 1 + 2 * HM)
    s = oracle.compact_flux_initiate(ntype, dim, wind, bfac)
    got = s.line(f)
    ref = _dense_flux(f, ntype, dim, wind, bfac)
    assert got.shape == (dim + 2,)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


def test_oracle_flux_rejects_other_schemes():
    with pytest.raises(ValueError):
        oracle.compact_flux_initiate(3, 32, "+", 0.0, scheme=553)


@pytest.mark.parametrize("wind", ["+", "-"])
def test_oracle_flux_periodic_is_exact_on_cubic_cell_averages(wind):
    """Interface values reconstructed from cell averages: a periodic line of cubic cell averages
    gives the cubic's interface values to rounding (the interior scheme is 5th order)."""
    dim = 48
    s = oracle.compact_flux_initiate(3, dim, wind, 1.0)
    t = np.arange(-HM, dim + HM + 1, dtype=float)
    c = (1.0, 0.3, 0.01, 5e-4)
    f = c[0] + c[1] * t + c[2] * (t * t + 1 / 12) + c[3] * (t ** 3 + t / 4)
    xi = np.arange(-1, dim + 1) + 0.5
    ex = c[0] + c[1] * xi + c[2] * xi ** 2 + c[3] * xi ** 3
    assert np.abs(s.line(f) - ex).max() <= 1e-12


@pytest.mark.parametrize("bfac,order", [(0.0, 5), (1.0, 6)])
def test_oracle_flux_difference_converges(bfac, order):
    """The conservative finite-difference derivative (fh(i) - fh(i-1))/dx of sin on a periodic
    line (point values in, as in the reference's flux test) converges in the middle of the line
    at 5th order for b = 0 (the upwind compact scheme) and 6th order for b = 1 (the MP-LD blend),
    for both winds."""
    errs = []
    for n in (64, 128):
        dx = 2 * np.pi / n
        x = dx * np.arange(-HM, n + HM + 1)
        f = np.sin(x)
        e = 0.0
        for wind in "+-":
            fh = oracle.compact_flux_initiate(3, n, wind, bfac).line(f)
            d = (fh[1:] - fh[:-1]) / dx
            e = max(e, np.abs(d - np.cos(x[HM:HM + n + 1]))[n // 4: 3 * n // 4].max())
        errs.append(e)
    assert errs[0] / errs[1] > 2 ** (order - 0.2)


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_oracle_chardecomp_eigenvectors(direction):
    """chardecomp's Roe-averaged eigenvectors (solver.F90:1959-2163): L is the inverse of R, and
    L A R is diagonal with the eigenvalues (ugp - c, ugp, ugp, ugp, ugp + c) of the Roe-averaged
    flux Jacobian A along the metric direction, for each branch of the metric test."""
    g = 1.4
    rng = np.random.default_rng(direction)
    def state():
        rho = 1.0 + 0.2 * rng.random()
        u = rng.standard_normal(3) * 0.3
        p = 1.0 / (g * 0.2 ** 2) * (1.0 + 0.1 * rng.random())
        return rho, p, p / (g - 1) + 0.5 * rho * (u @ u), u
    left, right = state(), state()
    ddi = np.zeros(3)
    ddi[direction] = 7.5
    R, L = oracle.chardecomp(g, left, right, ddi)
    assert np.abs(L @ R - np.eye(5)).max() < 1e-12
    # the Roe-averaged Jacobian of the flux along n = ddi/|ddi|, in conserved variables
    wl = np.sqrt(left[0]) / (np.sqrt(left[0]) + np.sqrt(right[0]))
    u = wl * left[3] + (1 - wl) * right[3]
    H = wl * (left[2] + left[1]) / left[0] + (1 - wl) * (right[2] + right[1]) / right[0]
    n = ddi / np.linalg.norm(ddi)
    un, k = u @ n, 0.5 * (u @ u)
    c = np.sqrt((g - 1) * (H - k))
    A = np.zeros((5, 5))
    A[0, 1:4] = n
    A[1:4, 0] = (g - 1) * k * n - u * un
    A[1:4, 1:4] = np.outer(u, n) - (g - 1) * np.outer(n, u) + un * np.eye(3)
    A[1:4, 4] = (g - 1) * n
    A[4, 0] = ((g - 1) * k - H) * un
    A[4, 1:4] = H * n - (g - 1) * u * un
    A[4, 4] = g * un
    D = L @ A @ R
    lam = np.array([un - c, un, un, un, un + c])
    assert np.abs(D - np.diag(lam)).max() < 1e-10 * np.abs(lam).max()


@pytest.mark.parametrize("direction", [0, 1, 2])
def test_oracle_steger_warming_split_sums_to_the_flux(direction):
    """flux_steger_warming (riemann.F90:23-161): f+ + f- is the Euler flux jacob*(q uu + dxi p e,
    (E + p) uu) at subsonic and supersonic nodes, the supersonic branches put all of it on one
    side, and f+ (f-) carries only non-negative (non-positive) eigenvalue weights: the mass
    flux f+_1 >= 0 >= f-_1."""
    g, mach, jb = 1.4, 0.3, 0.7
    rng = np.random.default_rng(7 + direction)
    metric = np.zeros(3)
    metric[direction] = 4.0
    for speed in (0.2, 0.9, 2.5, -2.5):   # |u| / c: subsonic, near sonic, supersonic both ways
        rho = 1.0 + 0.3 * rng.random()
        p = 1.0 / (g * mach ** 2) * (1.0 + 0.2 * rng.random())
        c = np.sqrt(g * p / rho)
        u = 0.1 * c * rng.standard_normal(3)
        u[direction] = speed * c
        fp, fm = oracle.sw_split(g, mach, rho, u, p, metric, jb)
        uu = metric[direction] * u[direction]
        E = p / (g - 1) + 0.5 * rho * (u @ u)
        F = jb * np.array([rho * uu, rho * u[0] * uu, rho * u[1] * uu, rho * u[2] * uu, (E + p) * uu])
        F[1 + direction] += jb * metric[direction] * p
        assert np.abs(fp + fm - F).max() <= 1e-13 * np.abs(F).max() + 1e-13 * np.abs(fp).max()
        if speed >= 1:
            assert np.all(fm == 0.0)
        elif speed <= -1:
            assert np.all(fp == 0.0)
        assert fp[0] >= 0.0 >= fm[0]


def test_oracle_mp5_limiter_properties():
    """MP5 (flux.F90:434-496) with a linear value ul: without the shock flag it returns ul; on
    smooth monotone data ul inside the monotonicity bounds passes unchanged; an overshooting ul
    next to a jump is pulled back to the bound u_MP = u3 + minmod(u4 - u3, 4 (u3 - u2))."""
    u = np.array([1.0, 1.0, 1.0, 0.0, 0.0])
    assert oracle.mp5(u, 1.7, discont=False) == 1.7
    # smooth monotone stencil, ul from the 5th-order upwind formula: unchanged
    x = np.arange(5) * 0.1
    us = np.sin(x)
    ul = (2 * us[0] - 13 * us[1] + 47 * us[2] + 27 * us[3] - 3 * us[4]) / 60
    assert oracle.mp5(us, ul) == ul
    # a step: an overshoot beyond u3 is clipped into [min, max] of the local data
    ustep = np.array([0.0, 0.0, 0.0, 1.0, 1.0])
    lim = oracle.mp5(ustep, 1.3)
    assert 0.0 <= lim <= 1.0
    lim = oracle.mp5(ustep, -0.2)
    assert 0.0 <= lim <= 1.0
