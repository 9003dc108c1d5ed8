"""Oracle self-checks that mirror the reference's own test drivers (src/test.F90): order of
accuracy of the compact derivative with periodic and non-periodic closures (gradtest,
test.F90:440-650), filter transfer properties (filtertest, :272-415), and the Thomas tables
(commfunc.F90:752-774)."""
import numpy as np
import pytest

import oracle

HM = oracle.HM


def _periodic_line(fn, n):
    x = 2 * np.pi * np.arange(-HM, n + HM + 1) / n
    return x, fn(x)


@pytest.mark.parametrize("n", [32, 64])
def test_deriv_periodic_accuracy(n):
    s = oracle.fd_scheme_initiate("643c", 3, n)
    x, f = _periodic_line(np.sin, n)
    dx = 2 * np.pi / n
    df = s.line(f) / dx
    err = np.abs(df - np.cos(x[HM:n + HM + 1])).max()
    assert err < 5e-7 * (64 / n) ** 6


def test_deriv_order_nonperiodic():
    # ntype 4 on [0, 2] (gradtest's y direction): sin(pi y / 2); closures are 3rd/4th order
    errs = []
    for n in (32, 64, 128):
        s = oracle.fd_scheme_initiate("643c", 4, n)
        y = 2.0 * np.arange(-HM, n + HM + 1) / n
        f = np.sin(0.5 * np.pi * y)
        dy = 2.0 / n
        df = s.line(f) / dy
        errs.append(np.abs(df - 0.5 * np.pi * np.cos(0.5 * np.pi * y[HM:n + HM + 1])).max())
    order = np.log2(errs[0] / errs[1]), np.log2(errs[1] / errs[2])
    assert min(order) > 2.5, (errs, order)


def test_explicit_matches_diff6ec_periodic():
    n = 48
    s = oracle.fd_scheme_initiate("643e", 3, n)
    x, f = _periodic_line(np.sin, n)
    df = s.line(f)
    i = np.arange(n + 1) + HM
    ref = 0.75 * (f[i + 1] - f[i - 1]) - 0.15 * (f[i + 2] - f[i - 2]) + (1 / 60) * (f[i + 3] - f[i - 3])
    np.testing.assert_array_equal(df, ref)


def test_filter_preserves_smooth_and_kills_nyquist():
    n = 64
    s = oracle.compact_filter_initiate(3, n, 0.49, 1.11, 1.09)
    x, f = _periodic_line(lambda x: np.sin(3 * x), n)
    ff = s.line(f)
    assert np.abs(ff - f[HM:n + HM + 1]).max() < 1e-9
    k = np.arange(-HM, n + HM + 1)
    nyq = np.cos(np.pi * k)          # (-1)^k, periodic for even n
    fn = s.line(nyq)
    # interior transfer function at the Nyquist wavenumber is exactly zero
    assert np.abs(fn[10:n - 10]).max() < 1e-10


def test_filter_boundary_reset_ntype4():
    n = 40
    s = oracle.compact_filter_initiate(4, n, 0.49, 1.11, 0.98)
    rng = np.random.default_rng(1)
    f = rng.standard_normal(n + 1 + 2 * HM)
    ff = s.line(f)
    assert ff[0] == f[HM] and ff[n] == f[HM + n]


def _thomas_factor(a, c):
    n = len(a)
    ac = np.zeros((3, n))
    ac[0, 0] = c[0]
    for i in range(1, n):
        ac[0, i] = c[i] / (1 - a[i] * ac[0, i - 1])
        ac[1, i] = 1 / (1 - a[i] * ac[0, i - 1])
        ac[2, i] = a[i] / (1 - a[i] * ac[0, i - 1])
    return ac


def test_thomas_tables_deriv_and_filter():
    n = 32
    f0, l0, a1, a2, a3 = oracle.fd_scheme_initiate("643c", 3, n).ac()
    assert (f0, l0) == (-1, n + 1)
    a = np.full(n + 3, 1 / 3)
    a[0] = a[-1] = 0
    ac = _thomas_factor(a, a)
    np.testing.assert_array_equal(a1, ac[0])
    np.testing.assert_array_equal(a2[1:], ac[1, 1:])
    np.testing.assert_array_equal(a3[1:], ac[2, 1:])
    f0, l0, a1, a2, a3 = oracle.compact_filter_initiate(3, n, 0.49).ac()
    assert (f0, l0) == (-3, n + 3)
    a = np.full(n + 7, 0.49)
    a[0] = a[-1] = 1.11
    ac = _thomas_factor(a, a)
    np.testing.assert_array_equal(a1, ac[0])


def test_oracle_3d_matches_lines():
    n = 24
    s = oracle.fd_scheme_initiate("643c", 3, n)
    rng = np.random.default_rng(2)
    f = np.asfortranarray(rng.standard_normal((n + 1 + 2 * HM, 5, 4)))
    out = s.apply3d(f, 0, lbound=(-HM, 0, 0))
    for j in range(5):
        for k in range(4):
            np.testing.assert_array_equal(out[:, j, k], s.line(f[:, j, k]))
