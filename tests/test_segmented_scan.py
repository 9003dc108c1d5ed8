"""CPU check of the segmented Thomas algorithm the kernels use (ops.cuh seg_solve_n): lanes of
S rows, per-lane recurrences from a zero carry, Hillis-Steele warp scans of the affine carry
maps with precomputed composite multipliers, cross-warp composition, and the pf/qb fix-ups.
Restated in numpy lane by lane and compared with the reference's sequential Thomas sweep
(commfunc.F90:790-813) on the oracle's ac tables, for every compiled (S, WPL) layout."""
import numpy as np
import pytest

import oracle


def _tables(a1, a2, a3, S, WPL):
    nseg = 32 * WPL
    nsys = len(a1)
    e1 = np.zeros((nseg, S)); e2 = np.zeros((nseg, S)); e3 = np.zeros((nseg, S))
    for seg in range(nseg):
        for t in range(S):
            r = seg * S + t
            if r < nsys:
                e1[seg, t] = 0.0 if r == nsys - 1 else a1[r]
                e2[seg, t] = 1.0 if r == 0 else a2[r]
                e3[seg, t] = 0.0 if r == 0 else a3[r]
    pf = np.cumprod(-e3, axis=1)
    qb = np.cumprod((-e1)[:, ::-1], axis=1)[:, ::-1]
    mf, mb = pf[:, -1], qb[:, 0]
    FS = np.zeros((5, nseg)); BS = np.zeros((5, nseg)); FE = np.ones(nseg); BE = np.ones(nseg)
    MW = np.zeros(WPL); MWB = np.zeros(WPL)
    for w in range(WPL):
        s0 = 32 * w
        for l in range(32):
            for k in range(5):
                off = 1 << k
                if l >= off:
                    FS[k, s0 + l] = np.prod(mf[s0 + l - off + 1:s0 + l + 1])
                if l + off <= 31:
                    BS[k, s0 + l] = np.prod(mb[s0 + l:s0 + l + off])
            FE[s0 + l] = np.prod(mf[s0:s0 + l])
            BE[s0 + l] = np.prod(mb[s0 + l + 1:s0 + 32])
        MW[w] = np.prod(mf[s0:s0 + 32]); MWB[w] = np.prod(mb[s0:s0 + 32])
    return e1, e2, e3, pf, qb, FS, FE, BS, BE, MW, MWB


def _up(x, off):
    y = x.copy(); y[off:] = x[:-off]; return y


def _down(x, off):
    y = x.copy(); y[:-off] = x[off:]; return y


def _seg_solve(d, tabs, S, WPL):
    e1, e2, e3, pf, qb, FS, FE, BS, BE, MW, MWB = tabs
    nseg = 32 * WPL
    v = np.zeros((nseg, S)); v.flat[:len(d)] = d
    g = np.zeros(nseg)
    for t in range(S):
        g = v[:, t] * e2[:, t] - g * e3[:, t]; v[:, t] = g
    cin = np.zeros(nseg); Gw = np.zeros(WPL)
    for w in range(WPL):
        sl = slice(32 * w, 32 * w + 32); G = g[sl].copy()
        for k in range(5):
            G = FS[k, sl] * _up(G, 1 << k) + G
        ge = _up(G, 1); ge[0] = 0.0; Gw[w] = G[31]; cin[sl] = ge
    for w in range(WPL):
        sl = slice(32 * w, 32 * w + 32); cw = 0.0
        for p in range(w):
            cw = MW[p] * cw + Gw[p]
        cin[sl] = FE[sl] * cw + cin[sl]
    v += pf * cin[:, None]
    h = np.zeros(nseg)
    for t in range(S - 1, -1, -1):
        h = v[:, t] - e1[:, t] * h; v[:, t] = h
    cb = np.zeros(nseg)
    for w in range(WPL):
        sl = slice(32 * w, 32 * w + 32); G = h[sl].copy()
        for k in range(5):
            G = BS[k, sl] * _down(G, 1 << k) + G
        ge = _down(G, 1); ge[31] = 0.0; Gw[w] = G[0]; cb[sl] = ge
    for w in range(WPL):
        sl = slice(32 * w, 32 * w + 32); cw = 0.0
        for p in range(WPL - 1, w, -1):
            cw = MWB[p] * cw + Gw[p]
        cb[sl] = BE[sl] * cw + cb[sl]
    v += qb * cb[:, None]
    return v.flat[:len(d)].copy()


def _thomas(d, a1, a2, a3):
    d = d.copy(); n = len(d)
    for i in range(1, n):
        d[i] = d[i] * a2[i] - d[i - 1] * a3[i]
    x = np.zeros(n); x[-1] = d[-1]
    for i in range(n - 2, -1, -1):
        x[i] = d[i] - a1[i] * x[i + 1]
    return x


@pytest.mark.parametrize("kind,ntype,dim,S,WPL", [
    ("d", 3, 64, 3, 1), ("f", 3, 64, 3, 1), ("f", 3, 128, 5, 1), ("d", 3, 256, 9, 1), ("f", 4, 256, 9, 1),
    ("f", 3, 512, 9, 2), ("d", 4, 512, 5, 4), ("f", 1, 300, 5, 2), ("f", 2, 1000, 9, 4)])
def test_segmented_scan_equals_thomas(kind, ntype, dim, S, WPL):
    sc = oracle.fd_scheme_initiate("643c", ntype, dim) if kind == "d" else oracle.compact_filter_initiate(ntype, dim)
    _, _, a1, a2, a3 = sc.ac()
    assert 32 * WPL * S >= len(a1)
    d = np.random.default_rng(dim + S).standard_normal(len(a1))
    x0 = _thomas(d, a1, a2, a3)
    x1 = _seg_solve(d, _tables(a1, a2, a3, S, WPL), S, WPL)
    assert np.abs(x1 - x0).max() / np.abs(x0).max() < 1e-14
