"""The spline forms the GPU's wow_spline_kernel builds, restated in numpy,
against scipy's make_interp_spline as the reference calls it
(lddecode/core.py:2602-2613), on the golden fields' line locations (also
with added wow and displaced lines):

* cubic, natural ends: the second-derivative form (one tridiagonal system
  for M_1 .. M_{n-2}); within 1e-5 samples of scipy (whose own B-spline
  solve leaves s''(x_0) slightly off zero) and the wow factor to 1e-8;
* quadratic, scipy's knots for even degree (the data points' midpoints
  without the first and last): the piecewise-linear derivative's values at
  the breakpoints from one tridiagonal system (the integral of s' over
  each data interval); within 1e-8 samples.

Host only."""

import numpy as np
import pytest
from scipy import interpolate

from conftest import golden
from ldgpu.rfdecode import RFParams


def thomas(sub, dia, sup, rhs):
    m = len(dia)
    cp, dp = np.zeros(m), np.zeros(m)
    for r in range(m):
        den = dia[r] - (sub[r] * cp[r - 1] if r else 0.0)
        cp[r] = sup[r] / den
        dp[r] = (rhs[r] - (sub[r] * dp[r - 1] if r else 0.0)) / den
    for r in range(m - 2, -1, -1):
        dp[r] -= cp[r] * dp[r + 1]
    return dp


def pieces(y, inl, k):
    """(left edge, anchor, c0, c1, c2, c3) per piece, as the kernel builds them."""
    n = len(y)
    x = np.array([i * inl for i in range(n)])
    if k == 3:
        h = np.diff(x)
        rhs = 6 * ((y[2:] - y[1:-1]) / h[1:] - (y[1:-1] - y[:-2]) / h[:-1])
        M = np.zeros(n)
        M[1:-1] = thomas(h[:-1], 2 * (h[:-1] + h[1:]), h[1:], rhs)
        c1 = (y[1:] - y[:-1]) / h - h * (2 * M[:-1] + M[1:]) / 6
        return np.stack([x[:-1], x[:-1], y[:-1], c1, M[:-1] / 2, (M[1:] - M[:-1]) / (6 * h)], 1)
    bk = np.concatenate([[x[0]], (x[1:-2] + x[2:-1]) / 2, [x[-1]]])  # n-1 breakpoints
    sub, dia, sup = np.zeros(n - 1), np.zeros(n - 1), np.zeros(n - 1)

    def integ(p, q, j, a, b, r):  # integral of s' over [p, q] inside segment j
        w = bk[j + 1] - bk[j]
        rp, rq = (p - bk[j]) / w, (q - bk[j]) / w
        hw = (q - p) / 2
        a[r] += hw * ((1 - rp) + (1 - rq))
        b[r] += hw * (rp + rq)

    for r in range(n - 1):
        if r == 0:
            integ(x[0], x[1], 0, dia, sup, r)
        elif r == n - 2:
            integ(x[n - 2], x[n - 1], n - 3, sub, dia, r)
        else:
            integ(x[r], bk[r], r - 1, sub, dia, r)
            integ(bk[r], x[r + 1], r, dia, sup, r)
    D = thomas(sub, dia, sup, y[1:] - y[:-1])
    out = []
    for p in range(n - 2):
        left, w = bk[p], bk[p + 1] - bk[p]
        a = 0 if p == 0 else (n - 1 if p == n - 3 else p + 1)
        dd = D[p + 1] - D[p]
        out.append([left, x[a], y[a], D[p] + dd * (x[a] - left) / w, dd / (2 * w), 0.0])
    return np.array(out)


def evaluate(pc, xs):
    p = np.clip(np.searchsorted(pc[:, 0], xs, side="right") - 1, 0, len(pc) - 1)
    c = pc[p]
    t = xs - c[:, 1]
    return c[:, 2] + t * (c[:, 3] + t * (c[:, 4] + t * c[:, 5])), c[:, 3] + t * (2 * c[:, 4] + 3 * t * c[:, 5])


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
@pytest.mark.parametrize("k", [2, 3])
def test_spline_forms_match_scipy(system, k):
    g = golden("wow_interp_" + system.lower())
    rf = RFParams(system=system)
    outw = rf.SysParams["outlinelen"]
    for case in ("c0_linelocs", "c2_linelocs"):
        y = g[case]
        x = np.array([i * rf.linelen for i in range(len(y))])
        spl = interpolate.make_interp_spline(x, y, k=k, bc_type="natural" if k == 3 else None, check_finite=False)
        xs = np.arange(int(g["c0_wow_stats"][0])) * (rf.linelen / outw)
        v, d = evaluate(pieces(y, rf.linelen, k), xs)
        tol_v, tol_d = (1e-5, 1e-8) if k == 3 else (1e-8, 1e-11)
        assert np.abs(v - spl(xs)).max() < tol_v, (case, np.abs(v - spl(xs)).max())
        assert np.abs(d - spl(xs, 1)).max() < tol_d, (case, np.abs(d - spl(xs, 1)).max())
        # the data points are interpolated, and the pieces join smoothly
        assert np.abs(evaluate(pieces(y, rf.linelen, k), x)[0] - y).max() < 1e-6
