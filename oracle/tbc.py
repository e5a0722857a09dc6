"""CPU oracle for the time-base corrector -- TEST INFRASTRUCTURE ONLY.

FP64 numpy restatement of the reference's field resampler:
  * Field.computewow_scaled (lddecode/core.py:2591-2623): a linear spline
    through (i * inlinelen, linelocs[i]) evaluated at every output pixel,
    giving the input coordinate and its derivative (the wow factor); the
    quadratic and cubic (natural) forms call scipy's make_interp_spline
    with the reference's arguments, as the reference does;
  * scale_field (lddecode/utils.py:127-183): wow level adjustment with the
    median / 15*MAD outlier rule, then a 16-tap windowed-sinc gather with
    linear interpolation between the 65536 LUT phases;
  * hz_to_output_array (lddecode/utils.py:1061-1075).

Two coordinate modes: `coord_f32=True` re-applies the reference's float32
cast of the resampling coordinate (utils.py:160) and reproduces the
reference as it is; `coord_f32=False` keeps the coordinate in FP64, which is
the accuracy target (the reference's own cast costs it up to ~130 LSB).
Only tests/, smoke() and bench.py's CPU-baseline leg import this file.
"""

import numpy as np

TAPS = 16
PHASES = 1 << 16


def pixel_coords(linelocs, inlinelen, outlinelen, outlinecount, lineoffset, method="linear"):
    """Input coordinate and wow (d coord / d x) of every output pixel,
    x = i * inlinelen/outlinelen for i in [0, (outlinecount+lineoffset+1) *
    outlinelen) (core.py:2595-2621).  Linear: pixel x uses the spline
    segment j with j*inlinelen <= x < (j+1)*inlinelen, clamped to the
    first/last segment, which is how a degree-1 B-spline picks its interval.
    Quadratic / cubic: core.py:2605-2613 (k = 2 with scipy's default knots,
    k = 3 with natural end conditions)."""
    act = np.asarray(linelocs, dtype=np.float64)
    n = len(act)
    exp = np.array([i * inlinelen for i in range(n)], dtype=np.float64)
    nout = outlinecount * outlinelen + (lineoffset + 1) * outlinelen
    x = np.arange(nout) * (inlinelen / outlinelen)
    if method != "linear":
        from scipy import interpolate
        k, bc = {"quadratic": (2, None), "cubic": (3, "natural")}[method]
        spl = interpolate.make_interp_spline(exp, act, k=k, bc_type=bc, check_finite=False)
        return spl(x), spl(x, 1)
    seg = np.searchsorted(exp, x, side="right") - 1
    seg = np.clip(seg, 0, n - 2)
    x0, x1 = exp[seg], exp[seg + 1]
    y0, y1 = act[seg], act[seg + 1]
    # degree-1 de Boor evaluation: basis weights w*(x1-x), w*(x-x0), w = 1/h
    w = 1.0 / (x1 - x0)
    coords = y0 * (w * (x1 - x)) + y1 * (w * (x - x0))
    wow = y0 * (-w) + y1 * w
    return coords, wow


def level_adjusts(wow, smoothing=0, outwidth=910, threshold=15):
    """Per-pixel amplitude correction (utils.py:132-149)."""
    med = np.median(wow)
    mad = np.median(np.abs(wow - med))
    thr = threshold * mad if mad > 0 else 0.001
    la = np.where(np.abs(wow - med) > thr, med, wow)
    if smoothing > 0:
        alpha = 1 / (smoothing * outwidth)
        la = la.copy()
        for i in range(1, len(la)):
            la[i] = alpha * la[i] + (1 - alpha) * la[i - 1]
    return la


def scale_field(buf, coords, wow, lut, lineoffset, outwidth, nout,
                coord_f32=False, smoothing=0, threshold=15):
    """16-tap sinc resampling of `buf` (float32) at coords (utils.py:127-183).

    Returns float32[nout]."""
    la = level_adjusts(wow, smoothing, outwidth, threshold)
    start = outwidth * (lineoffset + 1)
    idx = np.arange(start, start + nout)
    c = coords[idx]
    if coord_f32:
        c = c.astype(np.float32).astype(np.float64)
    ci = c.astype(np.int64)
    ph = (c - ci) * PHASES
    ps = ph.astype(np.int64)
    alpha = (ph - ps).astype(np.float32)
    w0 = lut[ps]
    w1 = lut[ps + 1]
    w = (w0 + alpha[:, None] * (w1 - w0)).astype(np.float32)
    taps = (ci - (TAPS // 2 - 1))[:, None] + np.arange(TAPS)[None, :]
    prod = (buf[taps].astype(np.float32) * w).astype(np.float64)
    res = prod.sum(axis=1)
    return (la[idx] * res).astype(np.float32)


def hz_to_output(x, ire0, hz_ire, output_zero, vsync_ire, out_scale):
    """uint16 = clip(x*scale + offset + 0.5) truncated (utils.py:1061-1075)."""
    scale = out_scale / hz_ire
    offset = output_zero - vsync_ire * out_scale - ire0 * scale
    v = np.asarray(x, dtype=np.float64) * scale + offset + 0.5
    return np.clip(v, 0, 65535).astype(np.uint16)
