"""The FM discriminator's arctan (csrc/ldg_demod.cu atan01 / arg_2pi): the
Abramowitz & Stegun 4.4.49 polynomial and the octant reflections, restated
in float32 steps, against numpy's FP64 angle -- the coefficients' published
bound (2e-8 on [0, 1]) and the reflections into [0, 2 pi)."""

import numpy as np

COEF = [0.0028662257, -0.0161657367, 0.0429096138, -0.0752896400, 0.1065626393, -0.1420889944,
        0.1999355085, -0.3333314528, 1.0]


def _fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def atan01(t):
    t = t.astype(np.float32)
    t2 = (t * t).astype(np.float32)
    p = np.full_like(t, np.float32(COEF[0]))
    for c in COEF[1:]:
        p = _fma32(p, t2, np.full_like(t, np.float32(c)))
    return (t * p).astype(np.float32)


def arg_2pi(im, re):
    im = im.astype(np.float32)
    re = re.astype(np.float32)
    ax, ay = np.abs(re), np.abs(im)
    mx, mn = np.maximum(ax, ay), np.minimum(ax, ay)
    with np.errstate(invalid="ignore", divide="ignore"):
        t = np.where(mx > 0, (mn / mx).astype(np.float32), np.float32(0))
    r = atan01(t)
    r = np.where(ay > ax, np.float32(np.pi / 2) - r, r).astype(np.float32)
    r = np.where(re < 0, np.float32(np.pi) - r, r).astype(np.float32)
    return np.where(im < 0, np.float32(2 * np.pi) - r, r).astype(np.float32)


def test_polynomial_bound():
    x = np.linspace(0.0, 1.0, 200001)
    p = np.zeros_like(x)
    for c in COEF:
        p = p * x * x + c
    assert np.abs(x * p - np.arctan(x)).max() <= 2e-8


def test_arg_all_quadrants():
    rng = np.random.default_rng(5)
    re = rng.standard_normal(400000).astype(np.float32) * np.float32(1e4)
    im = rng.standard_normal(400000).astype(np.float32) * np.float32(1e4)
    # axes and diagonals too
    re = np.concatenate([re, [1, 0, -1, 0, 1, -1, -1, 1, 0]]).astype(np.float32)
    im = np.concatenate([im, [0, 1, 0, -1, 1, 1, -1, -1, 0]]).astype(np.float32)
    got = arg_2pi(im, re).astype(np.float64)
    want = np.mod(np.arctan2(im.astype(np.float64), re.astype(np.float64)), 2 * np.pi)
    d = np.abs(got - want)
    d = np.minimum(d, 2 * np.pi - d)  # 0 and 2 pi are the same angle
    # float32's spacing just below 2 pi is 4.8e-7: within ~1.25 of it
    assert d.max() <= 6e-7, d.max()
    assert np.all((got >= 0) & (got <= np.float32(2 * np.pi)))
