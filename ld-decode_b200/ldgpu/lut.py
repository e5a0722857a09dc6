"""The TBC's windowed-sinc interpolation table, regenerated on the host.

The reference ships this table as lddecode/sinc_lut.npz and documents its
generator (lddecode/utils.py:73-124): 16 taps, 65536 fractional phases plus
one guard row, a sinc windowed by a Kaiser window with beta = 5, each
phase's float32 weights divided by their float32 sum.  Building it from
that recipe reproduces the shipped table bit for bit (checked against a
fixture of the shipped table in tests/test_host.py), so the file itself is
not needed at run time.
"""

import numpy as np

SINC_TAPS = 16
SINC_PHASES = 1 << 16
KAISER_BETA = 5


def build_sinc_lut(beta=KAISER_BETA, taps=SINC_TAPS, phases=SINC_PHASES):
    """float32[phases + 1, taps]; row p holds the weights for fractional
    position p/phases, tap t multiplies input sample floor(x) - taps/2+1 + t."""
    half = taps // 2
    offs = np.arange(half - 1, -half - 1, -1, dtype=np.float64)
    frac = np.arange(phases, dtype=np.float64) / phases
    x = frac[:, None] + offs[None, :]
    xpi = np.pi * x
    with np.errstate(divide="ignore", invalid="ignore"):
        sinc = np.where(x == 0, 1.0, np.sin(xpi) / xpi)
    r = x / half
    inside = (r >= -1) & (r <= 1)
    win = np.where(inside, np.i0(beta * np.sqrt(np.clip(1 - r * r, 0, None))) / np.i0(beta), 0.0)
    w = sinc * win
    w32 = w.astype(np.float32)
    norm = w.sum(axis=1, keepdims=True).astype(np.float32)
    out = np.empty((phases + 1, taps), dtype=np.float32)
    out[:phases] = w32 / norm
    out[phases] = out[phases - 1]
    return out
