"""Seeded EFM-like test signals for the EFM PLL, shared by make_golden.py and
the tests (no reference import).  Integer and basic float64 arithmetic only,
so a signal is the same on every CPU."""

import numpy as np

BIT_PERIOD = 40000000.0 / 4321800.0  # samples per EFM bit at 40 MSPS


def efm_signal(seed, nruns, drift=0.0, amp=1500, noise=40, ramp=4.0, dropout=None):
    """int16 samples of an NRZI signal whose runs are 3..11 bit periods
    (EFM's run lengths), the bit period scaled by 1 + drift * t / T (a
    linear speed change over the signal), edges ramped linearly over +-ramp
    samples, integer noise added; `dropout` = (start, length) replaces that
    span with low-level noise (many short invalid runs, then a long gap)."""
    rng = np.random.default_rng(seed)
    runs = rng.integers(3, 12, nruns).astype(np.float64)
    t = np.cumsum(runs)                      # edge times in bits
    scale = 1.0 + drift * (t / t[-1])
    edges = t * BIT_PERIOD * scale + 37.25
    n = int(edges[-1]) + 64
    x = np.empty(n, dtype=np.float64)
    idx = np.arange(n, dtype=np.float64)
    k = np.searchsorted(edges, idx, side="right")  # edges at or before sample
    level = np.where(k % 2 == 0, 1.0, -1.0)
    # distance to the nearest edge, signed toward the level after it
    prev_e = np.where(k > 0, edges[np.maximum(k - 1, 0)], -1e9)
    next_e = np.where(k < len(edges), edges[np.minimum(k, len(edges) - 1)], 1e9)
    d_prev = idx - prev_e
    d_next = next_e - idx
    near_prev = d_prev < ramp
    near_next = d_next < ramp
    x[:] = level
    x[near_prev] = level[near_prev] * (d_prev[near_prev] / ramp)
    x[near_next & ~near_prev] = level[near_next & ~near_prev] * (d_next[near_next & ~near_prev] / ramp)
    v = np.round(x * amp) + rng.integers(-noise, noise + 1, n)
    if dropout is not None:
        s0, ln = dropout
        v[s0:s0 + ln] = rng.integers(-3, 4, ln)
    v = np.clip(v, -32768, 32767).astype(np.int16)
    # exact zeros on some crossings (a zero counts as non-negative)
    z = rng.integers(0, n, n // 97)
    v[z] = np.where(np.abs(v[z]) < 60, 0, v[z])
    return v


EFM_CASES = [
    # name, seed, runs, drift, dropout, buffer lengths (cycled)
    ("steady", 901, 40000, 0.0, None, [65536]),
    ("drift_up", 902, 40000, 0.06, None, [31713, 100003, 7]),
    ("drift_down_clamped", 903, 40000, -0.14, None, [50000]),
    ("dropout", 904, 30000, 0.01, (500000, 20000), [65536, 1, 4095]),
]


def efm_case(name):
    for c in EFM_CASES:
        if c[0] == name:
            _, seed, nruns, drift, dropout, bufs = c
            return efm_signal(seed, nruns, drift=drift, dropout=dropout), bufs
    raise KeyError(name)


def split(x, bufs):
    """x cut into buffers of the cycled lengths `bufs`."""
    out, pos, i = [], 0, 0
    while pos < len(x):
        n = bufs[i % len(bufs)]
        out.append(x[pos:pos + n])
        pos += n
        i += 1
    return out
