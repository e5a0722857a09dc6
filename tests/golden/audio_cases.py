"""Seeded analog-audio downscale cases shared by make_golden.py and the tests
(no reference import: the tests run where the reference is absent)."""

import numpy as np

AUDIO_CASES = [
    # name, system, linecount, freq, timeoffset, audio dtype, audio length, glitch line
    ("ntsc_44100", "NTSC", 263, 44100, 1.2e-5, "float64", 28800, 120),
    ("ntsc_locked", "NTSC", 262, -2.8, 0.0, "float64", 28800, None),
    ("pal_44100", "PAL", 312, 44100, -5e-6, "float32", 32600, 200),
    ("ntsc_short", "NTSC", 263, 44100, 0.0, "float64", 20000, None),
]


def audio_case_inputs(system, linecount, dtype, alen, glitch, seed, line_period, audio_freqs):
    """Seeded line locations (linear wow plus a glitch line) and integer-valued
    FM-audio samples around the two carriers; shared with the tests."""
    rng = np.random.default_rng(seed)
    linelen = int(np.round(40e6 / (1e6 / line_period)))
    n = linecount + 12
    wow = 1 + 0.002 * np.sin(np.arange(n) / 37.0)
    lineinfo = 1000.5 + np.concatenate([[0], np.cumsum(wow[:-1] * linelen)])
    if glitch is not None:
        lineinfo[glitch:] += 60.0
    lf, rf_ = audio_freqs
    left = lf + rng.integers(-150000, 150000, alen).astype(np.float64)
    right = rf_ + rng.integers(-150000, 150000, alen).astype(np.float64)
    return lineinfo, left.astype(dtype), right.astype(dtype), linelen


AUDIO2_CASES = [("short", 28739), ("long", 80000)]
AUDIO2_STRIDE = 7


def audio2_inputs(audio_freqs, seed, n):
    """Seeded stage-1 audio (tones plus noise around the two carriers, with
    dropout spikes 2.5 MHz above the left carrier) for audio stage 2."""
    rng = np.random.default_rng(seed * 1000 + n)
    t = np.arange(n) / 1.25e6
    chans = []
    for cf, f0 in zip(audio_freqs, (1000.0, 440.0)):
        x = cf + 60e3 * np.sin(2 * np.pi * f0 * t) + rng.normal(0, 2e3, n)
        chans.append(x.astype(np.float32))
    for pos in rng.integers(50, n - 50, 6):
        chans[0][pos:pos + 3] = np.float32(audio_freqs[0] + 2.5e6)
    return chans
