"""Small host-side numeric helpers of the decoder (FP64, numpy).

calczc: sub-sample threshold crossing (lddecode/utils.py:795-854).
fm_wave: FM synthesis from an instantaneous-frequency array
(lddecode/utils.py:1009-1023, genwave), used for the delay calibration block.
"""

import numpy as np


def _first_cross(seg, target, rising):
    if rising:
        hit = np.nonzero((seg[:-1] < target) & (seg[1:] >= target))[0]
    else:
        hit = np.nonzero((seg[:-1] > target) & (seg[1:] <= target))[0]
    return int(hit[0]) + 1 if len(hit) else None


def calczc(data, start_offset, target, edge=0, count=16, reverse=False):
    """Location (fractional sample) where `data` first crosses `target`
    within `count` samples of `start_offset`; edge -1 falling, 0 either
    (decided by data[start]), 1 rising.  None if there is no crossing."""
    if reverse:
        rev = calczc(data[int(start_offset)::-1], 0, target, edge, count)
        return None if rev is None else start_offset - rev
    s = int(start_offset)
    icount = int(count + 1)
    if edge == 0:
        edge = 1 if float(data[s]) < target else -1
    # comparisons and interpolation in float64, as the reference's numba code
    # promotes float32 samples against a float64 target
    loc = _first_cross(np.asarray(data[s:s + icount], dtype=np.float64), target, edge == 1)
    if loc is None:
        return None
    x = s + loc
    a = float(data[x - 1]) - target
    b = float(data[x]) - target
    y = -a / (-a + b) if b - a != 0 else 0
    return x - 1 + y


def fm_wave(rate, freq, initialphase=0.0):
    """sin of the running phase pi * cumsum(rate/freq), starting at
    initialphase (phase wrapped to (-pi, pi] as it accumulates)."""
    rate = np.asarray(rate, dtype=np.float64)
    out = np.empty(len(rate), dtype=np.double)
    angle = initialphase
    step = np.pi * (rate / freq)
    tau = 2 * np.pi
    for i in range(len(rate)):
        out[i] = np.sin(angle)
        angle += step[i]
        if angle > np.pi:
            angle -= tau
    return out
