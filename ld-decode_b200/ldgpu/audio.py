"""Analog audio to 16-bit 44.1 kHz (or line-locked) output, per field.

Restates lddecode/core.py:1423-1580 (`_downscale_audio_compute_locs_and_swow`,
`_downscale_audio_to_output`, `downscale_audio`) and utils.py:1328-1332
(`dsa_rescale_and_clip`).  The work per field is ~1500 output samples, each
the mean of a ~28-sample run of the field's 1.25 MHz audio; it runs on the
host in FP64 numpy (vectorised; only the reference's 1.5 % wow clamp, which
depends on the previous clamped value, is a scalar scan, and only where a
jump exists).

Same call signature and results as the reference: int16 interleaved L/R,
negated (`-dsa_rescale_and_clip`), samples whose run falls outside the audio
muted to 0 with a warning, and the time offset for the next field.
"""

import logging

import numpy as np

logger = logging.getLogger("lddecode")


def compute_locs_and_swow(lineinfo, line_period, linelen, linecount, timeoffset, freq, scale):
    """core.py:1423-1490: (locs, swow, arange, frametime)."""
    if freq < 0:
        timeoffset = 0
        freq = (1000000 / line_period) * -freq
    frametime = linecount / (1000000 / line_period)
    soundgap = 1 / freq
    # the reference's compiled np.arange: ceil((stop - start) / step) ticks at
    # start + i * step (numpy's own arange steps by (start + step) - start)
    stop = frametime + (soundgap / 2)
    nticks = max(int(np.ceil((stop - timeoffset) / soundgap)), 0)
    arange = timeoffset + np.arange(nticks, dtype=np.float64) * soundgap

    li = np.asarray(lineinfo, dtype=np.float64)
    linenum = ((arange * 1000000) / line_period) + 1
    intlinenum = linenum.astype(np.int64)  # int() truncates toward zero
    cur = np.empty_like(linenum)
    nxt = np.empty_like(linenum)
    neg = linenum < 0
    inside = ~neg & (len(li) > linenum + 2)
    past = ~neg & ~inside
    if neg.any():
        c = (li[0] + (linelen * linenum[neg])).astype(np.int64).astype(np.float64)
        cur[neg] = c
        nxt[neg] = c + linelen
    if inside.any():
        k = intlinenum[inside]
        cur[inside] = li[k]
        nxt[inside] = li[k + 1]
    if past.any():
        cur[past] = li[-2]
        nxt[past] = li[-2] + linelen
    sampleloc = cur + (nxt - cur) * (linenum - np.floor(linenum))
    swow = (nxt - cur) / linelen
    swow = (swow - 1) + 1
    # no disc turns more than 1.5 % off speed: a jump larger than that keeps
    # the previous (already clamped) factor
    jumps = np.nonzero(np.abs(np.diff(swow)) > 0.015)[0]
    if len(jumps):
        for i in range(int(jumps[0]) + 1, len(swow)):
            if np.abs(swow[i] - swow[i - 1]) > 0.015:
                swow[i] = swow[i - 1]
    locs = sampleloc / scale
    return locs, swow, arange, frametime


def rescale_and_clip(x):
    """utils.py:1328-1332 over an array: round half to even, clip to +-32766."""
    v = np.round(np.asarray(x, dtype=np.float64) * 32767.0 / 371081.0)
    return np.clip(v, -32766, 32766).astype(np.int64)


def to_output(arange, locs, swow, audio_left, audio_right, audio_lfreq, audio_rfreq):
    """core.py:1493-1533: interleaved int16 L/R and whether any sample was
    muted.  Sample i is the mean of audio[int(locs[i]):int(locs[i+1])]."""
    n = len(arange) - 1
    out = np.zeros(2 * n, dtype=np.int16)
    if n <= 0:
        return out, False
    al = np.asarray(audio_left)
    ar = np.asarray(audio_right)
    start = locs[:-1].astype(np.int64)
    end = locs[1:].astype(np.int64)
    ok = (end > start) & (end < len(al))
    failed = not bool(ok.all())
    idx = np.nonzero(ok)[0]
    if len(idx):
        s, e = start[idx], end[idx]
        acc = al.dtype if al.dtype.kind == "f" else np.dtype(np.float64)
        ml = _run_means(al, s, e, acc)
        mr = _run_means(ar, s, e, acc)
        left = (ml * swow[idx]) - audio_lfreq
        right = (mr * swow[idx]) - audio_rfreq
        out[2 * idx] = -rescale_and_clip(left)
        out[2 * idx + 1] = -rescale_and_clip(right)
    return out, failed


def _run_means(a, s, e, acc):
    """Mean of a[s_i:e_i] for every run, each sum accumulated in order in the
    array's own precision (float32 audio sums in float32, as the reference's
    compiled np.mean does), vectorised across runs; the sum is divided by the
    run length in float64."""
    lens = e - s
    total = np.zeros(len(s), dtype=acc)
    for k in range(int(lens.max())):
        m = lens > k
        total[m] += a[s[m] + k].astype(acc, copy=False)
    return total.astype(np.float64) / lens


def downscale_audio(audio, lineinfo, rf, linecount, timeoffset=0, freq=44100, rv=None):
    """core.py:1538-1580: (int16 interleaved L/R, next field's time offset)."""
    locs, swow, arange, frametime = compute_locs_and_swow(
        lineinfo, rf.SysParams["line_period"], rf.linelen, linecount, timeoffset, freq,
        rf.Filters["audio_fdiv"])
    output16, failed = to_output(arange, locs, swow, audio["audio_left"], audio["audio_right"],
                                 rf.SysParams["audio_lfreq"], rf.SysParams["audio_rfreq"])
    if failed:
        logger.warning("Analog audio processing error, muting samples")
    if rv is not None:
        rv["dsaudio"] = output16
        rv["audio_next_offset"] = arange[-1] - frametime
    return output16, arange[-1] - frametime
