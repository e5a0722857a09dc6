"""CPU oracle for analog audio stage 2 -- TEST INFRASTRUCTURE ONLY.

Restates RFDecode.runfilter_audio_phase2 and audio_phase2
(lddecode/core.py:884-950) and findpeaks (lddecode/utils.py:1207-1216):
per transform of `blocklen` stage-1 samples, the carrier is removed, samples
within 8 of each left-channel spike above 500 kHz are zeroed in both
channels, the low-pass / de-emphasis filter is applied by FFT (complex128)
and the carrier restored; longer inputs are stitched from transforms that
overlap by 512 samples.  Only tests/, smoke() and bench.py's CPU-baseline
leg import this file.
"""

import numpy as np


def findpeaks(array, low=0):
    a2 = array.copy()
    a2[a2 < low] = 0
    return [int(i) - 1 for i in np.where(np.logical_and(a2[:-1] > a2[-1], a2[1:] > a2[:-1]))[0]]


def run_phase2(left, right, start, blocklen, centers, filters):
    outs = []
    clips = None
    for x, cf, filt, is_left in ((left, centers[0], filters[0], True), (right, centers[1], filters[1], False)):
        raw = np.asarray(x[start:start + blocklen], dtype=np.float32).copy()
        raw -= np.float32(cf)
        if is_left:
            clips = findpeaks(raw, 500000)
        for loc in clips:
            raw[max(0, loc - 8):min(loc + 8, len(raw))] = 0
        if len(raw) < len(filt):
            a2 = np.zeros(len(filt), dtype=np.complex128)
            a2[:len(raw)] = raw
        else:
            a2 = raw
        outs.append(np.fft.ifft(np.fft.fft(a2) * filt).real[:len(raw)] + cf)
    return outs


def audio_phase2(left, right, blocklen, centers, filters):
    """(left, right) float64 stage-2 audio."""
    n = len(left)
    first = run_phase2(left, right, 0, blocklen, centers, filters)
    if len(first[0]) >= n:
        return first[0][:n], first[1][:n]
    out = [np.zeros(n, np.float32), np.zeros(n, np.float32)]
    for c in range(2):
        out[c][:len(first[c])] = first[c]
    askip = 512
    sjump = blocklen - askip
    ostart = len(first[0])
    for sample in range(sjump, n - sjump, sjump):
        tmp = run_phase2(left, right, sample, blocklen, centers, filters)
        oend = ostart + len(tmp[0]) - askip
        for c in range(2):
            out[c][ostart:oend] = tmp[c][askip:]
        ostart += len(tmp[0]) - askip
    tmp = run_phase2(left, right, n - blocklen - 1, blocklen, centers, filters)
    for c in range(2):
        out[c][n - (len(tmp[c]) - askip):] = tmp[c][askip:]
    return out[0], out[1]
