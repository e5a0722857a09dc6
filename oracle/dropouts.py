"""CPU oracle for dropout detection -- TEST INFRASTRUCTURE ONLY.

Restates Field.dropout_detect (lddecode/core.py:2962-2983) and its stages:
  * dropout_detect_demod (core.py:2829-2887): the per-sample error mask --
    rfhpf beyond +-3 standard deviations (moved by video_rot), demod_raw
    above fs/2, demod outside its valid range and demod_05 outside its own
    (lower limits relaxed in the sync areas of every line and in whole
    vertical-sync lines), cleared outside the field's lines;
  * build_errlist (core.py:2889-2908): the sequential merge of error samples
    into padded spans;
  * dropout_errlist_to_tbc (core.py:2910-2960): spans to (TBC line, start x,
    end x), split at line ends.
The limits are float32 (the reference fills float32 arrays with them); the
rfhpf standard deviation is FP64 over the whole field read, as numba's
np.std computes it up to summation order.  Only tests/, smoke() and
bench.py's CPU-baseline leg import this file.
"""

import numpy as np


def limits(system, ire0, hz_ire, vsync_ire):
    """(vmin, vmax, vmin05, vmax05, sync_min, sync_min05) in Hz, float32,
    core.py:2846-2867 (iretohz with DecoderParams)."""
    pal = system == "PAL"

    def hz(ire):
        return np.float32(ire0 + hz_ire * ire)
    return (hz(-70 if pal else -50), hz(150 if pal else 160), hz(-30), hz(115),
            hz(vsync_ire - 60 if pal else vsync_ire - 35), hz(vsync_ire - 10))


def vsync_lines(system, isfirst):
    """Field.get_vsync_lines (core.py:2814-2827)."""
    rv = list(range(1, 10 if isfirst else 9))
    if system == "PAL":
        rv += list(range(311 if isfirst else 310, 318))
    return rv


def _py_slice(a, b, n):
    """[a:b] of a length-n array as Python normalises it."""
    return slice(*slice(a, b).indices(n)[:2])


def mask(demod, demod_05, demod_raw, rfhpf, linelocs, lineoffset, linecount, isfirst, hsync_len, system,
         video_rot, freq_hz_half, lim):
    """dropout_detect_demod: bool mask over the field read (core.py:2829-2887)."""
    n = len(demod)
    rf = np.asarray(rfhpf, np.float32).astype(np.float64)
    rfstd = float(np.sqrt(np.mean((rf - rf.mean()) ** 2)))
    bad_rf = (rf < -rfstd * 3) | (rf > rfstd * 3)
    iserr = np.zeros(n, bool)
    iserr[video_rot:] = bad_rf[:-video_rot]
    vmin, vmax, vmin05, vmax05, smin, smin05 = lim
    valid_min = np.full(n, vmin, np.float32)
    valid_max = np.full(n, vmax, np.float32)
    valid_min05 = np.full(n, vmin05, np.float32)
    valid_max05 = np.full(n, vmax05, np.float32)
    ll = np.asarray(linelocs, np.float64)
    vs = set(vsync_lines(system, isfirst))
    for line in range(1, len(ll)):
        a = int(ll[line])
        b = int(ll[line + 1]) if line in vs else a + hsync_len
        s = _py_slice(a, b, n)
        valid_min[s] = smin
        valid_min05[s] = smin05
    dr = np.asarray(demod_raw, np.float32)
    d = np.asarray(demod, np.float32)
    d5 = np.asarray(demod_05, np.float32)
    iserr |= dr.astype(np.float64) > freq_hz_half
    iserr |= (d < valid_min) | (d > valid_max)
    iserr |= (d5 < valid_min05) | (d5 > valid_max05)
    iserr[_py_slice(None, int(ll[lineoffset + 1]), n)] = False
    iserr[_py_slice(int(ll[lineoffset + linecount + 1]), None, n)] = False
    return iserr, rfstd


def build_errlist(errmap, linelocs, lineoffset, freq_mhz):
    """core.py:2889-2908 (pure Python loop over the error samples)."""
    errmap = [int(e) for e in errmap]
    ll0 = float(linelocs[lineoffset])
    firsterr = next(e for e in errmap if e >= ll0)
    cur = (firsterr, firsterr)
    out = []
    cap = freq_mhz * 12
    for e in errmap:
        if e > cur[0] and e <= cur[1] + 20:
            pad = (e - cur[0]) * 1.7
            pad = min(pad, cap)
            cur = (cur[0], cur[0] + pad)
        elif e > firsterr:
            out.append((cur[0] - 8, cur[1] + 4))
            cur = (e, e)
    out.append(cur)
    return out


def errlist_to_tbc(errlist, linelocs, lineoffset, linecount, outlinelen):
    """core.py:2910-2960: (line, start x, end x) per dropout, TBC lines
    counted from 1 (the reference's field lines before the final -1)."""
    drops = []
    if not errlist:
        return drops
    ll = np.asarray(linelocs, np.float64)
    rest = list(errlist)
    cur = rest.pop(0)
    while rest and cur[0] < ll[lineoffset]:
        cur = rest.pop(0)
    for line in range(lineoffset, linecount + lineoffset):
        while cur is not None and ll[line] <= cur[0] <= ll[line + 1]:
            span = ll[line + 1] - ll[line]
            start = int(((cur[0] - ll[line]) / span) * outlinelen)
            end = int(np.round(((cur[1] - ll[line]) / span) * outlinelen))
            first = line + 1 - lineoffset
            if end > outlinelen:
                k = end // outlinelen
                drops.append((first, start, outlinelen))
                for j in range(k - 1):
                    drops.append((first + j + 1, 0, outlinelen))
                drops.append((first + k, 0, end % outlinelen))
            else:
                drops.append((first, start, end))
            cur = rest.pop(0) if rest else None
    return drops


def detect(iserr, linelocs, lineoffset, linecount, freq_mhz, outlinelen):
    """Field.dropout_detect (core.py:2962-2983): (lines, starts, ends)."""
    errmap = np.nonzero(iserr)[0]
    lines, starts, ends = [], [], []
    if len(errmap) and errmap[-1] > linelocs[lineoffset]:
        el = build_errlist(errmap, linelocs, lineoffset, freq_mhz)
        for r in errlist_to_tbc(el, linelocs, lineoffset, linecount, outlinelen):
            lines.append(r[0] - 1)
            starts.append(int(r[1]))
            ends.append(int(r[2]))
    return lines, starts, ends
