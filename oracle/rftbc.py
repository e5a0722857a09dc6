"""CPU oracle for the RF TBC -- TEST INFRASTRUCTURE ONLY.

Restates Field.rf_tbc (lddecode/core.py:2724-2752) and the cubic scaler
`scale` (lddecode/utils.py:37-70) in FP64 numpy, each product and sum in the
reference's order (numpy rounds every elementwise operation on its own, as
numba does without fast-math).  Only tests/, smoke() and bench.py's
CPU-baseline leg import this file.
"""

import numpy as np


def scale(buf, begin, end, tgtlen):
    """utils.py:37-70 (mult = 1) over a whole line at once."""
    sfactor = (end - begin) / tgtlen
    coord = (np.arange(tgtlen, dtype=np.float64) * sfactor) + begin
    ic = coord.astype(np.int64)
    s = ic - 1
    if len(s) and (s.min() < 0 or s.max() + 4 > len(buf)):
        raise IndexError("cubic scaler tap outside the buffer")
    p0, p1, p2, p3 = buf[s], buf[s + 1], buf[s + 2], buf[s + 3]
    x = coord - ic
    return p1 + 0.5 * x * (p2 - p0 + x * (2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3 + x * (3.0 * (p1 - p2) + p3 - p0)))


def rf_tbc(inp, linelocs, delay, inlinelen, system, lineoffset, linecount):
    """core.py:2724-2752: int16 lines of the TBC'd raw RF."""
    fdata = np.asarray(inp).astype(np.float64)
    linelen = int(round(inlinelen))
    start = lineoffset if system == "NTSC" else 1
    out = []
    for line in range(start, start + linecount):
        v = scale(fdata, linelocs[line] - delay, linelocs[line + 1] - delay, linelen)
        out.append(np.round(v).astype(np.int16))
    return np.concatenate(out)
