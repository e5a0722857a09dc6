"""Field read windows over a capture's overlap-save blocks.

The reference reads a field by asking DemodCache for a run of 32768-sample
blocks and concatenating each block's cut outputs (lddecode/core.py:
1343-1413 DemodCache.read, 4030-4042 LDdecode.decodefield).  Block b covers
raw samples [b*U, b*U + N) and keeps outputs for raw samples
[b*U + blockcut, b*U + blockcut + U), U = N - blockcut - blockcut_end, so a
capture-wide output array indexed by b*U + i holds every block's cut output
back to back, and a field read is a window of it starting at
startloc = first_block * U.  Field-local sample 0 is raw sample
startloc + blockcut.
"""

from dataclasses import dataclass


@dataclass
class FieldWindow:
    readloc: int       # int(start - blockcut), clamped at 0
    first_block: int   # first demod block of the read
    nblocks: int       # blocks concatenated
    startloc: int      # first_block * U (capture-wide output index of field sample 0)
    length: int        # nblocks * U output samples


def readlen_for(rf):
    """Samples LDdecode reads per field (core.py:3625-3632)."""
    if rf.system == "PAL":
        return rf.linelen * 400
    return ((rf.linelen * 350) // 16384) * 16384


def field_window(rf, start, readlen=None):
    """The blocks decodefield(start) reads (core.py:4030-4042, 1358-1409)."""
    readlen = readlen_for(rf) if readlen is None else readlen
    bs = rf.blocklen
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    readloc = max(int(start - rf.blockcut), 0)
    begin = (readloc // bs) * bs
    length = ((readlen // bs) + 2) * bs
    end = begin + length
    first = begin // U
    last = end // U
    n = last - first + 1
    return FieldWindow(readloc, first, n, first * U, n * U)


def blocks_in_capture(rf, nsamples):
    """How many whole blocks a capture of `nsamples` raw samples holds."""
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    if nsamples < rf.blocklen:
        return 0
    return (nsamples - rf.blocklen) // U + 1
