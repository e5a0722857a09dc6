"""CPU oracle for .lds ingest -- TEST INFRASTRUCTURE ONLY.

Restates unpack_data_4_40 (lddecode/utils.py:371-391): four 10-bit samples
in 5 bytes, most significant bits first, returned as (v - 512) << 6 in
int16; and the inverse packing used to make test captures.  Only tests/,
smoke() and bench.py's CPU-baseline leg import this file.
"""

import numpy as np


def unpack_4_40(indata, readlen, offset):
    b = np.asarray(indata, np.uint8).astype(np.uint16)
    ng = len(b) // 5
    g = b[:ng * 5].reshape(ng, 5)
    v = np.empty((ng, 4), np.uint16)
    v[:, 0] = (g[:, 0] << 2) | ((g[:, 1] >> 6) & 0x03)
    v[:, 1] = ((g[:, 1] & 0x3F) << 4) | ((g[:, 2] >> 4) & 0x0F)
    v[:, 2] = ((g[:, 2] & 0x0F) << 6) | ((g[:, 3] >> 2) & 0x3F)
    v[:, 3] = ((g[:, 3] & 0x03) << 8) | g[:, 4]
    u = v.reshape(-1)[offset:offset + readlen].astype(np.int32)
    return ((u - 512) * 64).astype(np.int16)


def pack_4_40(values):
    """10-bit values (length a multiple of 4) to packed bytes."""
    v = np.asarray(values, np.uint16).reshape(-1, 4)
    out = np.empty((len(v), 5), np.uint8)
    out[:, 0] = v[:, 0] >> 2
    out[:, 1] = ((v[:, 0] & 0x03) << 6) | (v[:, 1] >> 4)
    out[:, 2] = ((v[:, 1] & 0x0F) << 4) | (v[:, 2] >> 6)
    out[:, 3] = ((v[:, 2] & 0x3F) << 2) | (v[:, 3] >> 8)
    out[:, 4] = v[:, 3] & 0xFF
    return out.reshape(-1)
