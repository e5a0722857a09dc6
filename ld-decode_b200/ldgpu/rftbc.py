"""RF TBC on the GPU (ldg_rf_tbc): Field.rf_tbc (lddecode/core.py:2724-2752),
the raw RF resampled line by line with the reference's cubic scaler
(utils.py:37-70) to int(round(inlinelen)) samples per line, int16 -- the
.tbc.ldf side output of LDdecode (core.py:4005-4007).  Bit-identical to the
reference for the same line locations and video delay."""

import ctypes

import numpy as np

from . import lib as L


def descriptor(rf, input_ptr, n, linelocs_ptr, nlines, lineoffset, linecount, out_ptr, delay=None):
    d = L.RfTbcField()
    d.input = input_ptr
    d.len = int(n)
    d.linelocs = linelocs_ptr
    d.nlines = int(nlines)
    d.startline = int(lineoffset) if rf.system == "NTSC" else 1
    d.linecount = int(linecount)
    d.linelen = int(round(rf.linelen))
    d.delay = float(rf.delays["video_white"] if delay is None else delay)
    d.out = out_ptr
    return d


def run(rf, descs, stream=None):
    """ldg_rf_tbc over DropoutField-style descriptors (RfTbcField); enqueued
    on `stream` (raw handle; None: torch's default stream)."""
    if not descs:
        return
    arr = (L.RfTbcField * len(descs))(*descs)
    L.check(rf._ctx._lib.ldg_rf_tbc(rf._ctx.handle, arr, len(arr), stream if stream else 1))


def line_samples(rf):
    return int(round(rf.linelen))


def rf_tbc_located(rf, fields, cap, out=None, stream=None, delay=None):
    """RF TBC of every field of LocatedFields over the raw capture `cap`
    (int16 device tensor; output index j of the demodulator is raw sample
    j + blockcut).  Returns the int16 device tensor of all fields' lines,
    field after field (linecount * linelen each), and the offsets."""
    import torch
    a = fields.arrays()
    n = len(a["startloc"])
    ll = line_samples(rf)
    counts = a["linecount"].astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(counts * ll)]).astype(np.int64)
    if out is None:
        out = torch.empty(max(int(offs[-1]), 1), dtype=torch.int16, device=cap.device)
    base = cap.data_ptr() + 2 * rf.blockcut
    descs = [descriptor(rf, base + 2 * int(a["startloc"][i]), a["length"][i], int(a["linelocs_ptr"][i]),
                        a["nlines"][i], a["lineoffset"][i], a["linecount"][i], out.data_ptr() + 2 * int(offs[i]),
                        delay) for i in range(n)]
    run(rf, descs, stream)
    return out, offs


def rf_tbc_host_field(rf, inp, linelocs, lineoffset, linecount, delay=None):
    """One field with host buffers (Field.data["input"], line locations):
    uploads, runs, waits; returns the int16 numpy output."""
    import torch
    from .field import tbc_status
    dev = torch.device("cuda", torch.cuda.current_device())
    ti = torch.from_numpy(np.ascontiguousarray(inp, np.int16)).to(dev)
    tl = torch.from_numpy(np.ascontiguousarray(linelocs, np.float64)).to(dev)
    ll = line_samples(rf)
    out = torch.empty(int(linecount) * ll, dtype=torch.int16, device=dev)
    run(rf, [descriptor(rf, ti.data_ptr(), ti.numel(), tl.data_ptr(), tl.numel(), lineoffset, linecount,
                        out.data_ptr(), delay)])
    res = out.cpu().numpy()
    tbc_status(rf)
    return res
