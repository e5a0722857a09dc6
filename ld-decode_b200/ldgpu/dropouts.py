"""Dropout detection on the GPU (ldg_dropouts): Field.dropout_detect
(lddecode/core.py:2829-2983) for one field or every located field of a
capture in one launch.

Results are the reference's: per field the lists (fieldLine, startx, endx)
that LDdecode writes as the field's dropOuts (core.py:4535-4542).  A field
whose error samples exceed `err_cap`, or whose dropouts exceed `out_cap`,
raises LdgError (raise the caps); so does a field the reference itself
could not process (a vertical-sync line past its line locations)."""

import ctypes

import numpy as np

from . import lib as L

ERR_CAP = 1 << 18
OUT_CAP = 4096


def dropout_params(rf, err_cap=ERR_CAP, out_cap=OUT_CAP):
    p = L.DropoutParams()
    p.system = L.LDG_PAL if rf.system == "PAL" else L.LDG_NTSC
    p.video_rot = int(rf.delays["video_rot"])
    p.outlinelen = int(rf.SysParams["outlinelen"])
    p.err_cap = int(err_cap)
    p.out_cap = int(out_cap)
    p.freq_mhz = float(rf.freq)
    p.freq_hz_half = float(rf.freq_hz_half)
    p.ire0 = float(rf.DecoderParams["ire0"])
    p.hz_ire = float(rf.DecoderParams["hz_ire"])
    p.vsync_ire = float(rf.SysParams["vsync_ire"])
    return p


def _field(demod, d05, raw, rfhpf, n, ll_ptr, nlines, lineoffset, linecount, isfirst, hsync_len):
    d = L.DropoutField()
    d.demod, d.demod_05, d.demod_raw, d.rfhpf = demod, d05, raw, rfhpf
    d.len = int(n)
    d.linelocs = ll_ptr
    d.nlines = int(nlines)
    d.lineoffset = int(lineoffset)
    d.linecount = int(linecount)
    d.isfirst = int(bool(isfirst))
    d.hsync_len = int(hsync_len)
    return d


def run(rf, descs, stream=None, err_cap=ERR_CAP, out_cap=OUT_CAP, rfstd=False):
    """ldg_dropouts over a list of DropoutField; waits and returns the
    per-field (lines, starts, ends) lists (and the rfhpf standard
    deviations when rfstd=True)."""
    import torch
    n = len(descs)
    if n == 0:
        return ([], []) if rfstd else []
    dev = torch.device("cuda", torch.cuda.current_device())
    drops = torch.empty(n * out_cap * 3, dtype=torch.int32, device=dev)
    counts = torch.empty(2 * n, dtype=torch.int32, device=dev)
    sd = torch.empty(n, dtype=torch.float64, device=dev)
    arr = (L.DropoutField * n)(*descs)
    p = dropout_params(rf, err_cap, out_cap)
    h = stream if stream else 1  # torch's default stream (cudaStreamLegacy)
    L.check(rf._ctx._lib.ldg_dropouts(rf._ctx.handle, ctypes.byref(p), arr, n, drops.data_ptr(), counts.data_ptr(),
                                      sd.data_ptr(), h))
    c = counts.cpu().numpy().reshape(n, 2)
    bad = np.nonzero((c[:, 0] < 0) | (c[:, 1] < 0))[0]
    if len(bad):
        code = int(c[bad[0], 0])
        why = {-1: f"more than {out_cap} dropouts", -2: "line locations out of order",
               -3: "a vertical-sync line past the line locations"}.get(code, str(code))
        if c[bad[0], 1] < 0:
            why = f"more than {err_cap} error samples"
        raise L.LdgError(L.LDG_ERR_RANGE, f"dropout detection, field {int(bad[0])}: {why}")
    d = drops.cpu().numpy().reshape(n, out_cap, 3)
    out = []
    for i in range(n):
        k = int(c[i, 0])
        rows = d[i, :k]
        out.append((rows[:, 0].tolist(), rows[:, 1].tolist(), rows[:, 2].tolist()))
    if rfstd:
        return out, sd.cpu().numpy()
    return out


def detect_located(rf, fields, arrays, stream=None, first=0, count=None, **kw):
    """Dropouts of LocatedFields [first, first + count) of a capture whose
    capture-wide device outputs are `arrays` (demod, demod_05, demod_raw,
    rfhpf)."""
    a = fields.arrays()
    count = len(a["startloc"]) - first if count is None else count
    base = {k: arrays[k].data_ptr() for k in ("demod", "demod_05", "demod_raw", "rfhpf")}
    descs = []
    for i in range(first, first + count):
        o = 4 * int(a["startloc"][i])
        descs.append(_field(base["demod"] + o, base["demod_05"] + o, base["demod_raw"] + o, base["rfhpf"] + o,
                            a["length"][i], int(a["linelocs_ptr"][i]), a["nlines"][i], a["lineoffset"][i],
                            a["linecount"][i], a["isfirst"][i], a["hsync_len"][i]))
    return run(rf, descs, stream, **kw)


def detect_host_field(rf, data, linelocs, lineoffset, linecount, isfirst, hsync_len, **kw):
    """One field whose read is host numpy (the reference's Field.data:
    video recarray and rfhpf): uploads it and runs the kernel."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    v = data["video"]
    t = {k: torch.from_numpy(np.ascontiguousarray(v[k], np.float32)).to(dev)
         for k in ("demod", "demod_05", "demod_raw")}
    t["rfhpf"] = torch.from_numpy(np.ascontiguousarray(data["rfhpf"], np.float32)).to(dev)
    ll = torch.from_numpy(np.ascontiguousarray(linelocs, np.float64)).to(dev)
    d = _field(t["demod"].data_ptr(), t["demod_05"].data_ptr(), t["demod_raw"].data_ptr(), t["rfhpf"].data_ptr(),
               t["demod"].numel(), ll.data_ptr(), ll.numel(), lineoffset, linecount, isfirst, hsync_len)
    return run(rf, [d], **kw)[0]
