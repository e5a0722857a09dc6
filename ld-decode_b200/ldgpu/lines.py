"""Line locations of every field of a capture, batched on the GPU.

The reference decodes fields one by one (LDdecode.readfield ->
decodefield -> Field.process(), lddecode/core.py:4018-4186, 1636-1653):
each field's read position comes from the previous field's line
locations, and a few decisions (line 0's vote, the NTSC burst phase seed,
the processVBlank limit) use the previous field's results.  `LineLocator`
produces the same per-field results for a whole capture that is already
demodulated on the device:

1. ldg_sync_runs (GPU): every run of demod_05 at or below the sync
   threshold in the capture-wide array, with the mean level of long runs;
2. ldg_field_chain (native host code): the read chain and the pulse-level
   line locations of every field (linelocs1, bad lines, field parity);
3. ldg_lines_refine (GPU): H-sync refinement, NTSC colour-burst / PAL pilot
   refinement and bad-line repair of all fields -> final FP64 line
   locations on the device, ready for ldg_tbc_fields.

Where a field's pulse-level result depends on the previous field's refined
line locations (or needs the reference's level re-calibration), the chain
stops before it; that field is decoded by the host restatement
(ldgpu.linelocs) with the previous field's results, and the batch resumes
after it.  `host_field_chain` is the one-field-at-a-time form over host
arrays (the reference's own order of work).
"""

import ctypes
import math
import time

import numpy as np

from . import lib as L
from .fieldread import field_window, readlen_for

LDG_ERR_RANGE = -5


def _dtype_of(struct, formats):
    """numpy dtype with the exact layout of a ctypes structure."""
    names = [n for n, _ in struct._fields_]
    return np.dtype({"names": names, "formats": [formats[n] for n in names],
                     "offsets": [getattr(struct, n).offset for n in names], "itemsize": ctypes.sizeof(struct)})


_ML = L.LDG_CHAIN_MAX_LINES
PLAN_DTYPE = _dtype_of(L.FieldPlan, {
    "start": "f8", "readloc": "i8", "first_block": "i8", "nblocks": "i8", "startloc": "i8", "length": "i8",
    "valid": "i4", "isfirst": "i4", "linecount": "i4", "proclines": "i4", "has_prev": "i4",
    "sync_confidence": "i4", "hsync_len": "i4", "prev_range": "i4", "nextfieldoffset": "f8", "linelocs1": ("f8", (_ML,)),
    "linebad": ("u1", (_ML,))})
TBC_DTYPE = _dtype_of(L.TbcField, {
    "buf": "u8", "buf_len": "i8", "linelocs": "u8", "nlines": "i4", "lineoffset": "i4", "outwidth": "i4",
    "linesout": "i4", "outlinecount": "i4", "coord_f32": "i4", "inlinelen": "f8", "outlinelen": "f8",
    "ire0": "f8", "hz_ire": "f8", "vsync_ire": "f8", "out_scale": "f8", "output_zero": "f8",
    "out_f32": "u8", "out_u16": "u8", "wow_smoothing": "f8", "wow_interp": "i4", "pad1": "i4"})


def proclines_for(rf):
    """Lines compute_linelocs returns (core.py:2353-2356)."""
    outlinecount = rf.SysParams["frame_lines"] // 2 + 1
    return outlinecount + 10 + (3 if rf.system == "PAL" else 0)


def chain_params(rf, nblocks):
    sp = rf.SysParams
    dp = rf.DecoderParams
    p = L.ChainParams()
    p.system = L.LDG_PAL if rf.system == "PAL" else L.LDG_NTSC
    p.num_pulses = int(sp["numPulses"])
    p.field_lines[0], p.field_lines[1] = int(sp["field_lines"][0]), int(sp["field_lines"][1])
    p.outlinecount = sp["frame_lines"] // 2 + 1
    p.proclines = proclines_for(rf)
    p.freq = float(rf.freq)
    p.freq_hz = float(int(rf.freq_hz))
    p.linelen = float(rf.linelen)
    p.inlinelen = float(rf.linelen)
    p.linefreq0 = float(rf.samplesperline * rf.linelen)
    p.hsync_pulse_us = float(sp["hsyncPulseUS"])
    p.eq_pulse_us = float(sp["eqPulseUS"])
    p.vsync_pulse_us = float(sp["vsyncPulseUS"])
    p.first_field_h[0], p.first_field_h[1] = float(sp["firstFieldH"][0]), float(sp["firstFieldH"][1])
    p.hsync_tolerance = float(rf.hsync_tolerance)
    p.ire0, p.hz_ire, p.vsync_ire = float(dp["ire0"]), float(dp["hz_ire"]), float(dp["vsync_ire"])
    p.max_pulse_len = 5000
    p.blocklen = rf.blocklen
    p.blockcut = rf.blockcut
    p.blockcut_end = rf.blockcut_end
    p.readlen = readlen_for(rf)
    p.nblocks = int(nblocks)
    return p


def lines_consts(rf):
    k = L.LinesConsts()
    k.system = L.LDG_PAL if rf.system == "PAL" else L.LDG_NTSC
    k.freq = float(rf.freq)
    k.linelen = float(rf.linelen)
    k.linefreq0 = float(rf.samplesperline * rf.linelen)
    k.samplesperline = float(rf.samplesperline)
    k.half_sync = float(rf.iretohz(rf.DecoderParams["vsync_ire"] / 2))
    k.lo_ok = float(rf.iretohz(-55))
    k.hi_ok = float(rf.iretohz(30))
    k.hz_ire = float(rf.DecoderParams["hz_ire"])
    k.fsc_mhz = float(rf.SysParams["fsc_mhz"])
    k.pilot_mhz = float(rf.SysParams["pilot_mhz"])
    return k


def sync_threshold(rf):
    """getpulses' pulse_hz_max (core.py:2244)."""
    return float(rf.iretohz(-20))


def run_chain(rf, runs, nblocks, state=None, max_plans=4096, out=None):
    """ldg_field_chain over host run arrays; returns (plans, stop, state)
    with plans a numpy record array (PLAN_DTYPE, the ldg_field_plan layout).
    `out` is an optional reusable PLAN_DTYPE buffer."""
    lib = L.load()
    starts, lens, means = runs
    starts = np.ascontiguousarray(starts, dtype=np.int64)
    lens = np.ascontiguousarray(lens, dtype=np.int64)
    means = np.ascontiguousarray(means, dtype=np.float64)
    params = chain_params(rf, nblocks)
    st_in = state if state is not None else L.ChainState()
    st_out = L.ChainState()
    plans = out if out is not None and len(out) >= max_plans else np.empty(max_plans, PLAN_DTYPE)
    n = ctypes.c_int32(0)
    stop = ctypes.c_int32(0)
    rc = lib.ldg_field_chain(ctypes.byref(params), starts.ctypes.data, lens.ctypes.data, means.ctypes.data,
                             len(starts), ctypes.byref(st_in), ctypes.byref(st_out), plans.ctypes.data, max_plans,
                             ctypes.byref(n), ctypes.byref(stop))
    if rc != 0:
        raise L.LdgError(rc, lib.ldg_chain_last_error().decode())
    return plans[:n.value].view(np.recarray), stop.value, st_out


def parallel_chain(rf, runs, nblocks, state=None, nthreads=8, max_plans=4096, out=None, margin_blocks=None,
                   min_seg_blocks=None):
    """ldg_field_chain_mt: the chain in `nthreads` pieces on host threads,
    joined at common chain states (equal to one walk).  Margin and minimum
    piece default to 5 fields + one read window and 6 fields of blocks."""
    lib = L.load()
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    field_blocks = int(rf.freq_hz / rf.SysParams["FPS"] / 2 / U) + 1
    margin = margin_blocks if margin_blocks is not None else 5 * field_blocks + field_window(rf, 0.0).nblocks
    min_seg = min_seg_blocks if min_seg_blocks is not None else 6 * field_blocks
    starts, lens, means = (np.ascontiguousarray(a, dtype=d) for a, d in zip(runs, (np.int64, np.int64, np.float64)))
    params = chain_params(rf, nblocks)
    st_in = state if state is not None else L.ChainState()
    st_out = L.ChainState()
    plans = out if out is not None and len(out) >= max_plans else np.empty(max_plans, PLAN_DTYPE)
    n = ctypes.c_int32(0)
    stop = ctypes.c_int32(0)
    rc = lib.ldg_field_chain_mt(ctypes.byref(params), starts.ctypes.data, lens.ctypes.data, means.ctypes.data,
                                len(starts), ctypes.byref(st_in), ctypes.byref(st_out), plans.ctypes.data,
                                max_plans, ctypes.byref(n), ctypes.byref(stop), int(nthreads), int(margin),
                                int(min_seg))
    if rc != 0:
        raise L.LdgError(rc, lib.ldg_chain_last_error().decode())
    return plans[:n.value].view(np.recarray), stop.value, st_out


def field_levels(rf):
    """(ire0, hz_ire, vsync_ire, out_scale, outputZero) of Field.hz_to_output
    (FieldNTSC / FieldPAL out_scale, core.py:3355, 3058)."""
    dp = rf.DecoderParams
    if rf.system == "PAL":
        out_scale = np.double(0xD300 - 0x0100) / (100 - dp["vsync_ire"])
    else:
        out_scale = np.double(0xC800 - 0x0400) / (100 - dp["vsync_ire"])
    return (dp["ire0"], dp["hz_ire"], dp["vsync_ire"], out_scale, rf.SysParams["outputZero"])


def host_sync_runs(rf, d05):
    """Runs of a host demod_05 array (numpy), as ldg_sync_runs reports them;
    for checks of the chain on the CPU."""
    x = np.asarray(d05)
    below = x.astype(np.float64) <= sync_threshold(rf)
    d = np.diff(np.concatenate([[False], below]).astype(np.int8))
    st = np.nonzero(d == 1)[0]
    en = np.nonzero(d == -1)[0]
    n = min(len(st), len(en))
    st, en = st[:n], en[:n]
    lens = en - st
    minlen = math.floor(10 * rf.samplesperline * rf.linelen)
    lo, hi = math.floor(rf.freq), math.ceil(rf.freq)
    means = np.full(n, np.nan)
    for k in np.nonzero(lens > minlen)[0]:
        seg = x[st[k] + lo:st[k] + lens[k] - hi]
        if len(seg):
            means[k] = float(np.mean(seg, dtype=np.float64))
    return st.astype(np.int64), lens.astype(np.int64), means


def host_field_chain(rf, arrays, nblocks, start=0.0, prev=None, fields_written=0, max_fields=None):
    """The reference's order of work over host capture-wide arrays
    (core.py:4030-4097, 4165-4186): Field.process() for one field after
    another.  Returns [(window, FieldLogic), ...] for every field read
    (valid or not) and the next start."""
    from .linelocs import FieldLogicNTSC, FieldLogicPAL
    cls = FieldLogicPAL if rf.system == "PAL" else FieldLogicNTSC
    out = []
    while max_fields is None or len(out) < max_fields:
        w = field_window(rf, start)
        if w.first_block + w.nblocks > nblocks:
            break
        sl = slice(w.startloc, w.startloc + w.length)
        dec = {"video": {k: v[sl] for k, v in arrays.items()}, "startloc": w.startloc}
        f = cls(rf, dec, prevfield=prev, fields_written=fields_written, readloc=w.startloc)
        f.process()
        out.append((w, f))
        if not f.valid:
            start += f.nextfieldoffset
            prev = None
            continue
        start += f.nextfieldoffset - (w.readloc - w.startloc)
        fields_written += 1
        if prev is not None:
            prev.prevfield = None  # one field of history, as readfield keeps
        prev = f
    return out, start


class FieldLines:
    """Line locations of one field of a capture (device or host)."""

    def __init__(self, window, isfirst, linecount, lineoffset, linelocs_ptr=None, linelocs=None, nlines=0,
                 field_phase=None, phase_adjust=None, sync_confidence=100, rows=None, hsync_len=0, linebad=None,
                 bad_rows=None, pal_adjust=None):
        self.window = window
        self.hsync_len = int(hsync_len)    # int(Field.LT["hsync"][1])
        self.sync_confidence = int(sync_confidence)
        self.isFirstField = bool(isfirst)
        self.linecount = int(linecount)
        self.lineoffset = int(lineoffset)
        self.linelocs_ptr = linelocs_ptr   # device pointer of the FP64 line locations
        self.linelocs = linelocs           # host array (host-decoded fields) or None
        self.nlines = int(nlines)
        self._phase = field_phase          # int, or (device tensor, row)
        self._pam = phase_adjust           # float, or (device tensor, row)
        self._rows = rows                  # (device tensor, row) of a batched field
        self._linebad = linebad            # host bool array (host-decoded fields) or None
        self._bad_rows = bad_rows          # (device uint8 tensor, row) of a batched field
        self._pal_adjust = pal_adjust      # PAL: dict, or (device (n, 4) tensor, row)

    @staticmethod
    def _value(v, cast):
        if isinstance(v, tuple):
            t, i = v
            return cast(t[i].item())
        return None if v is None else cast(v)

    @property
    def fieldPhaseID(self):
        return self._value(self._phase, int)

    @property
    def phase_adjust_median(self):
        return self._value(self._pam, float)

    @property
    def pal_phase_adjust(self):
        """PAL: FieldPAL.phase_adjust, the burst phase adjusts of lines 7,
        11, 15 and 19 that the next field's determine_field_number seeds from
        (None where the line had none)."""
        v = self._pal_adjust
        if isinstance(v, tuple):
            t, i = v
            v = t[i].cpu().numpy()
            return {l: (None if np.isnan(x) else float(x)) for l, x in zip(range(7, 22, 4), v)}
        return v

    @property
    def linebad(self):
        """Field.linebad: the bad-line flags of the line locations (bool array)."""
        if self._linebad is not None:
            return np.asarray(self._linebad, dtype=bool)
        t, i = self._bad_rows
        return t[i].cpu().numpy()[:self.nlines].astype(bool)

    def host_linelocs(self):
        """The line locations as a host float64 array."""
        if self.linelocs is not None:
            return self.linelocs
        t, i = self._rows
        return t[i].cpu().numpy()[:self.nlines].copy()


class LocatedFields:
    """The valid fields of a capture in read order: as arrays (read window,
    parity, line counts, device pointers of the line locations) for the
    batched TBC, and as FieldLines objects by index."""

    def __init__(self, rf):
        self.rf = rf
        self._parts = []   # ("batch", plans, ll, pam, fph, bad) | ("host", FieldLines, device tensor)
        self._cache = None

    def __len__(self):
        return sum(len(p[1]) if p[0] == "batch" else 1 for p in self._parts)

    def arrays(self):
        """dict of per-field numpy arrays: startloc, length, readloc, isfirst,
        linecount, lineoffset, nlines, linelocs_ptr."""
        if self._cache is not None:
            return self._cache
        pal = self.rf.system == "PAL"
        keys = ("startloc", "length", "readloc", "isfirst", "linecount", "lineoffset", "nlines", "linelocs_ptr",
                "hsync_len")
        cols = {k: [] for k in keys}
        for part in self._parts:
            if part[0] == "batch":
                _, pl, ll, _, _, _ = part
                n = len(pl)
                isf = pl.isfirst.astype(bool)
                cols["startloc"].append(pl.startloc)
                cols["length"].append(pl.length)
                cols["readloc"].append(pl.readloc)
                cols["isfirst"].append(isf)
                if pal:
                    cols["linecount"].append(np.where(isf, 312, 313))
                    cols["lineoffset"].append(np.where(isf, 2, 3))
                else:
                    cols["linecount"].append(pl.linecount.astype(np.int64))
                    cols["lineoffset"].append(np.zeros(n, np.int64))
                cols["nlines"].append(np.full(n, proclines_for(self.rf)))
                cols["hsync_len"].append(pl.hsync_len.astype(np.int64))
                rowb = ll.stride(0) * ll.element_size()
                cols["linelocs_ptr"].append(np.uint64(ll.data_ptr()) + np.uint64(rowb) * np.arange(n, dtype=np.uint64))
            else:
                _, fl, dev = part
                w = fl.window
                cols["startloc"].append([w.startloc])
                cols["length"].append([w.length])
                cols["readloc"].append([w.readloc])
                cols["isfirst"].append([fl.isFirstField])
                cols["linecount"].append([fl.linecount])
                cols["lineoffset"].append([fl.lineoffset])
                cols["nlines"].append([fl.nlines])
                cols["hsync_len"].append([fl.hsync_len])
                cols["linelocs_ptr"].append(np.array([dev.data_ptr()], np.uint64))
        self._cache = {k: (np.concatenate([np.asarray(x) for x in v]) if v else np.zeros(0, np.int64))
                       for k, v in cols.items()}
        return self._cache

    def __getitem__(self, k):
        if k < 0:
            k += len(self)
        for part in self._parts:
            if part[0] == "host":
                if k == 0:
                    return part[1]
                k -= 1
                continue
            _, pl, ll, pam, fph, bad = part
            if k < len(pl):
                from .fieldread import FieldWindow
                p = pl[k]
                w = FieldWindow(int(p.readloc), int(p.first_block), int(p.nblocks), int(p.startloc), int(p.length))
                pal = self.rf.system == "PAL"
                rowb = ll.stride(0) * ll.element_size()
                return FieldLines(w, p.isfirst, (312 if p.isfirst else 313) if pal else p.linecount,
                                  (2 if p.isfirst else 3) if pal else 0, linelocs_ptr=ll.data_ptr() + k * rowb,
                                  nlines=proclines_for(self.rf), field_phase=(fph, k),
                                  phase_adjust=None if pal else (pam, k), sync_confidence=p.sync_confidence,
                                  rows=(ll, k), hsync_len=int(p.hsync_len), bad_rows=(bad, k),
                                  pal_adjust=(pam, k) if pal else None)
            k -= len(pl)
        raise IndexError("field index out of range")

    def __iter__(self):
        for k in range(len(self)):
            yield self[k]


def tbc_batch(rf, fields, demod_ptr, out_u16_ptr, levels, coord_f32=False, first=0, count=None,
              wow_interpolation_method="linear", wow_smoothing=0.0):
    """ldg_tbc_field descriptors for LocatedFields (or a list of FieldLines),
    fields [first, first + count): field i is written as uint16
    outlinelen x outlinecount at out_u16_ptr + i * field bytes; built as one
    numpy record array.  wow_interpolation_method / wow_smoothing are the
    Field options of the same names (core.py:1598, 2602-2613)."""
    outw = rf.SysParams["outlinelen"]
    outl = rf.SysParams["frame_lines"] // 2 + 1
    if isinstance(fields, LocatedFields):
        a = fields.arrays()
        startloc, length, ptr, nlines, lineoffset = (a["startloc"], a["length"], a["linelocs_ptr"], a["nlines"],
                                                     a["lineoffset"])
    else:
        startloc = np.array([f.window.startloc for f in fields], np.int64)
        length = np.array([f.window.length for f in fields], np.int64)
        ptr = np.array([f.linelocs_ptr if f.linelocs_ptr is not None else f.linelocs.ctypes.data for f in fields],
                       np.uint64)
        nlines = np.array([f.nlines for f in fields])
        lineoffset = np.array([f.lineoffset for f in fields])
    count = len(startloc) - first if count is None else count
    sel = slice(first, first + count)
    startloc, length, ptr, nlines, lineoffset = (np.asarray(x)[sel] for x in (startloc, length, ptr, nlines,
                                                                              lineoffset))
    n = len(startloc)
    d = np.zeros(n, TBC_DTYPE)
    d["buf"] = np.uint64(demod_ptr) + np.uint64(4) * startloc.astype(np.uint64)
    d["buf_len"] = length
    d["linelocs"] = ptr
    d["nlines"] = nlines
    d["lineoffset"] = lineoffset
    d["outwidth"] = outw
    d["linesout"] = outl
    d["outlinecount"] = outl
    d["coord_f32"] = 1 if coord_f32 else 0
    d["inlinelen"] = float(rf.linelen)
    d["outlinelen"] = float(outw)
    d["ire0"], d["hz_ire"], d["vsync_ire"], d["out_scale"], d["output_zero"] = [float(v) for v in levels]
    d["out_u16"] = np.uint64(out_u16_ptr) + np.uint64(2 * outw * outl) * np.arange(first, first + n,
                                                                                   dtype=np.uint64)
    d["wow_interp"] = L.WOW_METHODS[wow_interpolation_method]
    d["wow_smoothing"] = float(wow_smoothing or 0.0)
    return (L.TbcField * n).from_buffer_copy(d.tobytes()) if n else (L.TbcField * 0)()


def _lib_stream(stream):
    """Stream handle for the C ABI: torch's default stream (handle 0 or
    None) becomes cudaStreamLegacy (1), since a NULL handle would select the
    context's own stream, which is not ordered with torch's work."""
    return stream if stream else 1


class LineLocator:
    """Batched Field.process() for a demodulated capture on the device."""

    def __init__(self, rf):
        import torch
        self.rf = rf
        self.torch = torch
        self.proclines = proclines_for(rf)
        self.pal = rf.system == "PAL"
        self.stats = {"batched": 0, "host": 0, "invalid": 0, "segments": 0, "resolved": 0, "resolved_early": 0}
        self.timing = {}
        self._rbuf, self._nruns = None, 0  # the capture's sync runs (grown in place)
        self._plans = np.empty(4096, PLAN_DTYPE)
        self._runbufs = None
        self._keep = []
        self.ready = []
        self.chain_range = 128   # NTSC fields per burst-chain launch
        import os
        self.threads = max(1, min(16, os.cpu_count() or 1))

    def _pinned(self, nbytes):
        """A pinned host block from a ring of four; a block is reused once
        the copy that last read it has completed."""
        torch = self.torch
        if not hasattr(self, "_pin_ring"):
            self._pin_ring = [[None, None] for _ in range(4)]
            self._pin_next = 0
        slot = self._pin_ring[self._pin_next % 4]
        self._pin_next = self._pin_next % 4 + 1
        if slot[1] is not None:
            slot[1].synchronize()
        if slot[0] is None or slot[0].numel() < nbytes:
            slot[0] = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8).pin_memory()
        slot[1] = torch.cuda.Event()
        return slot[0][:nbytes]

    def _tick(self, key, t0):
        t = time.perf_counter()
        self.timing[key] = self.timing.get(key, 0.0) + (t - t0) * 1e3
        return t

    def sync_runs(self, d05_ptr, n, stream=None, cap=None):
        """ldg_sync_runs over a device array; host (starts, lens, means)."""
        lib = L.load()
        rf = self.rf
        cap = int(cap or max(1024, n // 256))
        if self._runbufs is None or len(self._runbufs[0]) < cap:
            torch = self.torch
            # pinned host buffers: the copies back run at full PCIe speed
            self._runbufs = [torch.empty(cap, dtype=torch.int64).pin_memory(),
                             torch.empty(cap, dtype=torch.int64).pin_memory(),
                             torch.empty(cap, dtype=torch.float64).pin_memory()]
        starts, lens, means = (t.numpy() for t in self._runbufs)
        nr = ctypes.c_int64(0)
        minlen = math.floor(10 * rf.samplesperline * rf.linelen)
        rc = lib.ldg_sync_runs(rf._ctx.handle, ctypes.c_void_p(d05_ptr), int(n), sync_threshold(rf), minlen,
                               math.floor(rf.freq), math.ceil(rf.freq), starts.ctypes.data, lens.ctypes.data,
                               means.ctypes.data, cap, ctypes.byref(nr), _lib_stream(stream))
        if rc == LDG_ERR_RANGE:
            return self.sync_runs(d05_ptr, n, stream, cap=int(nr.value) + 16)
        L.check(rc)
        k = nr.value
        return starts[:k], lens[:k], means[:k]

    def process_field(self, field):
        """Field.process() of one field read on the GPU (the drop-in classes'
        path, core.py:3212-3239 / 3471-3495): the field's own demodulated
        read goes to the device, the sync-run scan, the native field chain
        (one read, seeded from field.prevfield) and the GPU refinement give
        its line locations, flags and field phase ID.  Returns False, with
        `field` untouched, when the read needs what only the host
        restatement does (the previous field's refined line locations, the
        reference's level re-calibration, or a read shorter than a field
        window); the caller then runs FieldLogic.process()."""
        torch = self.torch
        rf = self.rf
        v = field.data["video"]
        keys = self._keys()
        n = len(v["demod_05"])
        U = rf.blocklen - rf.blockcut - rf.blockcut_end
        nblocks = n // U
        dev = torch.device("cuda", torch.cuda.current_device())
        arrays = {k: torch.from_numpy(np.ascontiguousarray(v[k], dtype=np.float32)).to(dev) for k in keys}
        self.begin(arrays)
        runs = self.sync_runs(arrays["demod_05"].data_ptr(), n)
        prev = field.prevfield if getattr(field.prevfield, "valid", False) else None
        st = L.ChainState()
        st.start = float(rf.blockcut)  # the read window at the first block of the data
        st.prev_valid = 1 if prev is not None else 0
        st.prev_isfirst = int(bool(prev.isFirstField)) if prev is not None else 0
        st.fields_written = int(field.fields_written)
        plans, stop, _ = run_chain(rf, runs, nblocks, st, max_plans=1)
        if len(plans) == 0 and stop == L.LDG_CHAIN_STOP_PREV and prev is not None:
            # getLine0's inputs from the previous field (skip_check, line0loc_prev)
            st.prev_known = 1
            st.prev_skip = 1 if prev.skip_check() >= 50 else 0
            st.prev_line0 = st.prev_line0_hi = float(np.asarray(prev.linelocs, dtype=np.float64)[prev.linecount]
                                                     - (field.data["startloc"] - prev.data["startloc"]))
            st.prev_conf = int(prev.sync_confidence)
            plans, stop, _ = run_chain(rf, runs, nblocks, st, max_plans=1)
        if len(plans) == 0:
            return False
        p = plans[0]
        if not p.valid:
            field.valid = False
            field.nextfieldoffset = float(p.nextfieldoffset)
            return True
        valid = plans[:1].copy().view(np.recarray)
        pam_host = 0.0
        if self.pal:
            pa = (getattr(prev, "phase_adjust", None) or {}) if prev is not None else {}
            adj = [float("nan") if pa.get(l) is None else float(pa[l]) for l in range(7, 22, 4)]
            self._pal_seed = ("host", adj, int(prev.fieldPhaseID) if prev is not None else 0)
        elif prev is not None:
            pam_host = float(prev.phase_adjust_median)
        ll2 = None if self.pal else torch.empty((1, L.LDG_CHAIN_MAX_LINES), dtype=torch.float64, device=dev)
        ll, bad, pam, fph, _ = self._refine(self._ptrs, n, valid, pam_host, None, linelocs2=ll2)
        torch.cuda.synchronize()
        nl = self.proclines
        field.linelocs1 = np.array(p.linelocs1[:nl], dtype=np.float64)
        field.linebad = bad[0].cpu().numpy()[:nl].astype(bool)
        field.isFirstField = bool(p.isfirst)
        field.sync_confidence = int(p.sync_confidence)
        field.nextfieldoffset = float(p.nextfieldoffset)
        field.LT = {"hsync": (None, int(p.hsync_len))}
        field.fieldPhaseID = int(fph[0].item())
        field.valid = True
        final = ll[0].cpu().numpy()[:nl].copy()
        if self.pal:
            field.linelocs = final
            field.linecount, field.lineoffset = 263 if field.isFirstField else 262, 0
            field.burstmedian = field.calc_burstmedian()  # before the PAL line count and offset, as the reference
            field.linecount = 312 if field.isFirstField else 313
            field.lineoffset = 2 if field.isFirstField else 3
            field.linecode = [field.decodephillipscode(l + field.lineoffset) for l in (16, 17, 18)]
            adj = pam[0].cpu().numpy()
            field.phase_adjust = {l: (None if np.isnan(x) else float(x)) for l, x in zip(range(7, 22, 4), adj)}
        else:
            field.linecount = int(p.linecount)
            field.lineoffset = 0
            field.linelocs2 = ll2[0].cpu().numpy()[:nl].copy()
            field.linelocs = field.linelocs2  # linecode and the burst median read the H-sync line locations
            field.linecode = [field.decodephillipscode(l + field.lineoffset) for l in (16, 17, 18)]
            field.burstmedian = field.calc_burstmedian()
            field.phase_adjust_median = float(pam[0].item())
            field.linelocs = final
        return True

    def _refine(self, arrays, capture_len, plans, prev_pam, stream, prev_pam_dev=None, linelocs2=None):
        """ldg_lines_refine over valid plans (record array); device tensors.
        The NTSC burst seed of the first field is `prev_pam`, or the device
        double at `prev_pam_dev` when given (read in stream order)."""
        torch = self.torch
        lib = L.load()
        nf = len(plans)
        dev = torch.device("cuda", torch.cuda.current_device())
        ml = L.LDG_CHAIN_MAX_LINES
        # every per-field input in one pinned host block, one copy to the device
        nb_i = 2 * nf * 8 + 3 * nf * 4
        nb_i = (nb_i + 7) // 8 * 8
        total = nb_i + nf * ml * 8 + nf * ml
        hbuf = self._pinned(total)
        hb = hbuf.numpy()
        i64 = hb[:2 * nf * 8].view(np.int64).reshape(2, nf)
        i64[0] = plans.startloc
        i64[1] = plans.length
        i32 = hb[2 * nf * 8:2 * nf * 8 + 3 * nf * 4].view(np.int32).reshape(3, nf)
        i32[0] = plans.isfirst
        i32[1] = plans.linecount
        i32[2] = plans.has_prev
        hb[nb_i:nb_i + nf * ml * 8].view(np.float64).reshape(nf, ml)[:] = plans.linelocs1
        hb[nb_i + nf * ml * 8:].reshape(nf, ml)[:] = plans.linebad
        dbuf = torch.empty(total, dtype=torch.uint8, device=dev)
        # copied by SMs from the pinned block: a copy-engine transfer would
        # wait behind any bulk copies queued on the engines
        L.check(lib.ldg_copy_async(dbuf.data_ptr(), hbuf.data_ptr(), total, _lib_stream(stream)))
        self._pin_ring[self._pin_next - 1][1].record()
        base = dbuf.data_ptr()
        out_ll = torch.empty((nf, ml), dtype=torch.float64, device=dev)
        out_bad = torch.empty((nf, ml), dtype=torch.uint8, device=dev)
        # NTSC: phase_adjust_median per field; PAL: the line 7/11/15/19 burst phase adjusts
        pam = torch.zeros((nf, 4) if self.pal else nf, dtype=torch.float64, device=dev)
        fph = torch.zeros(nf, dtype=torch.int32, device=dev)
        scratch = torch.empty(max(int(lib.ldg_lines_scratch_bytes(nf)), 256), dtype=torch.uint8, device=dev)
        self._last_scratch = (scratch, nf)  # the last batch's work arrays (inspection)
        a = L.LinesArgs()
        a.k = lines_consts(self.rf)
        a.d05 = arrays["demod_05"]
        a.demod = arrays.get("demod")
        a.burst = arrays.get("demod_burst")
        a.pilot = arrays.get("demod_pilot")
        a.capture_len = int(capture_len)
        a.nfields = nf
        a.proclines = self.proclines
        a.startloc = base
        a.wlen = base + nf * 8
        a.isfirst = base + 2 * nf * 8
        a.linecount = base + 2 * nf * 8 + nf * 4
        a.has_prev = base + 2 * nf * 8 + 2 * nf * 4
        a.linelocs1 = base + nb_i
        a.linebad1 = base + nb_i + nf * ml * 8
        if self.pal:
            # the previous field's line phases and ID: host values or device copies
            kind, adj, fid = self._pal_seed
            if kind == "host":
                for j in range(4):
                    a.prev_pal_adjust[j] = adj[j]
                a.prev_field_phase = int(fid)
            else:
                a.prev_pal_adjust_dev = adj
                a.prev_field_phase_dev = fid
        else:
            a.prev_phase_adjust = float(prev_pam)
            a.prev_phase_adjust_dev = prev_pam_dev
        a.linelocs = out_ll.data_ptr()
        a.linebad = out_bad.data_ptr()
        a.phase_adjust = pam.data_ptr()
        a.field_phase = fph.data_ptr()
        a.scratch = scratch.data_ptr()
        a.stream = _lib_stream(stream)
        if linelocs2 is not None:
            a.linelocs2 = linelocs2.data_ptr()
        ts = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
        ready = []
        if self.pal:
            L.check(lib.ldg_lines_refine(self.rf._ctx.handle, ctypes.byref(a)))
            ev = torch.cuda.Event()
            ev.record(ts)
            ready.append((0, nf, ev))
        else:
            # H-sync of every field, then the burst chain range by range: each
            # finished range can go on (TBC) while the chain walks the next
            a.stages = 1
            L.check(lib.ldg_lines_refine(self.rf._ctx.handle, ctypes.byref(a)))
            for lo in range(0, nf, self.chain_range):
                a.first_field = lo
                a.count = min(self.chain_range, nf - lo)
                a.stages = 6
                L.check(lib.ldg_lines_refine(self.rf._ctx.handle, ctypes.byref(a)))
                ev = torch.cuda.Event()
                ev.record(ts)
                ready.append((lo, lo + a.count, ev))
        # device inputs and scratch return to the caching allocator on the
        # stream the kernels run on, so any reuse is ordered after them
        self._keep.append((hbuf, dbuf, scratch))
        return out_ll, out_bad, pam, fph, ready

    def locate(self, arrays, nblocks, stream=None, force_host=()):
        """Line locations of every field.  `arrays` maps output names
        (demod, demod_05, demod_burst[, demod_pilot]) to capture-wide float32
        device tensors of equal length; `stream` as for `advance`.  Returns a LocatedFields of the
        valid fields in read order; `self.stats` counts batched,
        host-decoded and invalid reads and `self.timing` the host time of
        each phase (ms).  `force_host` lists read indices to decode with the
        host restatement (checks of the resume path)."""
        self.begin(arrays)
        self.advance(nblocks, stream, force_host)
        return self.fields

    def begin(self, arrays):
        """Start a capture whose outputs are (or will be) in `arrays`; the
        fields come out as `advance` is told how many blocks are done."""
        self._arrays = arrays
        self._ptrs = {k: v.data_ptr() for k, v in arrays.items()}
        self._cap_len = int(arrays["demod_05"].numel())
        self._runs = (np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.float64))
        self._scan_lo = 0
        self._state = L.ChainState()
        self._pam = ("host", 0.0)       # NTSC burst seed for the next batched field
        self._pal_seed = ("host", [float("nan")] * 4, 0)  # PAL: the previous field's line phases and ID
        self._prev_host = None          # the previous field, if it was host-decoded
        self._last_dev = None           # index of the last batched field
        self._last_ready = None         # event: its line locations are final
        self._ire0 = float(self.rf.DecoderParams["ire0"])
        self._reads = 0
        self._keep = []
        self.fields = LocatedFields(self.rf)
        # (first, end, event): fields whose line locations are final once the
        # event has completed, in order
        self.ready = []

    def _scan(self, hi, stream):
        """Sync runs of demod_05 over [scan position, hi), appended."""
        lo = self._scan_lo
        if hi - lo < 2:
            return
        st, ln, mn = self.sync_runs(self._ptrs["demod_05"] + 4 * lo, hi - lo, stream)
        if len(st):
            st = st + lo
            # the next scan restarts after the last complete run: what follows
            # is above the threshold or the start of a run still open at hi
            self._scan_lo = int(st[-1] + ln[-1])
            self._append_runs(st, ln, mn)

    def _append_runs(self, st, ln, mn):
        """Append to the capture's run list in place (capacity doubling, so a
        scan per chunk does not copy every earlier run again)."""
        n0, k = self._nruns, len(st)
        if self._rbuf is None or n0 + k > len(self._rbuf[0]):
            cap = max(2 * (n0 + k), 4096)
            nb = (np.empty(cap, np.int64), np.empty(cap, np.int64), np.empty(cap, np.float64))
            if self._rbuf is not None:
                for dst, src in zip(nb, self._rbuf):
                    dst[:n0] = src[:n0]
            self._rbuf = nb
        for dst, src in zip(self._rbuf, (st, ln, mn)):
            dst[n0:n0 + k] = src
        self._nruns = n0 + k

    @property
    def _runs(self):
        if self._rbuf is None:
            return (np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.float64))
        return tuple(a[:self._nruns] for a in self._rbuf)

    @_runs.setter
    def _runs(self, runs):
        self._rbuf, self._nruns = None, 0
        if len(runs[0]):
            self._append_runs(*runs)

    def advance(self, nblocks, stream=None, force_host=(), scan_stream=None):
        """Fields whose read windows lie within the first `nblocks` blocks
        (demodulated and complete in stream order on `stream`): scans the
        new samples, walks the chain, refines on the GPU.  `stream` is a
        torch.cuda.Stream (device work and allocations are ordered on it) or
        None for torch's current stream.  The sync-run scan runs on `scan_stream` when given (so it need
        not queue behind earlier refinement work on `stream`).  Returns the
        range of new indices into `self.fields`."""
        raw_scan = scan_stream.cuda_stream if isinstance(scan_stream, self.torch.cuda.Stream) else scan_stream
        if stream is None:
            stream = self.torch.cuda.current_stream()
        if isinstance(stream, self.torch.cuda.Stream):
            with self.torch.cuda.stream(stream):
                return self._advance(nblocks, stream.cuda_stream, force_host,
                                     raw_scan if scan_stream is not None else stream.cuda_stream)
        return self._advance(nblocks, stream, force_host, raw_scan if scan_stream is not None else stream)

    def _advance(self, nblocks, stream, force_host, scan_stream):
        rf = self.rf
        torch = self.torch
        U = rf.blocklen - rf.blockcut - rf.blockcut_end
        first_new = len(self.fields)
        t = time.perf_counter()
        self._scan(min(nblocks * U, self._cap_len), scan_stream)
        t = self._tick("sync_runs", t)
        out = self.fields
        arrays, ptrs = self._arrays, self._ptrs
        state = self._state
        while True:
            plans, stop, st_out = parallel_chain(rf, self._runs, nblocks, state, self.threads, out=self._plans)
            t = self._tick("chain", t)
            # a forced host decode cuts the segment at that read index
            cut = None
            for i in range(len(plans)):
                if self._reads + i in force_host:
                    cut = i
                    break
            if cut is not None:
                plans = plans[:cut]
                stop = L.LDG_CHAIN_STOP_PREV
                st_out = self._state_after(plans, state)
            self._segment(plans, stream)
            t = self._tick("refine", t)
            state = st_out
            if stop in (L.LDG_CHAIN_STOP_END, L.LDG_CHAIN_STOP_FULL):
                if stop == L.LDG_CHAIN_STOP_FULL:
                    continue
                break
            w = field_window(rf, state.start)
            if w.first_block + w.nblocks > nblocks:
                break
            # a field whose line 0 needs the previous field's refined line
            # locations and that the chain could not decide from the range of
            # their pulse-level estimate: wait for them, hand them to the
            # chain (skip_check, line0loc_prev) and let it go on; the host
            # restatement only for what remains
            if stop == L.LDG_CHAIN_STOP_PREV and cut is None and state.prev_valid and self._prev_inputs(state, w):
                one, stop1, st1 = run_chain(rf, self._runs, nblocks, state, max_plans=1)
                t = self._tick("chain", t)
                if len(one):
                    self.stats["resolved"] += 1
                    self._segment(one, stream)
                    t = self._tick("refine", t)
                    state = st1
                    continue
                state.prev_known = 0
            # decode the next field on the host, with the previous field's results
            prevfield = None
            if state.prev_valid:
                if self._prev_host is not None:
                    prevfield = self._prev_host
                else:
                    fl = out[self._last_dev]
                    prevfield = self._proxy(arrays, fl, fl.phase_adjust_median if not self.pal else 0.0)
            f = self._host_field(arrays, w, prevfield, state.fields_written)
            self._reads += 1
            self.stats["host"] += 1
            if not f.valid:
                self.stats["invalid"] += 1
                state.start += f.nextfieldoffset
                state.prev_valid = 0
                state.prev_est_valid = 0
                self._prev_host = None
                self._pam = ("host", 0.0)
                self._pal_seed = ("host", [float("nan")] * 4, 0)
                t = self._tick("host_fields", t)
                continue
            ll_host = np.ascontiguousarray(f.linelocs, dtype=np.float64)
            fl = FieldLines(w, f.isFirstField, f.linecount, f.lineoffset, linelocs=ll_host, nlines=len(ll_host),
                            field_phase=getattr(f, "fieldPhaseID", None),
                            phase_adjust=getattr(f, "phase_adjust_median", None),
                            sync_confidence=f.sync_confidence, hsync_len=int(f.LT["hsync"][1]),
                            linebad=np.asarray(f.linebad, dtype=bool),
                            pal_adjust=dict(getattr(f, "phase_adjust", None) or {}) if self.pal else None)
            dev_ll = torch.from_numpy(ll_host).to(torch.device("cuda", torch.cuda.current_device()))
            fl.linelocs_ptr = dev_ll.data_ptr()
            out._parts.append(("host", fl, dev_ll))
            out._cache = None
            ev = torch.cuda.Event()
            ev.record()
            self.ready.append((len(out) - 1, len(out), ev))
            state.start += f.nextfieldoffset - (w.readloc - w.startloc)
            state.prev_valid = 1
            state.prev_isfirst = int(bool(f.isFirstField))
            state.prev_startloc = w.startloc
            state.fields_written += 1
            state.prev_est = float(w.startloc + ll_host[f.linecount])
            state.prev_est_valid = 1
            state.prev_est_conf = int(f.sync_confidence)
            self._prev_host = f
            self._pam = ("host", float(f.phase_adjust_median) if not self.pal else 0.0)
            if self.pal:
                pa = getattr(f, "phase_adjust", None) or {}
                adj = [float("nan") if pa.get(l) is None else float(pa[l]) for l in range(7, 22, 4)]
                self._pal_seed = ("host", adj, int(f.fieldPhaseID))
            if float(rf.DecoderParams["ire0"]) != self._ire0:
                # the level re-calibration changed the sync threshold: rescan
                self._ire0 = float(rf.DecoderParams["ire0"])
                self._scan_lo = 0
                self._runs = (np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.float64))
                self._scan(min(nblocks * U, self._cap_len), scan_stream)
            t = self._tick("host_fields", t)
        self._state = state
        return first_new, len(out)

    def _segment(self, plans, stream):
        """Refine the valid fields of a run of chain plans as one batch on
        the GPU, seeded from the field before them."""
        out = self.fields
        valid = plans[plans.valid != 0].copy().view(np.recarray)
        self.stats["invalid"] += len(plans) - len(valid)
        self._reads += len(plans)
        if not len(valid):
            return
        self.stats["segments"] += 1
        self.stats["batched"] += len(valid)
        self.stats["resolved_early"] += int(np.count_nonzero(valid.prev_range))
        pam_host, pam_dev = 0.0, None
        if not self.pal and valid.has_prev[0]:
            if self._pam[0] == "host":
                pam_host = self._pam[1]
            else:
                pam_dev = self._pam[1]
        base = len(out)
        ll, bad, pam, fph, ready = self._refine(self._ptrs, self._cap_len, valid, pam_host, stream, pam_dev)
        self.ready.extend((base + lo, base + hi, ev) for lo, hi, ev in ready)
        self._last_ready = ready[-1][2]
        out._parts.append(("batch", valid, ll, pam, fph, bad))
        out._cache = None
        self._last_dev = len(out) - 1
        self._prev_host = None
        if not self.pal:
            self._pam = ("dev", pam.data_ptr() + 8 * (len(valid) - 1))
        else:
            self._pal_seed = ("dev", pam.data_ptr() + 32 * (len(valid) - 1), fph.data_ptr() + 4 * (len(valid) - 1))
        self._keep.append((pam, fph))

    def _prev_inputs(self, state, w):
        """Fill state's previous-field inputs of getLine0 exactly from the
        last located field (skip_check() >= 50, line0loc_prev, sync
        confidence; for a batched field after waiting for its refinement).
        False when there is none."""
        if self._prev_host is not None:
            prev = self._prev_host
            ll = np.asarray(prev.linelocs, dtype=np.float64)
            skip = prev.skip_check()
            lc, conf, prev_start = prev.linecount, prev.sync_confidence, prev.data["startloc"]
        elif self._last_dev is not None:
            self._last_ready.synchronize()
            fl = self.fields[self._last_dev]
            ll = fl.host_linelocs()
            skip = self._proxy(self._arrays, fl, 0.0).skip_check()
            lc, conf, prev_start = fl.linecount, fl.sync_confidence, fl.window.startloc
        else:
            return False
        state.prev_known = 1
        state.prev_skip = 1 if skip >= 50 else 0
        state.prev_line0 = state.prev_line0_hi = float(ll[lc] - (w.startloc - prev_start))
        state.prev_conf = int(conf)
        return True

    def _state_after(self, plans, state):
        """Chain state after the given plans (for a forced cut)."""
        st = L.ChainState()
        ctypes.memmove(ctypes.byref(st), ctypes.byref(state), ctypes.sizeof(st))
        for p in plans:
            st.prev_known = 0
            if not p.valid:
                st.start += p.nextfieldoffset
                st.prev_valid = 0
                st.prev_est_valid = 0
                continue
            st.start += p.nextfieldoffset - (p.readloc - p.startloc)
            st.prev_valid = 1
            st.prev_isfirst = p.isfirst
            st.prev_startloc = p.startloc
            st.fields_written += 1
            lc = (312 if p.isfirst else 313) if self.pal else int(p.linecount)
            st.prev_est = float(p.startloc + p.linelocs1[lc])
            st.prev_est_valid = 1
            st.prev_est_conf = int(p.sync_confidence)
        return st

    def _window_host(self, arrays, w, keys):
        return {k: arrays[k][w.startloc:w.startloc + w.length].cpu().numpy() for k in keys if k in arrays}

    def _keys(self):
        # PAL's determine_field_number reads demod_burst too
        return ("demod", "demod_05", "demod_burst", "demod_pilot") if self.pal else ("demod", "demod_05", "demod_burst")

    def _host_field(self, arrays, w, prevfield, fields_written):
        from .linelocs import FieldLogicNTSC, FieldLogicPAL
        cls = FieldLogicPAL if self.pal else FieldLogicNTSC
        dec = {"video": self._window_host(arrays, w, self._keys()), "startloc": w.startloc}
        f = cls(self.rf, dec, prevfield=prevfield, fields_written=fields_written, readloc=w.startloc)
        f.process()
        return f

    def _proxy(self, arrays, fl, pam):
        """The previous (batched) field as a FieldLogic object with the
        attributes the next field's process() reads."""
        from .linelocs import FieldLogicNTSC, FieldLogicPAL
        cls = FieldLogicPAL if self.pal else FieldLogicNTSC
        dec = {"video": self._window_host(arrays, fl.window, ("demod",)), "startloc": fl.window.startloc}
        p = cls(self.rf, dec)
        p.valid = True
        p.linelocs = fl.host_linelocs()
        p.linecount = fl.linecount
        p.lineoffset = fl.lineoffset
        p.isFirstField = fl.isFirstField
        p.sync_confidence = fl.sync_confidence
        p.phase_adjust_median = pam if not self.pal else 0
        p.fieldPhaseID = fl.fieldPhaseID if fl.fieldPhaseID is not None else 1
        if self.pal:
            p.phase_adjust = fl.pal_phase_adjust or {}
        return p
