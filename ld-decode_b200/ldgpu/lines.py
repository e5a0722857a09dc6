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

import numpy as np

from . import lib as L
from .fieldread import field_window, readlen_for

LDG_ERR_RANGE = -5


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


def run_chain(rf, runs, nblocks, state=None, max_plans=4096):
    """ldg_field_chain over host run arrays; returns (plans, stop, state)."""
    lib = L.load()
    starts, lens, means = runs
    starts = np.ascontiguousarray(starts, dtype=np.int64)
    lens = np.ascontiguousarray(lens, dtype=np.int64)
    means = np.ascontiguousarray(means, dtype=np.float64)
    params = chain_params(rf, nblocks)
    st_in = state if state is not None else L.ChainState()
    st_out = L.ChainState()
    plans = (L.FieldPlan * max_plans)()
    n = ctypes.c_int32(0)
    stop = ctypes.c_int32(0)
    rc = lib.ldg_field_chain(ctypes.byref(params), starts.ctypes.data, lens.ctypes.data, means.ctypes.data,
                             len(starts), ctypes.byref(st_in), ctypes.byref(st_out), plans, max_plans,
                             ctypes.byref(n), ctypes.byref(stop))
    if rc != 0:
        raise L.LdgError(rc, lib.ldg_chain_last_error().decode())
    return [plans[i] for i in range(n.value)], stop.value, st_out


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
                 field_phase=None, phase_adjust=None, sync_confidence=100):
        self.window = window
        self.sync_confidence = int(sync_confidence)
        self.isFirstField = bool(isfirst)
        self.linecount = int(linecount)
        self.lineoffset = int(lineoffset)
        self.linelocs_ptr = linelocs_ptr   # device pointer (GPU batch) or None
        self.linelocs = linelocs           # host array (host-decoded fields) or None
        self.nlines = int(nlines)
        self.fieldPhaseID = field_phase
        self.phase_adjust_median = phase_adjust


class LineLocator:
    """Batched Field.process() for a demodulated capture on the device."""

    def __init__(self, rf):
        import torch
        self.rf = rf
        self.torch = torch
        self.proclines = proclines_for(rf)
        self.pal = rf.system == "PAL"
        self._bufs = []
        self.stats = {"batched": 0, "host": 0, "invalid": 0, "segments": 0}

    def sync_runs(self, d05_ptr, n, stream=None, cap=None):
        """ldg_sync_runs over a device array; host (starts, lens, means)."""
        lib = L.load()
        rf = self.rf
        cap = int(cap or max(1024, n // 256))
        starts = np.empty(cap, np.int64)
        lens = np.empty(cap, np.int64)
        means = np.empty(cap, np.float64)
        nr = ctypes.c_int64(0)
        minlen = math.floor(10 * rf.samplesperline * rf.linelen)
        rc = lib.ldg_sync_runs(rf._ctx.handle, ctypes.c_void_p(d05_ptr), int(n), sync_threshold(rf), minlen,
                               math.floor(rf.freq), math.ceil(rf.freq), starts.ctypes.data, lens.ctypes.data,
                               means.ctypes.data, cap, ctypes.byref(nr), stream)
        if rc == LDG_ERR_RANGE:
            return self.sync_runs(d05_ptr, n, stream, cap=int(nr.value) + 16)
        L.check(rc)
        k = nr.value
        return starts[:k], lens[:k], means[:k]

    def _refine(self, arrays, capture_len, plans, prev_pam, stream):
        """ldg_lines_refine over valid plans; returns device tensors."""
        torch = self.torch
        lib = L.load()
        nf = len(plans)
        dev = torch.device("cuda", torch.cuda.current_device())
        maxl = L.LDG_CHAIN_MAX_LINES
        startloc = torch.tensor([p.startloc for p in plans], dtype=torch.int64)
        wlen = torch.tensor([p.length for p in plans], dtype=torch.int64)
        isfirst = torch.tensor([p.isfirst for p in plans], dtype=torch.int32)
        linecount = torch.tensor([p.linecount for p in plans], dtype=torch.int32)
        has_prev = torch.tensor([p.has_prev for p in plans], dtype=torch.int32)
        ll1 = np.empty((nf, maxl), np.float64)
        bad1 = np.empty((nf, maxl), np.uint8)
        for i, p in enumerate(plans):
            ll1[i] = np.frombuffer(p.linelocs1, dtype=np.float64)
            bad1[i] = np.frombuffer(p.linebad, dtype=np.uint8)
        host = [startloc, wlen, isfirst, linecount, has_prev, torch.from_numpy(ll1), torch.from_numpy(bad1)]
        d = [t.to(dev) for t in host]
        out_ll = torch.empty((nf, maxl), dtype=torch.float64, device=dev)
        out_bad = torch.empty((nf, maxl), dtype=torch.uint8, device=dev)
        pam = torch.zeros(nf, dtype=torch.float64, device=dev)
        fph = torch.zeros(nf, dtype=torch.int32, device=dev)
        scratch = torch.empty(max(int(lib.ldg_lines_scratch_bytes(nf)), 256), dtype=torch.uint8, device=dev)
        a = L.LinesArgs()
        a.k = lines_consts(self.rf)
        a.d05 = arrays["demod_05"]
        a.demod = arrays.get("demod")
        a.burst = arrays.get("demod_burst")
        a.pilot = arrays.get("demod_pilot")
        a.capture_len = int(capture_len)
        a.nfields = nf
        a.proclines = self.proclines
        a.startloc, a.wlen, a.isfirst, a.linecount, a.has_prev = [t.data_ptr() for t in d[:5]]
        a.linelocs1 = d[5].data_ptr()
        a.linebad1 = d[6].data_ptr()
        a.prev_phase_adjust = float(prev_pam)
        a.linelocs = out_ll.data_ptr()
        a.linebad = out_bad.data_ptr()
        a.phase_adjust = pam.data_ptr()
        a.field_phase = fph.data_ptr()
        a.scratch = scratch.data_ptr()
        a.stream = stream
        L.check(lib.ldg_lines_refine(self.rf._ctx.handle, ctypes.byref(a)))
        self._bufs.append((d, scratch))
        return out_ll, out_bad, pam, fph

    def _field_lines(self, plan, ptr, fph=None, pam=None):
        rf = self.rf
        w = field_window(rf, plan.start)
        if self.pal:
            linecount = 312 if plan.isfirst else 313
            lineoffset = 2 if plan.isfirst else 3
        else:
            linecount = plan.linecount
            lineoffset = 0
        return FieldLines(w, plan.isfirst, linecount, lineoffset, linelocs_ptr=ptr, nlines=self.proclines,
                          field_phase=fph, phase_adjust=pam, sync_confidence=plan.sync_confidence)

    def locate(self, arrays, nblocks, stream=None, force_host=()):
        """Line locations of every field.  `arrays` maps output names
        (demod, demod_05, demod_burst[, demod_pilot]) to capture-wide
        float32 device tensors (one per output, equal lengths).  Returns the
        FieldLines of the valid fields in read order; `self.stats` counts
        batched, host-decoded and invalid reads.  `force_host` lists read
        indices to decode with the host restatement (checks of the resume
        path)."""
        rf = self.rf
        capture_len = int(arrays["demod_05"].numel())
        ptrs = {k: v.data_ptr() for k, v in arrays.items()}
        runs = self.sync_runs(ptrs["demod_05"], capture_len, stream)
        state = L.ChainState()
        prev_pam = 0.0
        prev_host = None     # host-decoded previous field (FieldLogic) if the last one was
        last_dev = None      # FieldLines of the last batched field
        ire0 = float(rf.DecoderParams["ire0"])
        fields = []
        reads = 0
        while True:
            plans, stop, st_out = run_chain(rf, runs, nblocks, state)
            # a forced host decode cuts the segment at that read index
            cut = None
            for i in range(len(plans)):
                if reads + i in force_host:
                    cut = i
                    break
            if cut is not None:
                plans = plans[:cut]
                stop = L.LDG_CHAIN_STOP_PREV
                st_out = self._state_after(plans, state)
            valid = [p for p in plans if p.valid]
            self.stats["invalid"] += len(plans) - len(valid)
            reads += len(plans)
            if valid:
                self.stats["segments"] += 1
                self.stats["batched"] += len(valid)
                if prev_host is not None and valid[0].has_prev and not self.pal:
                    prev_pam = float(prev_host.phase_adjust_median)
                ll, bad, pam, fph = self._refine(ptrs, capture_len, valid, prev_pam, stream)
                pam_h = pam.cpu().numpy() if not self.pal else None
                fph_h = fph.cpu().numpy() if not self.pal else None
                for i, p in enumerate(valid):
                    fl = self._field_lines(p, ll[i].data_ptr(),
                                           None if self.pal else int(fph_h[i]),
                                           None if self.pal else float(pam_h[i]))
                    fl._tensor = ll[i]
                    fields.append(fl)
                if not self.pal:
                    prev_pam = float(pam_h[-1])
                last_dev = fields[-1]
                prev_host = None
            if stop in (L.LDG_CHAIN_STOP_END,):
                break
            if stop == L.LDG_CHAIN_STOP_FULL:
                state = st_out
                continue
            # decode the next field on the host, with the previous field's results
            state = st_out
            w = field_window(rf, state.start)
            if w.first_block + w.nblocks > nblocks:
                break
            prevfield = None
            if state.prev_valid:
                prevfield = prev_host if prev_host is not None else self._proxy(arrays, last_dev, prev_pam)
            f = self._host_field(arrays, w, prevfield, state.fields_written)
            reads += 1
            self.stats["host"] += 1
            if not f.valid:
                self.stats["invalid"] += 1
                state.start += f.nextfieldoffset
                state.prev_valid = 0
                prev_host = None
                continue
            ll_host = np.ascontiguousarray(f.linelocs, dtype=np.float64)
            fl = FieldLines(w, f.isFirstField, f.linecount, f.lineoffset, linelocs=ll_host, nlines=len(ll_host),
                            field_phase=getattr(f, "fieldPhaseID", None),
                            phase_adjust=getattr(f, "phase_adjust_median", None),
                            sync_confidence=f.sync_confidence)
            fields.append(fl)
            state.start += f.nextfieldoffset - (w.readloc - w.startloc)
            state.prev_valid = 1
            state.prev_isfirst = int(bool(f.isFirstField))
            state.prev_startloc = w.startloc
            state.fields_written += 1
            prev_host = f
            if not self.pal:
                prev_pam = float(f.phase_adjust_median)
            if float(rf.DecoderParams["ire0"]) != ire0:
                ire0 = float(rf.DecoderParams["ire0"])
                runs = self.sync_runs(ptrs["demod_05"], capture_len, stream)
        return fields

    def _state_after(self, plans, state):
        """Chain state after the given plans (for a forced cut)."""
        st = L.ChainState()
        ctypes.memmove(ctypes.byref(st), ctypes.byref(state), ctypes.sizeof(st))
        for p in plans:
            if not p.valid:
                st.start += p.nextfieldoffset
                st.prev_valid = 0
                continue
            st.start += p.nextfieldoffset - (p.readloc - p.startloc)
            st.prev_valid = 1
            st.prev_isfirst = p.isfirst
            st.prev_startloc = p.startloc
            st.fields_written += 1
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
        p.linelocs = fl._tensor.cpu().numpy()[:fl.nlines].copy()
        p.linecount = fl.linecount
        p.lineoffset = fl.lineoffset
        p.isFirstField = fl.isFirstField
        p.sync_confidence = fl.sync_confidence
        p.phase_adjust_median = pam if not self.pal else 0
        p.fieldPhaseID = fl.fieldPhaseID if fl.fieldPhaseID is not None else 1
        # the batch does not keep the PAL burst phases of lines 7-19 that
        # determine_field_number seeds from (field phase ID metadata only)
        p.phase_adjust = {l: None for l in range(7, 22, 4)}
        return p

