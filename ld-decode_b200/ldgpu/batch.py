"""Mixed batches: many captures of uneven length, NTSC and PAL together.

The reference decodes one capture at a time, its blocks demodulated by
DemodCache worker threads (lddecode/core.py:1165-1200) and its fields read
one after another (LDdecode.readfield, core.py:4060-4200).  Here:

* `DemodQueue` (ldg_queue_*): every block of every capture in one
  persistent demodulator launch whose CTAs pop blocks from a device work
  queue, replayed from a CUDA graph.  Each block's outputs are bit-identical
  to demodulating its capture alone.
* `autotune` times the queue's schedules (blocks per pop, persistent CTAs)
  on the submitted batch and keeps the fastest.
* `MixedBatch` runs the whole path for a list of device-resident captures:
  the queue demodulation, line locations per capture (`LineLocator`), and
  one TBC launch over the fields of all captures.
* `waves` splits a list of captures into groups whose outputs fit a device
  memory budget.
"""

import ctypes

import numpy as np

from . import lib as L

U_KEYS = ("demod", "demod_raw", "demod_05", "demod_burst", "demod_pilot", "rfhpf", "efm")
FIELD_KEYS = ("demod", "demod_05", "demod_burst", "demod_pilot")


def _raw_stream(stream):
    """Raw cudaStream_t of a torch.cuda.Stream or handle; None: torch's
    current stream.  Torch's default stream (handle 0) is passed as
    cudaStreamLegacy (1) so that work stays ordered with it (a NULL handle
    would select the queue's own stream)."""
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    h = getattr(stream, "cuda_stream", stream)
    return 1 if not h else h


class DemodQueue:
    """One ldg_queue: captures submitted together, demodulated in one launch."""

    def __init__(self, device=0):
        self._lib = L.load()
        h = L.c_p()
        L.check(self._lib.ldg_queue_create(ctypes.byref(h), int(device)))
        self.handle = h
        self.device = device
        self.schedule = (1, 0)

    def submit(self, items):
        """items: (rf, in_ptr, nblocks, in_stride, outs, mtf_level) per
        capture, as for RFDecode.demod_blocks_device (device pointers).  The
        queue reads each capture's filters from its RFDecode's context when
        it runs, so captures sharing an RFDecode must share mtf_level."""
        mtf = {}
        arr = (L.WorkItem * len(items))()
        for i, (rf, in_ptr, nblocks, stride, outs, level) in enumerate(items):
            if mtf.setdefault(id(rf), level) != level:
                raise ValueError("captures sharing an RFDecode must use one mtf_level per queue")
            a, _ = rf.demod_args(in_ptr, nblocks, stride, outs, level)
            arr[i].ctx = rf._ctx.handle
            arr[i].args = a
        self._items = list(items)  # keep the RFDecodes alive while the queue may run
        L.check(self._lib.ldg_queue_submit(self.handle, arr, len(arr)))

    def set_schedule(self, grab=1, ctas=0):
        L.check(self._lib.ldg_queue_set_schedule(self.handle, int(grab), int(ctas)))
        self.schedule = (int(grab), int(ctas))

    def info(self):
        """(blocks submitted, CTAs a run launches)."""
        total = ctypes.c_int64(0)
        grid = ctypes.c_int32(0)
        L.check(self._lib.ldg_queue_info(self.handle, ctypes.byref(total), ctypes.byref(grid)))
        return total.value, grid.value

    def set_variant(self, variant):
        """FFT decomposition of the launch (-1: the first item's context's)."""
        L.check(self._lib.ldg_queue_set_variant(self.handle, int(variant)))

    def run(self, stream=None, graph=True):
        """Enqueue one pass over every submitted block on `stream` (a
        torch.cuda.Stream or raw handle; None: torch's current stream)."""
        L.check(self._lib.ldg_queue_run(self.handle, _raw_stream(stream), 1 if graph else 0))

    def close(self):
        if getattr(self, "handle", None):
            self._lib.ldg_queue_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(queue, stream=None, grabs=(1, 2, 4, 8), ctas=(0,), reps=3, graph=True, variants=(None,)):
    """Time every (grab, ctas, variant) schedule on the queue's submitted
    batch with CUDA events on `stream` (one untimed run each, then the best
    of `reps`) and keep the fastest.  `variants`: FFT decompositions to try
    (None: the first item's context's).  Returns {"best": (grab, ctas,
    variant), "ms": {...}}."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    times = {}
    for v in variants:
        queue.set_variant(-1 if v is None else v)
        for g in grabs:
            for c in ctas:
                queue.set_schedule(g, c)
                queue.run(st, graph)
                best = None
                for _ in range(reps):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    queue.run(st, graph)
                    e1.record(st)
                    e1.synchronize()
                    ms = e0.elapsed_time(e1)
                    best = ms if best is None else min(best, ms)
                times[(g, c, v)] = best
    choice = min(times, key=times.get)
    queue.set_variant(-1 if choice[2] is None else choice[2])
    queue.set_schedule(choice[0], choice[1])
    return {"best": choice, "ms": times}


_DEMOD_TUNED = {}  # (device, system) -> (variant, blocks_per_cta), the winner kept per device


def autotune_demod(rf, in_ptr, nblocks, in_stride, outs, mtf_level=1, stream=None, variants=(0, 1),
                   blocks_per_cta=(1, 2, 4), reps=3, keep=True):
    """Time ldg_demod_blocks on a device batch (the caller's input and
    outputs, e.g. the first blocks of a capture) under every FFT
    decomposition (`variants`: L.LDG_VARIANT_STOCKHAM / LDG_VARIANT_IN_PLACE)
    and blocks per CTA, with CUDA events on `stream` (one untimed launch
    each, then the best of `reps`), and leave `rf` set to the fastest.
    With `keep`, the winner is remembered for the device and system and
    `tuned_demod` hands it to later contexts.  Returns {"best": (variant,
    blocks_per_cta), "ms": {(variant, bpc): ms}, "blocks": nblocks}."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    sh = st.cuda_stream if hasattr(st, "cuda_stream") else st
    times = {}
    for v in variants:
        rf.fft_variant = v
        for b in blocks_per_cta:
            rf.blocks_per_cta = b
            rf.demod_blocks_device(in_ptr, nblocks, in_stride, outs, mtf_level=mtf_level, stream=sh)
            best = None
            for _ in range(reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                rf.demod_blocks_device(in_ptr, nblocks, in_stride, outs, mtf_level=mtf_level, stream=sh)
                e1.record(st)
                e1.synchronize()
                ms = e0.elapsed_time(e1)
                best = ms if best is None else min(best, ms)
            times[(v, b)] = best
    choice = min(times, key=times.get)
    rf.fft_variant = choice[0]
    rf.blocks_per_cta = choice[1]
    if keep:
        _DEMOD_TUNED[(rf.device, rf.system)] = choice
    return {"best": choice, "ms": times, "blocks": nblocks}


def tuned_demod(rf):
    """Apply the schedule autotune_demod kept for rf's device and system, if
    any; returns it or None."""
    choice = _DEMOD_TUNED.get((rf.device, rf.system))
    if choice is not None:
        rf.fft_variant = choice[0]
        rf.blocks_per_cta = choice[1]
    return choice


def output_bytes_per_sample(system, audio=True, efm=True):
    """Device bytes the demodulator's outputs take per input sample."""
    n = 4 * (5 if system == "PAL" else 4) + 4 + (2 if efm else 0) + (8 * 991 / 31712 if audio else 0)
    return n


def waves(lengths, systems, budget_bytes, in_bytes=2):
    """Group capture indices (in order) so that each group's inputs and
    demodulator outputs stay within `budget_bytes`."""
    groups, cur, used = [], [], 0
    for i, (n, s) in enumerate(zip(lengths, systems)):
        need = n * (in_bytes + output_bytes_per_sample(s))
        if cur and used + need > budget_bytes:
            groups.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += need
    if cur:
        groups.append(cur)
    return groups


class MixedBatch:
    """The demod + TBC path over many device-resident captures at once.

    captures: list of (system, int16 device tensor).  One RFDecode per
    system (analog audio and EFM outputs on), one DemodQueue over all
    captures' blocks, one LineLocator per capture, one TBC launch; with
    pipeline = K > 1, K queues over consecutive groups of captures whose
    line locations and TBC overlap the next group's demodulation.  Work is
    enqueued on `self.stream` (a torch.cuda.Stream of its own) unless a
    stream is given; wait for it (or torch.cuda.synchronize()) before
    reading the outputs."""

    def __init__(self, captures, device=0, mtf_level=1, rfs=None, queue=None, locate_threads=1, locate_rfs=None,
                 pipeline=1, reserve_sms=24):
        import torch
        from .fieldread import blocks_in_capture
        from .rfdecode import RFDecode
        self.torch = torch
        self.device = device
        self.stream = torch.cuda.Stream(device=device)
        # the captures may still be being written on the caller's stream
        self.stream.wait_stream(torch.cuda.current_stream(device))
        self.captures = captures
        self.mtf_level = mtf_level
        self.rfs = dict(rfs or {})
        for system, _ in captures:
            if system not in self.rfs:
                self.rfs[system] = RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=True,
                                            device=device)
        dev = torch.device("cuda", device)
        self.items = []
        self.outs = []
        self.nblocks = []
        for system, cap in captures:
            rf = self.rfs[system]
            U = rf.blocklen - rf.blockcut - rf.blockcut_end
            nb = blocks_in_capture(rf, int(cap.numel()))
            nout = nb * U
            keys = [k for k in U_KEYS if k != "demod_pilot" or system == "PAL"]
            o = {k: torch.empty(nout, dtype=torch.int16 if k == "efm" else torch.float32, device=dev) for k in keys}
            o["audio_left"] = torch.empty(nb * 991, dtype=torch.float32, device=dev)
            o["audio_right"] = torch.empty(nb * 991, dtype=torch.float32, device=dev)
            self.outs.append(o)
            self.nblocks.append(nb)
            self.items.append((rf, cap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in o.items()}, mtf_level))
        # line locations of the captures on `locate_threads` host threads, each
        # with its own contexts (a context's sync-run scratch serves one call
        # at a time) and its own stream; locate_rfs: one {system: RFDecode}
        # per thread, reused across batches
        self.locate_threads = max(1, int(locate_threads))
        self.locate_rfs = locate_rfs if locate_rfs is not None else []
        if self.locate_threads > 1:
            while len(self.locate_rfs) < self.locate_threads:
                self.locate_rfs.append({})
            for d in self.locate_rfs[:self.locate_threads]:
                for system, _ in captures:
                    if system not in d:
                        d[system] = RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=True,
                                             device=device)
        self.queue = queue if queue is not None else DemodQueue(device)
        self.queue.submit(self.items)
        self.fields = None
        self.pictures = None
        self.picture_offsets = None
        self._pics = {}       # slot -> (uint16 device tensor, {capture: offset})
        self._pic_index = {}  # capture -> (tensor, offset)
        # pipelined form: the captures in `pipeline` consecutive groups of
        # about equal blocks, one queue each, launched back to back with
        # `reserve_sms` SMs left free, so that a group's line locations and
        # TBC run beside the next group's demodulation
        self.pipeline = max(1, min(int(pipeline), len(captures)))
        self.reserve_sms = int(reserve_sms)
        self._groups = [list(range(len(captures)))]
        self._group_queues = []
        if self.pipeline > 1:
            cum = np.cumsum(self.nblocks)
            total = cum[-1]
            cuts = [0]
            for g in range(1, self.pipeline):
                cuts.append(int(np.searchsorted(cum, g * total / self.pipeline)) + 1)
            cuts.append(len(captures))
            cuts = sorted(set(min(max(c, 0), len(captures)) for c in cuts))
            self._groups = [list(range(a, b)) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
            sms = torch.cuda.get_device_properties(device).multi_processor_count
            for idx in self._groups:
                q = DemodQueue(device)
                q.submit([self.items[i] for i in idx])
                q.set_schedule(self.queue.schedule[0] or 1, max(1, sms - self.reserve_sms))
                self._group_queues.append(q)

    @property
    def samples(self):
        """Input samples demodulated (block outputs kept) per pass."""
        tot = 0
        for (rf, _, nb, U, _, _) in self.items:
            tot += nb * U
        return tot

    def demod(self, stream=None, graph=True):
        self.queue.run(stream or self.stream, graph)

    def locate(self, stream=None):
        """Line locations of every capture's fields (LocatedFields per
        capture, in capture order)."""
        stream = stream or self.stream
        ev = self.torch.cuda.Event()
        ev.record(stream)
        self.fields = [None] * len(self.captures)
        self._locate(list(range(len(self.captures))), ev)
        for st in self._loc_streams:
            stream.wait_stream(st)
        return self.fields

    def _locate(self, indices, ready):
        """Locate captures `indices` once event `ready` has completed, on the
        locate threads (capture i by thread i % T) and their streams."""
        import os
        from .lines import LineLocator
        torch = self.torch
        T = self.locate_threads
        n = len(self.captures)
        if getattr(self, "locators", None) is None:
            # one per capture, kept across passes (pinned staging buffers); a
            # pass releases the previous pass's line-location buffers in
            # stream order
            cores = max(1, (os.cpu_count() or 1) // T)
            self.locators = []
            for i, (system, _) in enumerate(self.captures):
                rf = self.rfs[system] if T == 1 else self.locate_rfs[i % T][system]
                loc = LineLocator(rf)
                loc.threads = max(1, min(loc.threads, cores))
                self.locators.append(loc)
            self._loc_streams = [torch.cuda.Stream(device=self.device) for _ in range(T)]
        if self.fields is None or len(self.fields) != n:
            self.fields = [None] * n
        for st in self._loc_streams:
            st.wait_event(ready)

        def work(ti):
            st = self._loc_streams[ti]
            with torch.cuda.stream(st):
                for i in indices:
                    if i % T != ti:
                        continue
                    arrays = {k: self.outs[i][k] for k in FIELD_KEYS if k in self.outs[i]}
                    self.fields[i] = self.locators[i].locate(arrays, self.nblocks[i], st)

        if T == 1:
            work(0)
            return
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(T) as ex:
            list(ex.map(work, range(T)))

    def field_geometry(self, system):
        rf = self.rfs[system]
        w = rf.SysParams["outlinelen"]
        h = rf.SysParams["frame_lines"] // 2 + 1
        return w, h

    def tbc(self, stream=None):
        """One TBC launch over every located field of every capture; uint16
        pictures, capture after capture, field after field, in
        `self.pictures` (offsets per capture in `self.picture_offsets`)."""
        stream = stream or self.stream
        pics, offs = self._tbc(list(range(len(self.captures))), stream, 0)
        self.pictures = pics
        self.picture_offsets = np.array([offs[i] for i in range(len(self.captures))] +
                                        [offs[len(self.captures) - 1] + self._pic_size(len(self.captures) - 1)])
        return pics

    def _pic_size(self, i):
        w, h = self.field_geometry(self.captures[i][0])
        return len(self.fields[i]) * w * h

    def _tbc(self, indices, stream, slot):
        """One TBC launch over the located fields of captures `indices`, into
        picture buffer `slot`; returns (buffer, {capture: offset})."""
        from .field import tbc_fields
        from .lines import field_levels, tbc_batch
        torch = self.torch
        offs, total = {}, 0
        for i in indices:
            offs[i] = total
            total += self._pic_size(i)
        buf = self._pics.get(slot, (None, None))[0]
        if buf is None or buf.numel() < total:
            with torch.cuda.stream(stream):
                buf = torch.empty(max(total, 1), dtype=torch.uint16, device=torch.device("cuda", self.device))
        self._pics[slot] = (buf, offs)
        for i in indices:
            self._pic_index[i] = (buf, offs[i])
        base = buf.data_ptr()
        descs = []
        for i in indices:
            system = self.captures[i][0]
            rf = self.rfs[system]
            if len(self.fields[i]):
                descs.append(tbc_batch(rf, self.fields[i], self.outs[i]["demod"].data_ptr(), base + 2 * offs[i],
                                       field_levels(rf)))
        n = sum(len(d) for d in descs)
        if n:
            allf = (L.TbcField * n)()
            k = 0
            for d in descs:
                ctypes.memmove(ctypes.addressof(allf) + k * ctypes.sizeof(L.TbcField), ctypes.addressof(d),
                               ctypes.sizeof(d))
                k += len(d)
            # the sinc table is the same for both systems: any context runs the batch
            rf0 = self.rfs[self.captures[indices[0]][0]]
            tbc_fields(rf0, allf, stream=_raw_stream(stream), asynchronous=True)
        return buf[:max(total, 0)], offs

    def picture(self, capture, field):
        """uint16 (lines, width) view of one field's picture."""
        system = self.captures[capture][0]
        w, h = self.field_geometry(system)
        buf, off = self._pic_index[capture]
        o = off + field * w * h
        return buf[o:o + w * h].view(h, w)

    def set_variant(self, variant):
        """FFT decomposition of the launch (-1: the first item's context's)."""
        L.check(self._lib.ldg_queue_set_variant(self.handle, int(variant)))

    def run(self, stream=None, graph=True):
        """Demodulate, locate and resample everything; returns the number of
        fields.  Pipelined when built with pipeline > 1: the group queues
        are launched back to back, and each group's line locations and TBC
        are enqueued as soon as its demodulation is done."""
        stream = stream or self.stream
        if self.pipeline == 1:
            self.demod(stream, graph)
            self.locate(stream)
            self.tbc(stream)
            return sum(len(f) for f in self.fields)
        torch = self.torch
        if not hasattr(self, "_tbc_stream"):
            self._tbc_stream = torch.cuda.Stream(device=self.device, priority=-1)
        grab = self.queue.schedule[0]  # the autotuned blocks per pop, if any
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        evs = []
        for q in self._group_queues:
            if q.schedule != (grab, max(1, sms - self.reserve_sms)):
                q.set_schedule(grab, max(1, sms - self.reserve_sms))
            q.run(stream, graph)
            ev = torch.cuda.Event()
            ev.record(stream)
            evs.append(ev)
        self.fields = [None] * len(self.captures)
        for g, (idx, ev) in enumerate(zip(self._groups, evs)):
            self._locate(idx, ev)
            for st in self._loc_streams:
                self._tbc_stream.wait_stream(st)
            self._tbc(idx, self._tbc_stream, g)
        stream.wait_stream(self._tbc_stream)
        return sum(len(f) for f in self.fields)

    def close(self):
        self.queue.close()
        for q in self._group_queues:
            q.close()
