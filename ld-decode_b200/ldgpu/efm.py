"""EFM phase-locked loop: the .efm stream (T-values) from the demodulator's
EFM output.

`EFM_PLL` keeps the reference's class API (lddecode/efm_pll.py:80-244):
construct one per decode, feed it each field's int16 EFM samples in write
order with `process`, get that call's T-values (int8, 3..11 on valid EFM)
as a numpy array; the loop state carries from call to call.  The loop runs
in native host code (ldg_efm_pll_*, csrc/ldg_efm.cpp): it is serial and
edge-driven, so one PLL runs per decoded stream and several streams run on
several threads (the C call releases the GIL).  The EFM samples may come
from a device tensor (the batched path's `efm` output); they are copied to
the host first.

Or only the crossings cross to the host: `efm_edges` finds every zero
crossing of a device EFM array on the GPU (ldg_efm_edges: position and the
two sample values, 8 bytes per crossing, one crossing every ~25 samples),
and `EFM_PLL.process_edges` runs the loop from them over one field's slice
of that array, with the same T-values and state as `process` on the
samples.
"""

import ctypes

import numpy as np

from . import lib as L


class EFM_PLL:
    """efm_pll.EFM_PLL: process(inputBuffer) -> int8 T-values."""

    def __init__(self):
        self._lib = L.load()
        h = ctypes.c_void_p()
        L.check(self._lib.ldg_efm_pll_create(ctypes.byref(h)))
        self._h = h
        self._out = np.empty(1 << 16, np.int8)

    def process(self, inputBuffer):
        """T-values of `inputBuffer` (int16 samples; numpy, or a torch
        tensor on any device), continuing from the previous call's state."""
        x = inputBuffer
        if hasattr(x, "detach"):  # torch tensor
            x = x.detach().cpu().numpy()
        x = np.ascontiguousarray(x)
        if x.dtype != np.int16:
            raise TypeError(f"EFM_PLL.process needs int16 samples, got {x.dtype}")
        if len(self._out) < len(x):
            self._out = np.empty(len(x), np.int8)
        n = ctypes.c_int64(0)
        L.check(self._lib.ldg_efm_pll_process(self._h, x.ctypes.data, len(x), self._out.ctypes.data,
                                              len(self._out), ctypes.byref(n)))
        return self._out[:n.value].copy()

    def process_edges(self, edges, lo, hi, first, last):
        """T-values of the samples [lo, hi) of an array known only by its
        zero crossings `edges` (an EFM_EDGE_DTYPE array sorted by position,
        from `efm_edges` / ldg_efm_edges) and its samples first = [lo] and
        last = [hi - 1]: the same values and state as `process` on those
        samples."""
        e = np.ascontiguousarray(edges, dtype=L.EFM_EDGE_DTYPE)
        if len(self._out) < hi - lo:
            self._out = np.empty(hi - lo, np.int8)
        n = ctypes.c_int64(0)
        L.check(self._lib.ldg_efm_pll_process_edges(self._h, e.ctypes.data, len(e), int(lo), int(hi), int(first),
                                                    int(last), self._out.ctypes.data, len(self._out),
                                                    ctypes.byref(n)))
        return self._out[:n.value].copy()

    def state(self):
        """{zcPreviousInput, delta, currentPeriod, phaseAdjust, refClockTime,
        frequencyHysteresis, tCounter} (the reference's attribute names)."""
        d = (ctypes.c_double * 4)()
        i = (ctypes.c_int32 * 3)()
        L.check(self._lib.ldg_efm_pll_state(self._h, d, i))
        return {"zcPreviousInput": i[0], "delta": d[0], "currentPeriod": d[1], "phaseAdjust": d[2],
                "refClockTime": d[3], "frequencyHysteresis": i[1], "tCounter": i[2]}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ldg_efm_pll_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def efm_edges(efm, has_before=False, pos_offset=0, stream=None):
    """Zero crossings of a device int16 tensor `efm` (ldg_efm_edges, on the
    GPU) as an EFM_EDGE_DTYPE numpy array: the positions (pos_offset + i),
    and the values before and at each crossing.  With has_before the sample
    before efm[0] (efm.data_ptr() - 2 bytes) is read for position 0."""
    import torch
    lib = L.load()
    n = int(efm.numel())
    dev = efm.device
    scratch = torch.empty(max(int(lib.ldg_efm_edges_scratch_bytes(n)), 256), dtype=torch.uint8, device=dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    sh = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    cap = n
    out = torch.empty(max(cap, 1) * L.EFM_EDGE_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    L.check(lib.ldg_efm_edges(efm.data_ptr(), n, 1 if has_before else 0, int(pos_offset), out.data_ptr(), cap,
                              count.data_ptr(), scratch.data_ptr(), sh))
    k = int(count.item())
    return out[:k * L.EFM_EDGE_DTYPE.itemsize].cpu().numpy().view(L.EFM_EDGE_DTYPE)


def field_efm_slices(fields, efm, first=0, count=None):
    """The EFM slice Field.downscale hands to the PLL for each of
    fields[first:first + count] (a LocatedFields): data['efm'][int(linelocs[1])
    : int(linelocs[linecount + 1])] (core.py:2704-2707) as capture-wide sample
    ranges [lo, hi), with the samples at lo and hi - 1 -- what
    EFM_PLL.process_edges needs besides the crossings.  Device tensors
    (int64 (count, 2), int16 (count, 2)) made by gathers on the current
    stream from the fields' device line locations; the few per-field
    integers from the host go over by an SM copy from pinned memory, not by
    a copy-engine transfer that would queue behind bulk copies."""
    import torch
    n = len(fields) if count is None else count
    dev = efm.device
    lib = L.load()
    stream = torch.cuda.current_stream(dev)

    def to_dev(a):
        a = np.ascontiguousarray(a, np.int64)
        h = torch.from_numpy(a).pin_memory()
        d = torch.empty(a.shape, dtype=torch.int64, device=dev)
        if a.size:
            L.check(lib.ldg_copy_async(d.data_ptr(), h.data_ptr(), a.nbytes, stream.cuda_stream))
        return d, h

    bounds, samples, keep = [], [], []
    k = 0  # field index of the part's first field
    for part in fields._parts:
        m = len(part[1]) if part[0] == "batch" else 1
        lo, hi = max(first, k), min(first + n, k + m)
        if lo < hi:
            if part[0] == "batch":
                _, pl, ll, _, _, _ = part
                rows = torch.arange(lo - k, hi - k, device=dev)
                if fields.rf.system == "PAL":
                    lc = np.where(pl.isfirst[lo - k:hi - k] != 0, 312, 313)
                else:
                    lc = pl.linecount[lo - k:hi - k].astype(np.int64)
                lc_t, h1 = to_dev(np.asarray(lc, np.int64) + 1)
                st, h2 = to_dev(pl.startloc[lo - k:hi - k])
                keep.extend((h1, h2))
                a = st + ll[rows, 1].to(torch.int64)   # int() of a positive location truncates
                b = st + ll[rows, lc_t].to(torch.int64)
            else:
                fl = part[1]
                ll = np.asarray(fl.host_linelocs(), np.float64)
                st = fl.window.startloc
                ab, h1 = to_dev(np.array([[st + int(ll[1]), st + int(ll[fl.linecount + 1])]], np.int64))
                keep.append(h1)
                a, b = ab[:, 0], ab[:, 1]
            bounds.append(torch.stack([a, b], 1))
            samples.append(torch.stack([efm[a], efm[b - 1]], 1))
        k += m
    if not bounds:
        return (torch.zeros((0, 2), dtype=torch.int64, device=dev), torch.zeros((0, 2), dtype=torch.int16, device=dev))
    out = torch.cat(bounds), torch.cat(samples)
    # the pinned sources stay alive until the copies that read them have run
    ev = torch.cuda.Event()
    ev.record(stream)
    _PINNED_IN_FLIGHT.append((ev, keep))
    while _PINNED_IN_FLIGHT and _PINNED_IN_FLIGHT[0][0].query():
        _PINNED_IN_FLIGHT.pop(0)
    return out


_PINNED_IN_FLIGHT = []
