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


def field_efm_slices(fields, efm, first=0, count=None, bounds=None, samples=None, stream=None):
    """The EFM slice Field.downscale hands to the PLL for each of
    fields[first:first + count] (a LocatedFields): data['efm'][int(linelocs[1])
    : int(linelocs[linecount + 1])] (core.py:2704-2707) as capture-wide sample
    ranges [lo, hi), with the samples at lo and hi - 1 -- what
    EFM_PLL.process_edges needs besides the crossings.  One kernel
    (ldg_efm_field_slices) on `stream` (default: torch's current stream),
    reading the fields' device line locations; it writes into `bounds`
    (int64 (count, 2)) and `samples` (int16 (count, 2)) when given -- device
    or pinned host tensors, so the results can land on the host without a
    copy -- else into new device tensors.  Returns (bounds, samples)."""
    import torch
    lib = L.load()
    a = fields.arrays()
    n = len(a["startloc"]) - first if count is None else count
    dev = efm.device
    if bounds is None:
        bounds = torch.empty((n, 2), dtype=torch.int64, device=dev)
    if samples is None:
        samples = torch.empty((n, 2), dtype=torch.int16, device=dev)
    if n == 0:
        return bounds, samples
    sel = slice(first, first + n)
    # the per-field inputs, read by the kernel from pinned host memory
    h = torch.empty(n * 20, dtype=torch.uint8).pin_memory()
    hb = h.numpy()
    hb[:8 * n].view(np.int64)[:] = a["startloc"][sel]
    hb[8 * n:16 * n].view(np.uint64)[:] = a["linelocs_ptr"][sel]
    hb[16 * n:].view(np.int32)[:] = np.asarray(a["linecount"][sel], np.int32) + 1
    st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    L.check(lib.ldg_efm_field_slices(h.data_ptr(), h.data_ptr() + 8 * n, h.data_ptr() + 16 * n, n, efm.data_ptr(),
                                     int(efm.numel()), bounds.data_ptr(), samples.data_ptr(), st))
    # the pinned inputs stay alive until the kernel that reads them has run
    ev = torch.cuda.Event()
    ev.record(torch.cuda.ExternalStream(st) if stream is not None else torch.cuda.current_stream(dev))
    _PINNED_IN_FLIGHT.append((ev, h))
    while _PINNED_IN_FLIGHT and _PINNED_IN_FLIGHT[0][0].query():
        _PINNED_IN_FLIGHT.pop(0)
    return bounds, samples


_PINNED_IN_FLIGHT = []
