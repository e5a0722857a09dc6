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
