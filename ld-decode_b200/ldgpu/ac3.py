"""AC3-RF (2.88 MHz differential QPSK) demodulator: GPU front end, native DPLL.

Same interface as lddecode.ac3rf.Ac3RfDemodulator (lddecode/ac3rf.py:
302-396): `Ac3RfDemodulator(input_sample_frequency).demodulate_to_symbols(
float32 block) -> bytes`, streaming (any block lengths).  The front end
(half-band /2 stages, 14-bit NCO mix at 2.88 MHz, complex half-band /2
stages, RRC matched filter) runs on the GPU through ldg_ac3_frontend; the
symbol-timing DPLL runs in native code through ldg_ac3_dpll_reclock.  The
filter taps are designed here exactly as the reference designs them
(ac3rf.py:48-96, 315-357).
"""

import ctypes

import numpy as np

from . import lib as L

SYMBOL_RATE = 288e3
CARRIER_FREQ = 2.88e6
KAISER_BETA_80DB = 7.857
PHASE_ACCUM_BITS = 14
HISTORY = 2048  # raw samples kept between calls (>= the filters' 1134-sample history)


def halfband_kaiser(ntaps, beta=KAISER_BETA_80DB):
    """Kaiser-windowed half-band low-pass (cutoff fs/4), ntaps = 4k+3
    (ac3rf.py:48-61)."""
    assert ntaps % 4 == 3, "half-band length must be 4k+3"
    m = (ntaps - 1) // 2
    n = np.arange(-m, m + 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        h = np.sin(n * np.pi / 2) / (n * np.pi)
    h[m] = 0.5
    h[n % 2 == 0] = 0
    h[m] = 0.5
    return h * np.kaiser(ntaps, beta)


def rrc_filter(ntaps, samples_per_symbol, beta):
    """Unit-energy root-raised-cosine FIR (ac3rf.py:64-96)."""
    if ntaps % 2 == 0:
        ntaps += 1
    T = samples_per_symbol
    t = np.arange(ntaps) - ntaps // 2
    h = np.empty(ntaps)
    for i, ti in enumerate(t):
        if ti == 0:
            h[i] = 1 / T * (1 + beta * (4 / np.pi - 1))
        elif abs(abs(4 * beta * ti / T) - 1) < 1e-10:
            h[i] = beta / (T * np.sqrt(2)) * ((1 + 2 / np.pi) * np.sin(np.pi / (4 * beta))
                                              + (1 - 2 / np.pi) * np.cos(np.pi / (4 * beta)))
        else:
            h[i] = (1 / T * (np.sin(np.pi * ti / T * (1 - beta))
                             + 4 * beta * ti / T * np.cos(np.pi * ti / T * (1 + beta)))
                    / (np.pi * ti / T * (1 - (4 * beta * ti / T) ** 2)))
    return h / np.sqrt(np.sum(h * h))


class Ac3Design:
    """Rates, stage counts and float32 taps for an input sample rate
    (ac3rf.py:315-357).  The GPU path is built for the 40 MSPS layout: two
    pre-mix /2 stages, two post-mix /2 stages (19 then 23 taps)."""

    def __init__(self, input_sample_frequency):
        fs = float(input_sample_frequency)
        self.pre_mix_stages = int(np.log2(fs / 7e6))
        self.mix_frequency = fs / (1 << self.pre_mix_stages)
        self.post_mix_stages = int(np.log2(self.mix_frequency / 5 / SYMBOL_RATE))
        self.final_frequency = self.mix_frequency / (1 << self.post_mix_stages)
        if self.pre_mix_stages != 2 or self.post_mix_stages != 2:
            raise NotImplementedError("the GPU AC3 front end is built for 2 + 2 half-band stages (28-56 MSPS input)")
        self.hb19 = np.asarray(halfband_kaiser(19), np.float32)
        self.hb23 = np.asarray(halfband_kaiser(23), np.float32)
        sps = self.final_frequency / SYMBOL_RATE
        ntaps = int(np.ceil(3 * sps)) * 2 + 1
        self.rrc = np.asarray(rrc_filter(ntaps, sps, 0.7), np.float32)
        lut_size = 1 << PHASE_ACCUM_BITS
        ph = 2 * np.pi * np.arange(lut_size) / lut_size
        self.cos_lut = np.cos(ph).astype(np.float32)
        self.sin_lut = np.sin(ph).astype(np.float32)
        self.phase_step = int(lut_size * CARRIER_FREQ / self.mix_frequency)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


class Ac3Frontend:
    """GPU front end: raw RF -> baseband I/Q at fs/16."""

    def __init__(self, input_sample_frequency, device=0):
        lib = L.load()
        self._lib = lib
        self.design = d = Ac3Design(input_sample_frequency)
        h = ctypes.c_void_p()
        rc = lib.ldg_ac3_create(ctypes.byref(h), int(device), _p(d.hb19), len(d.hb19), _p(d.hb23), len(d.hb23),
                                _p(d.rrc), len(d.rrc), PHASE_ACCUM_BITS, _p(d.cos_lut), _p(d.sin_lut),
                                int(d.phase_step))
        if rc != 0:
            raise L.LdgError(rc, lib.ldg_ac3_last_error().decode())
        self.handle = h

    def run(self, samples, in_first, out_first, out_count, out_i=None, out_q=None, stream=None):
        """I/Q outputs [out_first, out_first+out_count) from `samples` (numpy
        float32/int16 array, or (device pointer, kind, count)) whose first
        element is absolute sample `in_first`."""
        if isinstance(samples, tuple):
            ptr, kind, n = samples
        else:
            a = np.ascontiguousarray(samples)
            kind = L.LDG_IN_INT16 if a.dtype == np.int16 else L.LDG_IN_FLOAT32
            if kind == L.LDG_IN_FLOAT32 and a.dtype != np.float32:
                a = a.astype(np.float32)
            ptr, n = a.ctypes.data, len(a)
            samples = a
        oi = np.empty(out_count, np.float32) if out_i is None else out_i
        oq = np.empty(out_count, np.float32) if out_q is None else out_q
        pi = oi if isinstance(oi, int) else oi.ctypes.data
        pq = oq if isinstance(oq, int) else oq.ctypes.data
        rc = self._lib.ldg_ac3_frontend(self.handle, ctypes.c_void_p(ptr), kind, int(in_first), int(n),
                                        int(out_first), int(out_count), ctypes.c_void_p(pi), ctypes.c_void_p(pq),
                                        stream)
        if rc != 0:
            raise L.LdgError(rc, self._lib.ldg_ac3_last_error().decode())
        return oi, oq

    def close(self):
        if getattr(self, "handle", None):
            self._lib.ldg_ac3_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ac3Dpll:
    """Native symbol-timing DPLL (ac3rf.py:200-299), streaming."""

    def __init__(self, final_frequency):
        lib = L.load()
        self._lib = lib
        h = ctypes.c_void_p()
        rc = lib.ldg_ac3_dpll_create(ctypes.byref(h), float(final_frequency))
        if rc != 0:
            raise L.LdgError(rc, lib.ldg_ac3_last_error().decode())
        self.handle = h

    def reclock_symbols(self, i, q):
        i = np.ascontiguousarray(i, np.float32)
        q = np.ascontiguousarray(q, np.float32)
        out = np.empty(len(i), np.uint8)
        n = ctypes.c_int64(0)
        rc = self._lib.ldg_ac3_dpll_reclock(self.handle, _p(i), _p(q), len(i), _p(out), ctypes.byref(n))
        if rc != 0:
            raise L.LdgError(rc, self._lib.ldg_ac3_last_error().decode())
        return out[:n.value]

    def __del__(self):
        try:
            self._lib.ldg_ac3_dpll_destroy(self.handle)
        except Exception:
            pass


class Ac3RfDemodulator:
    """Streaming AC3-RF demodulator with the reference interface
    (ac3rf.py:302-396)."""

    def __init__(self, input_sample_frequency, logger=None, device=0):
        self.input_sample_frequency = input_sample_frequency
        self.frontend = Ac3Frontend(input_sample_frequency, device)
        self.dpll = Ac3Dpll(self.frontend.design.final_frequency)
        self._tail = np.zeros(0, np.float32)
        self._total = 0      # raw samples consumed
        self._emitted = 0    # I/Q samples produced (= ceil(total / 16))
        if logger is not None:
            d = self.frontend.design
            logger.debug("AC3 demodulator: mix Fs=%.0f, final Fs=%.0f, %.1f samples/symbol"
                         % (d.mix_frequency, d.final_frequency, d.final_frequency / SYMBOL_RATE))

    def input_sample_alignment(self):
        return 1

    def demodulate_iq(self, input_buffer):
        data = np.asarray(input_buffer, np.float32)
        buf = np.concatenate([self._tail, data])
        in_first = self._total - len(self._tail)
        self._total += len(data)
        target = (self._total + 15) // 16
        i, q = self.frontend.run(buf, in_first, self._emitted, target - self._emitted)
        self._emitted = target
        self._tail = buf[-HISTORY:].copy()
        return i, q

    def demodulate_to_symbols(self, input_buffer):
        i, q = self.demodulate_iq(input_buffer)
        return self.dpll.reclock_symbols(i, q).tobytes()
