"""ORACLE (test infrastructure only): AC3-RF QPSK front end and DPLL on the CPU.

Restates lddecode/ac3rf.py for parity checks of the GPU front end
(ldg_ac3_frontend) and the native DPLL (ldg_ac3_dpll_reclock).  Only tests/,
the smoke check and the CPU baseline of bench.py use this module.

* Each FIR-decimate stage (ac3rf.py:99-151) is a causal FIR over the whole
  input with zero history, output j = sum_k h[k] u[D*j - k] (the decimation
  phase (ntaps-1) % D is 0 for the 19/23-tap half-bands), evaluated in
  float64 over the full signal.
* The mixer (ac3rf.py:382-392) multiplies stage-2 sample j by the float32
  cos/sin tables at (phase_step * j) mod 2^14.
* The DPLL (ac3rf.py:200-299) is a pure-Python loop (small inputs only).

Pinned against golden vectors of the reference (tests/golden/ac3_loopback.npz,
made by tests/golden/make_golden.py).
"""

import math

import numpy as np

SYMBOL_RATE = 288e3
CARRIER_FREQ = 2.88e6


def halfband_kaiser(ntaps, beta=7.857):
    """ac3rf.py:48-61."""
    m = (ntaps - 1) // 2
    n = np.arange(-m, m + 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        h = np.sin(n * np.pi / 2) / (n * np.pi)
    h[n % 2 == 0] = 0
    h[m] = 0.5
    return h * np.kaiser(ntaps, beta)


def rrc_filter(ntaps, sps, beta):
    """ac3rf.py:64-96 (unit energy)."""
    if ntaps % 2 == 0:
        ntaps += 1
    t = np.arange(ntaps) - ntaps // 2
    h = np.empty(ntaps)
    for i, ti in enumerate(t):
        x = 4 * beta * ti / sps
        if ti == 0:
            h[i] = (1 + beta * (4 / np.pi - 1)) / sps
        elif abs(abs(x) - 1) < 1e-10:
            h[i] = beta / (sps * np.sqrt(2)) * ((1 + 2 / np.pi) * np.sin(np.pi / (4 * beta))
                                                + (1 - 2 / np.pi) * np.cos(np.pi / (4 * beta)))
        else:
            h[i] = (np.sin(np.pi * ti / sps * (1 - beta)) + x * np.cos(np.pi * ti / sps * (1 + beta))) \
                / (np.pi * ti / sps * (1 - x * x)) / sps
    return h / np.sqrt(np.sum(h * h))


def design(fs=40e6):
    """float32 taps, rates and NCO tables as ac3rf.py:315-357 builds them."""
    pre = int(np.log2(fs / 7e6))
    fmix = fs / (1 << pre)
    post = int(np.log2(fmix / 5 / SYMBOL_RATE))
    ffinal = fmix / (1 << post)
    sps = ffinal / SYMBOL_RATE
    lut = 1 << 14
    ph = 2 * np.pi * np.arange(lut) / lut
    return {
        "pre": [np.asarray(halfband_kaiser(19), np.float32)] * pre,
        "post": [np.asarray(halfband_kaiser(23 if i == post - 1 else 19), np.float32) for i in range(post)],
        "rrc": np.asarray(rrc_filter(int(np.ceil(3 * sps)) * 2 + 1, sps, 0.7), np.float32),
        "cos": np.cos(ph).astype(np.float32),
        "sin": np.sin(ph).astype(np.float32),
        "step": int(lut * CARRIER_FREQ / fmix),
        "mask": lut - 1,
        "final_fs": ffinal,
    }


def _fir(u, h, d):
    """Causal FIR with zero history, every d-th output from index 0."""
    y = np.convolve(u, np.asarray(h, np.float64))[: len(u)]
    return y[::d]


def frontend(x, fs=40e6):
    """Baseband I/Q (float64) at the final rate for the whole input `x`."""
    p = design(fs)
    u = np.asarray(x, np.float64)
    for h in p["pre"]:
        u = _fir(u, h, 2)
    j = np.arange(len(u), dtype=np.int64)
    ph = (j * p["step"]) & p["mask"]
    i = u * p["cos"][ph]
    q = u * p["sin"][ph]
    for h in p["post"]:
        i, q = _fir(i, h, 2), _fir(q, h, 2)
    return _fir(i, p["rrc"], 1), _fir(q, p["rrc"], 1)


class Dpll:
    """ac3rf.py:207-299 (float32 differential products, int counters)."""

    def __init__(self, fs):
        self.sd = int(round(fs / SYMBOL_RATE))
        self.nominal_add = int((1 << 10) * SYMBOL_RATE / fs)
        self.prev_i = np.zeros(self.sd, np.float32)
        self.prev_q = np.zeros(self.sd, np.float32)
        self.prev_symbol = 0
        self.error_sum = 0
        self.filter_out = 0
        self.clk = 0
        self.toggle_pos = 0
        self.toggles = 0
        w, z, ts, g = 2 * math.pi * 1800, 0.6, 1.0 / SYMBOL_RATE, 0.3
        self.g1 = (1 - math.exp(-2 * z * w * ts)) / g
        self.g2 = (1 + math.exp(-2 * w * z * ts) - 2 * math.exp(-w * z * ts) * math.cos(w * ts * math.sqrt(1 - z * z))) / g

    def reclock(self, i, q):
        i = np.asarray(i, np.float32)
        q = np.asarray(q, np.float32)
        sd = self.sd
        ci = np.concatenate([self.prev_i, i])
        cq = np.concatenate([self.prev_q, q])
        # products in float32 as the reference computes them
        re = (ci[sd:] * ci[:-sd] + cq[sd:] * cq[:-sd]).astype(np.float32)
        im = (cq[sd:] * ci[:-sd] - ci[sd:] * cq[:-sd]).astype(np.float32)
        sym = np.where(np.abs(re) >= np.abs(im), np.where(re >= 0, 0, 3), np.where(im >= 0, 1, 2))
        out = []
        for s in sym.tolist():
            if s != self.prev_symbol:
                self.toggle_pos = self.clk
                self.toggles += 1
            self.prev_symbol = s
            new = (self.clk + self.nominal_add + self.filter_out) & 1023
            self.filter_out = 0
            if new < self.clk:
                out.append(s)
                err = -(self.toggle_pos - 512) if self.toggles == 1 else 0
                es = (self.error_sum + err) & 0x7FFF
                if es >= 0x4000:
                    es -= 0x8000
                self.error_sum = es
                self.filter_out = int(err * self.g1 + es * self.g2)
                self.toggles = 0
            self.clk = new
        self.prev_i = ci[-sd:].copy()
        self.prev_q = cq[-sd:].copy()
        return np.array(out, np.uint8)


def dqpsk_signal(symbols, amplitude=1.0, noise_int=0, noise_scale=0.0, seed=0, cos_table=None):
    """Real DQPSK at 2.88 MHz, 40 MSPS, rectangular symbols (symbol of
    sample t = floor(t * 288e3 / 40e6) = (36 t) // 5000).  The carrier phase
    is an exact index (72 t + 250 k) mod 1000 into a 1000-entry cos table (k
    = quarter turns so far; symbol 1 steps the transmitted phase by -90
    degrees, 2 by +90, 3 by 180), so every CPU makes the same samples.
    Optional noise: sum of four uniform integers in [-noise_int, noise_int]
    times noise_scale."""
    steps = np.array([0, -1, 1, 2], np.int64)[np.asarray(symbols, np.int64)]
    k = np.cumsum(steps) % 4
    n = len(symbols) * 5000 // 36
    t = np.arange(n, dtype=np.int64)
    idx = (72 * t + 250 * k[(36 * t) // 5000]) % 1000
    if cos_table is None:
        cos_table = np.cos(2 * np.pi * np.arange(1000) / 1000).astype(np.float32)
    x = amplitude * cos_table[idx].astype(np.float64)
    if noise_int:
        rng = np.random.default_rng(seed)
        nz = rng.integers(-noise_int, noise_int + 1, (4, n)).sum(axis=0)
        x = x + nz * noise_scale
    return x.astype(np.float32)


def match_rate(tx, rx, probe_start=500, probe_len=64):
    """Align rx to tx by a probe subsequence and return the match rate over
    the overlap (the reference's loopback criterion)."""
    tx = np.asarray(tx, np.uint8)
    rx = np.asarray(rx, np.uint8)
    probe = tx[probe_start:probe_start + probe_len].tobytes()
    pos = rx.tobytes().find(probe)
    if pos < 0:
        return 0.0
    tail = tx[probe_start:]
    r = rx[pos:pos + len(tail)]
    n = min(len(tail), len(r))
    return float(np.mean(tail[:n] == r[:n])) if n else 0.0
