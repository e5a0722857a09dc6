"""Seeded synthetic LaserDisc RF captures (NTSC / PAL) for tests and benchmarks.

No real disc captures are available, so every input is made here: a composite
video raster (equalising / broad vertical-sync pulses, H-sync, colour burst,
75 % colour bars with chroma at fsc; PAL adds the V-switch and a line-locked
3.75 MHz pilot during sync), band-limited and pre-emphasised with the
decoder's own emphasis time constants, FM-modulated onto the video carrier
(NTSC sync tip 7.61 MHz / white 9.31 MHz; PAL 6.76 / 7.9 MHz), plus the two
analog-audio FM carriers (NTSC 2.30/2.81 MHz, PAL 683.6/1066.4 kHz) carrying
seeded tones, a random-run-length EFM band below 1.75 MHz, optionally a
2.88 MHz root-raised-cosine QPSK carrier, and white noise at a given SNR,
scaled to a 12-bit range and rounded to int16 at 40 MSPS.

Generation is chunked and runs in torch float64 on any device, so a 400 M
sample capture can be built on the GPU in a few seconds; the video content is
a closed-form function of the absolute sample index, the FM phase is carried
across chunks, and the random parts are seeded per chunk.
"""

import math

import numpy as np
import scipy.signal as sps
import torch

from . import params
from .filters import emphasis_ba

FS_HZ = 40e6
CHUNK = 1 << 22
LEAD = 512  # FIR lead-in samples kept from before each chunk
PHASE_ONE = 1 << 24

_BARS = [(1, 1, 1), (1, 1, 0), (0, 1, 1), (0, 1, 0), (1, 0, 1), (1, 0, 0), (0, 0, 1)]


def _bar_tables(black, span):
    ys, us, vs = [], [], []
    for r, g, b in _BARS:
        r, g, b = 0.75 * r, 0.75 * g, 0.75 * b
        y = 0.299 * r + 0.587 * g + 0.114 * b
        ys.append(black + y * span)
        us.append(0.492 * (b - y) * span)
        vs.append(0.877 * (r - y) * span)
    return ys, us, vs


class _System:
    def __init__(self, system):
        sp = params.sysparams(system)
        fp = params.filterparams(system)
        self.name = system
        self.sp = sp
        self.lp = float(sp["line_period"])
        self.frame_lines = sp["frame_lines"]
        self.npulse = sp["numPulses"]
        self.hsync_us = sp["hsyncPulseUS"]
        self.eq_us = sp["eqPulseUS"]
        self.vsync_us = sp["vsyncPulseUS"]
        self.sync_ire = float(sp["vsync_ire"])
        self.ire0 = float(sp["ire0"])
        self.hz_ire = float(sp["hz_ire"])
        self.fsc = float(sp["fsc_mhz"]) * 1e6
        self.burst = sp["colorBurstUS"]
        self.active = sp["activeVideoUS"]
        self.pal = system == "PAL"
        black = 0.0 if self.pal else 7.5
        self.bar_y, self.bar_u, self.bar_v = _bar_tables(black, 100.0 - black)
        self.black = black
        self.burst_amp = 21.43 if self.pal else 20.0
        self.audio_f = (float(sp["audio_lfreq"]), float(sp["audio_rfreq"]))
        self.video_lpf = 5.5e6 if self.pal else 4.8e6
        t_hi, t_lo = fp["video_deemp"]
        self.emp_ba = emphasis_ba(t_lo, t_hi, FS_HZ)


def composite_ire(sysd, n, shift=None, pal8=False, bruch_line=(8, 7)):
    """Composite video level in IRE at absolute sample indices n (int64),
    the video time base moved by `shift` samples (float64 per sample) when
    given.  PAL with `pal8`: the V-switch alternates line after line across
    frames (a 625-line frame flips it) and the burst is blanked at the start
    of each field in a 4-field Bruch sequence, so that the decoder's line 6
    carries burst in the second and third fields of the sequence and none in
    the first and fourth; with the subcarrier's 4-frame phase cycle this
    gives the 8-field sequence.  The raster's field starting at frame
    half-line 0 is the one the decoder calls the second field; the blanking
    ends at line bruch_line[0] (or one line later) of that field and at line
    bruch_line[1] (or one later) of the other, counted from each field's
    first full line."""
    d = sysd
    tn = n.to(torch.float64)
    if shift is not None:
        tn = tn + shift
    t = tn / (FS_HZ / 1e6)  # microseconds
    hl_len = d.lp / 2
    frame_len = d.frame_lines * d.lp
    tf = torch.remainder(t, frame_len)
    hl = torch.floor(tf / hl_len)
    th = tf - hl * hl_len
    hl = hl.to(torch.int64)
    hf = torch.remainder(hl, d.frame_lines)
    np_ = d.npulse

    ire = torch.full_like(t, 0.0)
    eq = (hf < np_) | ((hf >= 2 * np_) & (hf < 3 * np_))
    vs = (hf >= np_) & (hf < 2 * np_)
    reg = hf >= 3 * np_
    # the line grid is continuous over the frame: lines start on even
    # frame half-lines, so the second field's vblank begins mid-line
    first = torch.remainder(hl, 2) == 0
    tau = torch.where(first, th, th + hl_len)
    line = hl // 2

    sync = (eq & (th < d.eq_us)) | (vs & (th < d.vsync_us)) | (reg & first & (th < d.hsync_us))
    w = 2 * math.pi * d.fsc * (t * 1e-6)
    sinw, cosw = torch.sin(w), torch.cos(w)
    vsw = torch.where(torch.remainder(line, 2) == 0, 1.0, -1.0) if d.pal else 1.0
    if d.pal and pal8:
        # absolute line count for the V-switch, absolute field count for the Bruch sequence
        frame = torch.floor(t / frame_len).to(torch.int64)
        vsw = torch.where(torch.remainder(frame * d.frame_lines + line, 2) == 0, 1.0, -1.0)
        second = hl >= d.frame_lines
        field_abs = 2 * frame + second.to(torch.int64)
        lf = torch.where(second, (hl - d.frame_lines) // 2, hl // 2)  # line within the field
        f4 = torch.remainder(field_abs, 4)
        keep = (f4 == 0) | (f4 == 1)
        b0 = torch.where(second, bruch_line[1], bruch_line[0])
        blanked = lf < torch.where(keep, b0, b0 + 1)
    in_burst = reg & (tau >= d.burst[0]) & (tau < d.burst[1])
    if d.pal and pal8:
        in_burst = in_burst & ~blanked
    if d.pal:
        burst = d.burst_amp * (-sinw * 0.70710678 + vsw * cosw * 0.70710678)
    else:
        burst = -d.burst_amp * sinw
    ire = torch.where(in_burst, burst, ire)

    a0, a1 = d.active
    in_act = reg & (tau >= a0) & (tau < a1)
    bar = torch.clamp(((tau - a0) / ((a1 - a0) / 7)).floor().to(torch.int64), 0, 6)
    by = torch.tensor(d.bar_y, dtype=torch.float64, device=n.device)[bar]
    bu = torch.tensor(d.bar_u, dtype=torch.float64, device=n.device)[bar]
    bv = torch.tensor(d.bar_v, dtype=torch.float64, device=n.device)[bar]
    act = by + bu * sinw + bv * cosw * vsw
    ire = torch.where(in_act, act, ire)
    if not d.pal:
        ire = torch.where(reg & ~in_burst & ~in_act & (tau >= d.hsync_us + 0.6) & (tau >= a1),
                          torch.full_like(ire, 0.0), ire)
    ire = torch.where(sync, torch.full_like(ire, d.sync_ire), ire)
    if d.pal:
        # line-locked 3.75 MHz pilot during the first 5 us of every line
        pil = 10.0 * torch.sin(2 * math.pi * 3.75 * tau)
        ire = ire + torch.where(tau < 5.0, pil, torch.zeros_like(pil))
    return ire


def _fir_video(sysd):
    """Band-limit + pre-emphasis as one FIR (impulse response of the IIR
    emphasis convolved with a linear-phase low-pass)."""
    lpf = sps.firwin(63, sysd.video_lpf / (FS_HZ / 2))
    imp = np.zeros(256)
    imp[0] = 1.0
    emp = sps.lfilter(sysd.emp_ba[0], sysd.emp_ba[1], imp)
    return np.convolve(lpf, emp)


def _fftconv(x, taps):
    n = x.shape[0] + taps.shape[0] - 1
    nf = 1 << (n - 1).bit_length()
    y = torch.fft.irfft(torch.fft.rfft(x, nf) * torch.fft.rfft(taps, nf), nf)
    return y[:x.shape[0]]


def _efm_wave(gen, n0, length, device):
    """+/-1 NRZ with run lengths 3T..11T at the EFM channel rate."""
    tbit = FS_HZ / 4.3218e6
    nrun = int(length / (3 * tbit)) + 64
    runs = torch.randint(3, 12, (nrun,), generator=gen, device=device).to(torch.float64) * tbit
    edges = torch.cumsum(runs, 0) - float(torch.rand(1, generator=gen, device=device).item()) * 11 * tbit
    pos = torch.arange(length, device=device, dtype=torch.float64)
    k = torch.searchsorted(edges, pos)
    return torch.where(torch.remainder(k, 2) == 0, 1.0, -1.0)


def _rrc(beta, sps_, span):
    t = np.arange(-span * sps_, span * sps_ + 1) / sps_
    h = np.zeros_like(t)
    for i, ti in enumerate(t):
        if abs(ti) < 1e-12:
            h[i] = 1 - beta + 4 * beta / np.pi
        elif abs(abs(ti) - 1 / (4 * beta)) < 1e-9:
            h[i] = beta / np.sqrt(2) * ((1 + 2 / np.pi) * np.sin(np.pi / (4 * beta))
                                        + (1 - 2 / np.pi) * np.cos(np.pi / (4 * beta)))
        else:
            h[i] = (np.sin(np.pi * ti * (1 - beta)) + 4 * beta * ti * np.cos(np.pi * ti * (1 + beta))) / (
                np.pi * ti * (1 - (4 * beta * ti) ** 2))
    return h / np.sqrt(np.sum(h * h))


def synth_capture(system, nsamples, seed=0, snr_db=40.0, tones=(1000.0, 440.0),
                  efm=True, qpsk=False, device="cpu", start=0, scale=2000.0, return_symbols=False, wow=None,
                  pal8=False, bruch_line=(8, 7)):
    """int16 torch tensor of `nsamples` RF samples at 40 MSPS.

    `wow` = (amplitude, period) in samples moves the video time base
    sinusoidally, as a disc's speed error does: the video at sample n is the
    raster's at n + amplitude * sin(2 pi n / period).  PAL with `pal8`: the
    8-field sequence (see composite_ire).

    `start` offsets the absolute sample index (so different seeds/offsets give
    different field phases).  With qpsk=True the 2.88 MHz carrier is
    differential QPSK at 288 kbaud (RRC, alpha 0.5), one continuous symbol
    stream over the whole capture; return_symbols=True also returns the
    transmitted symbols.  The same (system, nsamples, seed, start, device
    type) always gives the same capture.
    """
    dev = torch.device(device)
    sysd = _System(system)
    taps = torch.tensor(_fir_video(sysd), dtype=torch.float64, device=dev)
    efm_taps = torch.tensor(sps.firwin(127, 1.75e6 / (FS_HZ / 2)), dtype=torch.float64, device=dev)
    if qpsk:
        sym_rate = 288e3
        sps_ = 40  # generate symbols at 11.52 MS/s then interpolate
        rrc = torch.tensor(_rrc(0.5, sps_, 6), dtype=torch.float64, device=dev)
        # the whole symbol stream up front, so the symbol clock and the
        # differential phase run on across chunks: symbol k of the stream is
        # centred on sample (k + 6) * FS / sym_rate (the RRC's 6-symbol delay)
        nsym_all = int(nsamples * sym_rate / FS_HZ) + 2
        sgen = torch.Generator(device=dev)
        sgen.manual_seed(int(seed) * 1000003 + 999331)
        qsyms = torch.randint(0, 4, (nsym_all,), generator=sgen, device=dev)
        # differential QPSK: symbol s advances the transmitted carrier phase by
        # 0, -90, +90 or 180 degrees; a receiver mixing with exp(+j w t) sees
        # the negated step, which its differential detector reports as s
        quarter = torch.remainder(torch.cumsum(torch.tensor([0, -1, 1, 2], device=dev)[qsyms], 0), 4)
        ph = math.pi / 4 + (math.pi / 2) * quarter.to(torch.float64)
        qiq = torch.complex(torch.cos(ph), torch.sin(ph))
    sigma = math.sqrt(0.5 / (10 ** (snr_db / 10)))
    out = torch.empty(nsamples, dtype=torch.int16, device=dev)
    phase = 0
    for c0 in range(0, nsamples, CHUNK):
        clen = min(CHUNK, nsamples - c0)
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(seed) * 1000003 + c0 // CHUNK)
        n = torch.arange(start + c0 - LEAD, start + c0 + clen, device=dev, dtype=torch.int64)
        shift = None
        if wow is not None:
            shift = wow[0] * torch.sin(n.to(torch.float64) * (2 * math.pi / wow[1]))
        ire = composite_ire(sysd, n, shift, pal8, bruch_line)
        base = _fftconv(ire, taps)[LEAD:]
        fhz = sysd.ire0 + base * sysd.hz_ire
        # FM phase as an exact integer accumulator (2^24 steps per cycle) so
        # the capture does not depend on floating-point summation order
        inc = torch.round(fhz * (PHASE_ONE / FS_HZ)).to(torch.int64)
        acc = phase + torch.cumsum(inc, 0)
        phase = int(torch.remainder(acc[-1], PHASE_ONE).item())
        sig = torch.cos(torch.remainder(acc, PHASE_ONE).to(torch.float64) * (2 * math.pi / PHASE_ONE))
        tsec = (n[LEAD:].to(torch.float64)) / FS_HZ
        dev_hz = 100e3
        for fc, ft, amp in ((sysd.audio_f[0], tones[0], 0.1), (sysd.audio_f[1], tones[1], 0.1)):
            if qpsk and fc == sysd.audio_f[1] and system == "NTSC":
                continue
            aph = 2 * math.pi * fc * tsec - (dev_hz / ft) * torch.cos(2 * math.pi * ft * tsec)
            sig = sig + amp * torch.cos(aph)
        if efm:
            e = _efm_wave(gen, c0, clen + 256, dev)
            sig = sig + 0.12 * _fftconv(e, efm_taps)[128:128 + clen]
        if qpsk:
            # upsampled symbols k0 .. k1 (the RRC reaches 12 symbols back), filtered,
            # evaluated at this chunk's absolute sample times
            rs = sym_rate * sps_ / FS_HZ
            k0 = int(c0 * sym_rate / FS_HZ) - 13
            k1 = int((c0 + clen) * sym_rate / FS_HZ) + 2
            up = torch.zeros((k1 - k0) * sps_, dtype=torch.complex128, device=dev)
            ka, kb = max(k0, 0), min(k1, nsym_all)
            if kb > ka:
                up[(ka - k0) * sps_:(kb - k0) * sps_:sps_] = qiq[ka:kb]
            bb = torch.complex(_fftconv(up.real, rrc), _fftconv(up.imag, rrc))
            ti = (torch.arange(c0, c0 + clen, device=dev, dtype=torch.float64) * rs) - k0 * sps_
            i0 = torch.clamp(ti.floor().to(torch.int64), 0, bb.shape[0] - 2)
            fr = ti - i0
            bbi = bb[i0] * (1 - fr) + bb[i0 + 1] * fr
            car = torch.exp(1j * 2 * math.pi * 2.88e6 * tsec)
            sig = sig + 0.15 * (bbi * car).real
        sig = sig + sigma * torch.randn(clen, generator=gen, device=dev, dtype=torch.float64)
        out[c0:c0 + clen] = torch.clamp(torch.round(sig * scale), -32768, 32767).to(torch.int16)
    if return_symbols:
        return out, (qsyms.to(torch.uint8).cpu().numpy() if qpsk else None)
    return out


def inject_dropouts(cap, seed, count, min_len=40, max_len=1200, level=30):
    """Replace `count` seeded spans of a capture (numpy int16 array or torch
    int16 tensor, in place) with low-level noise: the RF carrier lost for
    min_len..max_len samples, as a disc dropout looks.  Integer arithmetic
    only, so the result is the same on every CPU and device.  Returns the
    spans as (start, length) pairs, sorted."""
    n = int(cap.shape[0])
    rng = np.random.default_rng(seed)
    starts = np.sort(rng.integers(0, max(n - max_len, 1), count))
    lens = rng.integers(min_len, max_len + 1, count)
    spans = []
    for s0, ln in zip(starts.tolist(), lens.tolist()):
        ln = min(ln, n - s0)
        noise = rng.integers(-level, level + 1, ln).astype(np.int16)
        if isinstance(cap, torch.Tensor):
            cap[s0:s0 + ln] = torch.from_numpy(noise).to(cap.device)
        else:
            cap[s0:s0 + ln] = noise
        spans.append((s0, ln))
    return spans
