"""Host-side FP64 design of the demodulator's frequency-domain filters.

The filters are designed once per RFDecode (and again whenever the decoder
parameters change) with scipy.signal on the host, exactly as the reference
designs them (lddecode/core.py:405-737, utils.py:763-962): same scipy
calls, same arguments, same products.  Only their single-precision copies
travel to the GPU (see `half_spectrum` and `FilterSet.device_arrays`).
"""

import math
import types

import numpy as np
import scipy.interpolate as spi
import scipy.signal as sps


def freqresp(b, a, n):
    """Whole-circle frequency response of B/A sampled on n FFT bins
    (utils.py:782-783, filtfft)."""
    return sps.freqz(b, a, n, whole=1)[1]


def emphasis_ba(t1, t2, fs):
    """First-order shelving (pre/de)emphasis as an IIR (b, a) pair: a zero at
    1/t1 and a pole at 1/t2, bilinear-transformed with pre-warping
    (utils.py:766-778)."""
    w1 = 2 * fs * np.tan((1 / t1) / (2 * fs))
    w2 = 2 * fs * np.tan((1 / t2) / (2 * fs))
    b, a = sps.zpk2tf([-w1], [-w2], w2 / w1)
    return sps.bilinear(b, a, fs)


def analytic_mask(n):
    """One-sided spectrum weights (1, 2, ..., 2, 1, 0, ..., 0) that turn a
    real signal's spectrum into its analytic signal's (utils.py:882-890)."""
    if n % 2:
        raise ValueError("analytic_mask: n must be even")
    m = np.zeros(n)
    m[0] = m[n // 2] = 1
    m[1:n // 2] = 2
    return m


def _supergauss(x, width, order, center):
    return np.exp(-2 * np.power(
        (2 * (x - center) * (math.log(2.0) / 2.0) ** (1 / (2 * order))) / width,
        2 * order))


def supergauss_band(f_lo, f_hi, order, nyquist_hz, n):
    """Symmetric super-Gaussian band window over n bins (utils.py:859-877)."""
    half = _supergauss(np.linspace(0, nyquist_hz, n // 2 + 1),
                       f_hi - f_lo, order, (f_hi + f_lo) / 2.0)[:-1]
    return np.concatenate([half, np.flip(half)])


def audio_bin_slice(center_hz, min_bw_hz, fs_hz, nbins_in):
    """(lowbin, nbins, decimated_rate) of the FFT sub-band that holds an audio
    carrier +/- min_bw (utils.py:929-950)."""
    binwidth = fs_hz / nbins_in
    cbin = int(np.round(center_hz / binwidth))
    bbins = int(np.round(min_bw_hz / binwidth))
    nbins = 2 * (2 ** math.ceil(math.log2(bbins * 2)))
    return cbin - nbins // 4, nbins, binwidth * nbins


def take_audio_bins(spec, lowbin, nbins, blocklen):
    """Cut the positive band [lowbin, lowbin+nbins/2) and its mirror
    (utils.py:953-962)."""
    h = nbins // 2
    return np.concatenate([spec[lowbin:lowbin + h],
                           spec[blocklen - lowbin - h:blocklen - lowbin]])


def half_spectrum(f):
    """Bins 0..N/2 of the Hermitian part of a whole-circle response f.

    For a real input signal x with spectrum X, Re(ifft(X * f)) equals the
    real inverse transform of X[k] * h[k] (k = 0..N/2) with
    h[k] = (f[k] + conj(f[N-k])) / 2 and h[0], h[N/2] real.  This is how
    every ".real" output of demodblock (core.py:769, 811-820, 848) is
    carried to the GPU's real-output transforms; for a Hermitian f it is f
    itself, for a one-sided f (the EFM equaliser) it is f / 2.
    """
    n = len(f)
    m = n // 2
    h = np.empty(m + 1, dtype=np.complex128)
    k = np.arange(1, m)
    h[1:m] = 0.5 * (f[k] + np.conj(f[n - k]))
    h[0] = f[0].real
    h[m] = f[m].real
    return h


class FilterSet:
    """The filter bank of one RFDecode configuration (FP64, whole circle).

    Attribute names follow the reference's Filters dict keys.
    """

    def __init__(self, filters, audio):
        self.Filters = filters
        self.audio = audio


def _notch_band(f, width, fs_half_hz):
    return [(f - width) / fs_half_hz, (f + width) / fs_half_hz]


def group_delay_equalizer(system, lpf_resp, blocklen, fs, lpf_freq):
    """Unit-magnitude all-pass whose group delay brings the video LPF onto
    the IEC 60856 (PAL) / IEC 60857 (NTSC) curve (core.py:480-542)."""
    bf = np.abs(np.fft.fftfreq(blocklen, 1.0 / fs))
    if system == "PAL":
        knots_f = np.array([0.0, 0.5e6, 2.0e6, 3.0e6, 4.0e6, 4.4336e6, 4.8e6, 5.5e6])
        knots_t = np.array([0.0, 0.0, 10e-9, 35e-9, 85e-9, 135e-9, 200e-9, 200e-9])
    else:
        knots_f = np.array([0.0, 0.5e6, 2.0e6, 3.0e6, 3.58e6, 4.0e6, 4.2e6, 4.8e6])
        knots_t = np.array([0.0, 0.0, 15e-9, 45e-9, 80e-9, 135e-9, 200e-9, 200e-9])
    target = np.interp(bf, knots_f, knots_t)

    ph = np.unwrap(np.angle(lpf_resp))
    gd = -np.gradient(ph) / (2 * np.pi * (fs / blocklen))
    ref_bin = np.argmin(np.abs(bf - 0.5e6))
    resid = target - (gd - gd[ref_bin])

    lo, hi = lpf_freq + 0.3e6, lpf_freq + 1.3e6
    resid = resid * np.clip((hi - bf) / (hi - lo), 0.0, 1.0)
    resid[bf < 0.4e6] = 0.0

    half = blocklen // 2
    phi = -2 * np.pi * np.cumsum(resid[:half + 1]) * (fs / blocklen)
    eq = np.ones(blocklen, dtype=complex)
    eq[:half + 1] = np.exp(1j * phi)
    eq[half + 1:] = np.conj(eq[1:half][::-1])
    eq[0] = 1.0
    eq[half] = 1.0
    return eq


def design_video(system, sp, dp, freq_mhz, blocklen, ntsc_color_notch=False):
    """Video, RF high-pass, MTF and sync/burst/pilot filters
    (core.py:544-679)."""
    fs = freq_mhz * 1e6
    fs_half = fs / 2
    f_half_mhz = freq_mhz / 2
    F = {}

    b, a = sps.butter(1, 10 / f_half_mhz, btype="highpass")
    F["Frfhpf"] = freqresp(b, a, blocklen)

    # MTF compensation: two poles mirrored about fs/4
    plo = dp["MTF_freq"] / f_half_mhz
    phi = (f_half_mhz + (f_half_mhz - dp["MTF_freq"])) / f_half_mhz
    pole = lambda p: dp["MTF_poledist"] * np.exp(1j * (np.pi * p))
    b, a = sps.zpk2tf([], [pole(plo), pole(phi)], 1)
    F["MTF"] = freqresp(b, a, blocklen)

    if "video_bpf_low_order" in dp:
        b1, a1 = sps.butter(dp["video_bpf_low_order"], dp["video_bpf_low"] / fs_half,
                            btype="highpass")
        b2, a2 = sps.butter(dp["video_bpf_high_order"], dp["video_bpf_high"] / fs_half,
                            btype="lowpass")
        F["RFVideo"] = freqresp(b1, a1, blocklen) * freqresp(b2, a2, blocklen)
    else:
        b, a = sps.butter(dp["video_bpf_order"],
                          [dp["video_bpf_low"] / fs_half, dp["video_bpf_high"] / fs_half],
                          btype="bandpass")
        F["RFVideo"] = freqresp(b, a, blocklen)

    if sp["analog_audio"] and system == "NTSC":
        b, a = sps.butter(dp["audio_notchorder"],
                          _notch_band(sp["audio_lfreq"], dp["audio_notchwidth"], fs_half),
                          btype="bandstop")
        F["Fcutl"] = freqresp(b, a, blocklen)
        b, a = sps.butter(dp["audio_notchorder"],
                          _notch_band(sp["audio_rfreq"], dp["audio_notchwidth"], fs_half),
                          btype="bandstop")
        F["Fcutr"] = freqresp(b, a, blocklen)
        F["RFVideo"] *= F["Fcutl"] * F["Fcutr"]

    F["hilbert"] = analytic_mask(blocklen)
    F["RFVideo"] *= F["hilbert"]

    b, a = sps.butter(dp["video_lpf_order"], dp["video_lpf_freq"] / fs_half, "low")
    F["Fvideo_lpf"] = freqresp(b, a, blocklen)
    if system == "NTSC" and ntsc_color_notch:
        b, a = sps.butter(3, [dp["video_lpf_freq"] / 1000000 / f_half_mhz, 5.0 / f_half_mhz],
                          "bandstop")
        F["Fvideo_lpf"] *= freqresp(b, a, blocklen)

    t_hi, t_lo = dp["video_deemp"]
    b, a = emphasis_ba(t_hi, t_lo, fs)
    F["Fdeemp"] = freqresp(b, a, blocklen)
    b, a = emphasis_ba(t_lo, t_hi, fs)
    F["Femp"] = freqresp(b, a, blocklen)

    F["FVideo"] = F["Fvideo_lpf"] * (F["Fdeemp"] ** dp["video_deemp_strength"])
    F["FVideoGD"] = group_delay_equalizer(system, F["Fvideo_lpf"], blocklen, fs,
                                          dp["video_lpf_freq"])
    F["FVideo"] = F["FVideo"] * F["FVideoGD"]

    taps05 = sps.firwin(65, [0.5 / f_half_mhz], pass_zero=True)
    F["F05_offset"] = 32
    F["FVideo05"] = F["Fvideo_lpf"] * F["Fdeemp"] * freqresp(taps05, [1.0], blocklen)

    fsc = sp["fsc_mhz"]
    tapsb = sps.firwin(81, [(fsc - 0.2) / f_half_mhz, (fsc + 0.2) / f_half_mhz],
                       pass_zero=False)
    F["FVideoBurst_offset"] = 40
    F["Fburst"] = freqresp(tapsb, [1.0], blocklen)
    F["FVideoBurst"] = F["Fvideo_lpf"] * F["Fdeemp"] * F["Fburst"]

    if system == "PAL":
        pil = sp["pilot_mhz"]
        b, a = sps.butter(1, [(pil - 0.1) / f_half_mhz, (pil + 0.1) / f_half_mhz],
                          btype="bandpass")
        F["Fpilot"] = freqresp(b, a, blocklen)
        F["FVideoPilot"] = F["Fvideo_lpf"] * F["Fdeemp"] * F["Fpilot"]
    return F


def design_audio(sp, dp, freq_mhz, blocklen, F):
    """Two analog-audio carriers: stage-1 band slice + FIR + analytic mask,
    stage-2 LPF + 75 us de-emphasis (core.py:681-737)."""
    fs = freq_mhz * 1e6
    audio = {}
    for ch, fc in (("left", sp["audio_lfreq"]), ("right", sp["audio_rfreq"])):
        a = types.SimpleNamespace()
        fir = sps.firwin(dp["audio_filterorder"],
                         _notch_band(fc, dp["audio_filterwidth"], fs / 2),
                         pass_zero=False)
        resp = freqresp(fir, 1.0, blocklen)
        a.lowbin, a.nbins, a.a1_freq = audio_bin_slice(fc, 200000, fs, blocklen)
        a.low_freq = fs * (a.lowbin / blocklen)
        a.filt1 = take_audio_bins(resp, a.lowbin, a.nbins, blocklen) * analytic_mask(a.nbins)
        order, wn = sps.buttord(20000 / (a.a1_freq / 2), 24000 / (a.a1_freq / 2), 1, 9)
        b, aa = sps.butter(order, wn)
        lpf = freqresp(b, aa, blocklen)
        b, aa = emphasis_ba(5.3e-6, 75e-6, a.a1_freq)
        a.audio2_filter = lpf * freqresp(b, aa, blocklen)
        audio[ch] = a
        F["audio_fdiv"] = blocklen // a.nbins
    return audio


def design_efm(freq_mhz, blocklen, F):
    """EFM equaliser: cubic-interpolated amplitude/phase table times 8 and a
    super-Gaussian band window (core.py:422-465)."""
    fs = freq_mhz * 1e6
    knots = np.linspace(0.0e6, 1.9e6, num=11)
    per_bin = fs / blocklen
    amp = np.array([0.0, 0.215, 0.41, 0.73, 0.98, 1.03, 0.99, 0.81, 0.59, 0.42, 0.0])
    phase = np.array([0.0, -0.92, -1.03, -1.11, -1.2, -1.2, -1.2, -1.2, -1.05, -0.95, -0.8])
    phase = [p * 1.25 for p in phase]
    coeffs = np.zeros(blocklen, dtype=complex)
    amp_i = spi.interp1d(knots, amp, kind="cubic")
    ph_i = spi.interp1d(knots, phase, kind="cubic")
    nz = int(knots[-1] / per_bin) + 1
    bf = np.arange(nz) * per_bin
    ba, bp = amp_i(bf), ph_i(bf)
    coeffs[:nz] = ba * (np.cos(bp) + (complex(0, -1) * np.sin(bp)))
    F["Fefm"] = coeffs * 8
    F["Fefm"] *= supergauss_band(20000, 1600000, 60, 20000000, 32768)
