"""CPU oracle for one demodulator block -- TEST INFRASTRUCTURE ONLY.

A complex128 numpy restatement of the reference's per-block RF
demodulator, RFDecode.demodblock_cpu (lddecode/core.py:755-879), and of
the conjugate-product FM discriminator unwrap_hilbert
(lddecode/utils.py:898-926).  It is imported only by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the checker
of the CUDA path; nothing in the product calls it.

Parity of this oracle is pinned against the reference itself: the fixtures
in tests/golden/ were produced by running the unmodified reference on the
same seeded inputs (tests/golden/make_golden.py), and
tests/test_oracle_golden.py checks this file against them.
"""

import numpy as np

TAU = 2 * np.pi


def fm_discriminate(z, rate_hz):
    """Instantaneous frequency in [0, rate_hz) of analytic signal z:
    arg(z[n] * conj(z[n-1])) wrapped to [0, 2pi) and scaled by rate/2pi,
    with out[0] = 0 (utils.py:916-926)."""
    out = np.empty(len(z), dtype=np.float64)
    out[0] = 0.0
    d = np.angle(z[1:] * np.conj(z[:-1]))
    out[1:] = np.where(d < 0.0, d + TAU, d)
    return out * (rate_hz / TAU)


def audio_slice(spec, lowbin, nbins, blocklen):
    """fft_do_slice (utils.py:953-962)."""
    h = nbins // 2
    return np.concatenate([spec[lowbin:lowbin + h],
                           spec[blocklen - lowbin - h:blocklen - lowbin]])


def notch_v4300d(X, blocklen, freq_mhz):
    """PAL_V4300D_NotchFilter (core.py:774-798): in 8.42-8.6 MHz, bins whose
    magnitude exceeds mean + 3 std of the band are zeroed with their two
    neighbours and the mirrored negative-frequency bins.  Returns a copy."""
    X = np.array(X, copy=True)
    sl = slice(int(blocklen * (8.42 / freq_mhz)), int(1 + (blocklen * (8.6 / freq_mhz))))
    sq = np.sqrt(X[sl].real ** 2 + X[sl].imag ** 2)
    m = np.mean(sq) + (np.std(sq) * 3)
    for i in np.where(sq > m)[0]:
        for d in (-1, 0, 1):
            X[i + d + sl.start] = 0
            X[blocklen - (i + d + sl.start)] = 0
    return X


def demodblock(data, filters, system="NTSC", freq_hz=40e6, blocklen=32768,
               blockcut=1024, blockcut_end=32, video_rot=3, mtf_level=0.0,
               cut=True, efm=False, audio=None, fftdata=None, pal_notch=False, out_dtype=np.float32):
    """Restatement of RFDecode.demodblock_cpu (core.py:755-879).

    `mtf_level` is the already-scaled exponent (core.py:747-752 applies the
    MTF_level/offset/basemult scaling before calling demodblock_cpu).
    `audio` is None or a dict {'left': ns, 'right': ns} with lowbin, nbins,
    a1_freq, low_freq and filt1 per channel.  Returns a dict with the same
    keys the reference returns; 'video' is a dict of float32 arrays instead
    of a record array.  `out_dtype=np.float64` keeps the video and rfhpf
    outputs in FP64 (the reference casts them to float32) for error
    statistics.
    """
    F = filters
    if fftdata is not None:
        X = fftdata
    elif data is not None:
        X = np.fft.fft(np.asarray(data[:blocklen], dtype=np.float64))
    else:
        raise Exception("demodblock called without raw or FFT data")

    rv = {}
    hp = np.fft.ifft(X * F["Frfhpf"]).real
    end = -blockcut_end - video_rot
    rv["rfhpf"] = hp[blockcut - video_rot:end if end != 0 else None].astype(out_dtype)

    if pal_notch and system == "PAL":
        X = notch_v4300d(X, blocklen, freq_hz / 1e6)

    Y = X * F["RFVideo"]
    if mtf_level != 0:
        Y = Y * (F["MTF"] ** mtf_level)
    demod = fm_discriminate(np.fft.ifft(Y), freq_hz)

    D = np.fft.fft(np.clip(demod, 1500000, freq_hz * 0.75))
    video = np.fft.ifft(D * F["FVideo"]).real
    v05 = np.roll(np.fft.ifft(D * F["FVideo05"]).real, -F["F05_offset"])
    vburst = np.roll(np.fft.ifft(D * F["FVideoBurst"]).real, -F["FVideoBurst_offset"])
    out = {
        "demod": video.astype(out_dtype),
        "demod_raw": demod.astype(out_dtype),
        "demod_05": v05.astype(out_dtype),
        "demod_burst": vburst.astype(out_dtype),
    }
    if system == "PAL":
        out["demod_pilot"] = np.fft.ifft(D * F["FVideoPilot"]).real.astype(out_dtype)
    if cut:
        out = {k: v[blockcut:-blockcut_end] for k, v in out.items()}
    rv["video"] = out

    if efm:
        e = np.fft.ifft(X * F["Fefm"])
        if cut:
            e = e[blockcut:-blockcut_end]
        rv["efm"] = np.int16(np.clip(e.real, -32768, 32767))

    if audio is not None:
        chans = []
        for ch in ("left", "right"):
            a = audio[ch]
            a1 = np.fft.ifft(audio_slice(X, a.lowbin, a.nbins, blocklen) * a.filt1)
            chans.append((fm_discriminate(a1, a.a1_freq) + a.low_freq).astype(out_dtype))
        fdiv = blocklen // len(chans[0])
        if cut:
            chans = [c[blockcut // fdiv:-blockcut_end // fdiv] for c in chans]
        rv["audio"] = {"audio_left": chans[0], "audio_right": chans[1]}
    return rv
