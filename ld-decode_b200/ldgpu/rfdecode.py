"""RFDecode: the reference decoder's RF demodulator API, running on the GPU.

Same constructor, attributes and methods as lddecode.core.RFDecode
(lddecode/core.py:253-1046) for the parts on the demod path:
`demodblock(data, mtf_level, fftdata, cut)` returns the same dict
({'rfhpf', 'video', 'efm', 'audio', 'setupcount'}) with the same record
layout, and `computefilters()`, `iretohz()`, `hztoire()`, `audio_phase2()`,
`computedelays()`, `Filters`, `audio`, `delays`, `limits`, `SysParams`,
`DecoderParams`, `linelen` ... behave as in the reference.  The filters
are designed on the host in FP64 (ldgpu.filters) and uploaded as float32
half spectra; every block is demodulated by the fused CUDA kernel behind
the C ABI (include/ldgpu.h).  There is no CPU fallback.
"""

import ctypes

import numpy as np

from . import filters as flt
from . import lib as L
from .hostmath import calczc, fm_wave
from .lut import build_sinc_lut
from .params import BLOCKSIZE, BLOCKCUT, filterparams, sysparams


def _slice_len(a, b, n):
    start, stop, _ = slice(a, b).indices(n)
    return start, max(0, stop - start)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class RFParams:
    """Host-only part of RFDecode: parameter tables and FP64 filter design
    (core.py:284-402, 405-737), without a GPU context."""

    def __init__(self, inputfreq=40, system="NTSC", blocklen=BLOCKSIZE,
                 decode_digital_audio=False, decode_analog_audio=0, has_analog_audio=True,
                 extra_options={}, decoder_params_override={}, _design=True):
        self.downscale_sinc_lut = build_sinc_lut()
        self.blocklen = blocklen
        self.blockcut = BLOCKCUT
        self.blockcut_end = 0
        self.system = system
        self.setupcount = 0

        self.NTSC_ColorNotchFilter = extra_options.get("NTSC_ColorNotchFilter", False)
        self.PAL_V4300D_NotchFilter = extra_options.get("PAL_V4300D_NotchFilter", False)
        lowband = extra_options.get("lowband", False)

        self.freq = inputfreq
        self.freq_half = inputfreq / 2
        self.freq_hz = self.freq * 1000000
        self.freq_hz_half = self.freq_hz / 2

        self.mtf_mult = extra_options.get("MTF_level", 1.0)
        self.mtf_offset = extra_options.get("MTF_offset", 0)

        self.SysParams = sysparams(system)
        self.DecoderParams = filterparams(system, lowband)
        for k in ("ire0", "hz_ire", "vsync_ire"):
            self.DecoderParams[k] = self.SysParams[k]
        for k, v in decoder_params_override.items():
            self.DecoderParams[k] = v

        self.SysParams["analog_audio"] = has_analog_audio
        self.SysParams["AC3"] = extra_options.get("AC3", False)
        if self.SysParams["AC3"]:
            self.SysParams["audio_rfreq"] = self.SysParams["audio_rfreq_AC3"]

        fw = extra_options.get("audio_filterwidth", 0)
        if fw is not None and fw > 0:
            self.DecoderParams["audio_filterwidth"] = fw

        deemp = list(self.DecoderParams["video_deemp"])
        deemp_low, deemp_high = extra_options.get("deemp_coeff", (0, 0))
        if deemp_low > 0:
            deemp[1] = 1 / (deemp_low * 1000000)
        if deemp_high > 0:
            deemp[0] = 1 / (deemp_high * 1000000)
        self.DecoderParams["video_deemp"] = deemp
        self.DecoderParams["video_deemp_strength"] = extra_options.get("deemp_str", 1.0)

        self.linelen = int(np.round(self.freq_hz / (1000000.0 / self.SysParams["line_period"])))
        self.samplesperline = self.freq / self.linelen
        self.hsync_tolerance = 0.4

        self.decode_digital_audio = decode_digital_audio
        self.decode_analog_audio = decode_analog_audio
        if _design:
            self.design_filters()
            self.blockcut_end = self.Filters["F05_offset"]

    def design_filters(self):
        self.computevideofilters()
        if self.decode_analog_audio != 0:
            self.computeaudiofilters()
        if self.decode_digital_audio:
            self.computeefmfilter()

    def computevideofilters(self):
        self.Filters = flt.design_video(self.system, self.SysParams, self.DecoderParams, self.freq,
                                        self.blocklen, self.NTSC_ColorNotchFilter)

    def computeaudiofilters(self):
        self.audio = flt.design_audio(self.SysParams, self.DecoderParams, self.freq, self.blocklen,
                                      self.Filters)

    def computeefmfilter(self):
        flt.design_efm(self.freq, self.blocklen, self.Filters)

    def iretohz(self, ire, spec=False):
        params = self.SysParams if spec else self.DecoderParams
        return params["ire0"] + (params["hz_ire"] * ire)

    def hztoire(self, hz, spec=False):
        params = self.SysParams if spec else self.DecoderParams
        return (hz - params["ire0"]) / params["hz_ire"]

    def scaled_mtf(self, mtf_level):
        """mtf_level as demodblock scales it (core.py:748-750)."""
        mtf_level *= self.mtf_mult
        mtf_level += self.mtf_offset
        mtf_level *= self.DecoderParams["MTF_basemult"]
        return mtf_level

    def output_slices(self, cut, rotdelay=None):
        """(start, len) of every output within an N-sample block, with the
        reference's slicing semantics (core.py:769-772, 843-875)."""
        n = self.blocklen
        if rotdelay is None:
            d = getattr(self, "delays", None)
            rotdelay = d.get("video_rot", 0) if d else 0
        hp = _slice_len(self.blockcut - rotdelay, -self.blockcut_end - rotdelay, n)
        vid = _slice_len(self.blockcut, -self.blockcut_end, n) if cut else (0, n)
        fdiv = n // 1024
        aud = _slice_len(self.blockcut // fdiv, -self.blockcut_end // fdiv, 1024) if cut else (0, 1024)
        return {"rfhpf": hp, "video": vid, "efm": vid, "audio": aud}


class RFDecode(RFParams):
    """GPU RF demodulator with the reference RFDecode interface."""

    def __init__(self, inputfreq=40, system="NTSC", blocklen=BLOCKSIZE,
                 decode_digital_audio=False, decode_analog_audio=0, has_analog_audio=True,
                 extra_options={}, decoder_params_override={}, device=0, fft_variant=None):
        super().__init__(inputfreq, system, blocklen, decode_digital_audio, decode_analog_audio,
                         has_analog_audio, extra_options, decoder_params_override, _design=False)
        self.device = device
        self._ctx = L.Context(system, blocklen, self.freq_hz, device)
        if fft_variant is not None:
            self.fft_variant = fft_variant
        if self.system == "PAL" and self.PAL_V4300D_NotchFilter:
            # the reference's search band (core.py:783-786)
            lo = int(self.blocklen * (8.42 / self.freq))
            hi = int(1 + (self.blocklen * (8.6 / self.freq)))
            L.check(self._ctx._lib.ldg_set_notch(self._ctx.handle, lo, hi))
        self._mtf_loaded = None
        self._lut_loaded = False
        self.computefilters()
        self.blockcut_end = self.Filters["F05_offset"]

    # ---- FFT decomposition of the demodulator (no counterpart in the reference)

    @property
    def fft_variant(self):
        """L.LDG_VARIANT_STOCKHAM or L.LDG_VARIANT_IN_PLACE (ldg_set_demod_variant)."""
        v = ctypes.c_int32()
        L.check(self._ctx._lib.ldg_get_demod_variant(self._ctx.handle, ctypes.byref(v)))
        return v.value

    @fft_variant.setter
    def fft_variant(self, v):
        L.check(self._ctx._lib.ldg_set_demod_variant(self._ctx.handle, int(v)))

    @property
    def blocks_per_cta(self):
        """Consecutive blocks a demodulator CTA takes (ldg_set_demod_schedule;
        0: the library's choice, 2 for large batches, else 1)."""
        return getattr(self, "_blocks_per_cta", 0)

    @blocks_per_cta.setter
    def blocks_per_cta(self, n):
        L.check(self._ctx._lib.ldg_set_demod_schedule(self._ctx.handle, int(n)))
        self._blocks_per_cta = int(n)

    # ---- filter upload (float32 half spectra)

    def computefilters(self):
        """(Re)compute the filter sets and delays (core.py:405-420)."""
        self.setupcount += 1
        self.design_filters()
        self._upload_filters()
        self.computedelays()

    def _set_filter(self, slot, f_half):
        buf = np.ascontiguousarray(np.stack([f_half.real, f_half.imag], axis=1).reshape(-1),
                                   dtype=np.float64)
        L.check(self._ctx._lib.ldg_set_filter(self._ctx.handle, slot, _ptr(buf), len(f_half)))

    def _upload_filters(self):
        F = self.Filters
        self._set_filter(L.LDG_F_RFHPF, flt.half_spectrum(F["Frfhpf"]))
        self._set_filter(L.LDG_F_DEMOD, flt.half_spectrum(F["FVideo"]))
        self._set_filter(L.LDG_F_05, flt.half_spectrum(F["FVideo05"]))
        self._set_filter(L.LDG_F_BURST, flt.half_spectrum(F["FVideoBurst"]))
        if self.system == "PAL":
            self._set_filter(L.LDG_F_PILOT, flt.half_spectrum(F["FVideoPilot"]))
        if "Fefm" in F:
            self._set_filter(L.LDG_F_EFM, flt.half_spectrum(F["Fefm"]))
        if self.decode_analog_audio != 0:
            self._set_filter(L.LDG_F_AUDIO2_LEFT, flt.half_spectrum(self.audio["left"].audio2_filter))
            self._set_filter(L.LDG_F_AUDIO2_RIGHT, flt.half_spectrum(self.audio["right"].audio2_filter))
            for ch, name in enumerate(("left", "right")):
                a = self.audio[name]
                f1 = np.ascontiguousarray(np.stack([a.filt1.real, a.filt1.imag], axis=1).reshape(-1))
                L.check(self._ctx._lib.ldg_set_audio(self._ctx.handle, ch, int(a.lowbin), int(a.nbins),
                                                     _ptr(f1), float(a.a1_freq), float(a.low_freq)))
        self._mtf_loaded = None

    def _load_mtf(self, mtf_level):
        """Upload RFVideo * MTF**mtf_level (core.py:800-803), FP64 product."""
        if self._mtf_loaded == mtf_level:
            return
        g = self.Filters["RFVideo"]
        if mtf_level != 0:
            g = g * (self.Filters["MTF"] ** mtf_level)
        m = self.blocklen // 2
        gh = np.ascontiguousarray(g[:m + 1])
        self._set_filter(L.LDG_F_VIDEO_G, gh)
        # odd output samples of the one-sided inverse: G[k] * exp(+2 pi i k / N)
        k = np.arange(m + 1)
        self._set_filter(L.LDG_F_VIDEO_G_ODD, gh * np.exp(2j * np.pi * k / self.blocklen))
        self._mtf_loaded = mtf_level

    def _load_lut(self):
        if not self._lut_loaded:
            lut = np.ascontiguousarray(self.downscale_sinc_lut, dtype=np.float32)
            L.check(self._ctx._lib.ldg_set_sinc_lut(self._ctx.handle, _ptr(lut), lut.shape[0], lut.shape[1]))
            self._lut_loaded = True

    # ---- demodulation

    def demodblock(self, data=None, mtf_level=0, fftdata=None, cut=False):
        """Demodulate one block (core.py:747-752); see demodblock_gpu."""
        return self.demodblock_gpu(data, self.scaled_mtf(mtf_level), fftdata, cut)

    def demodblock_gpu(self, data=None, mtf_level=0, fftdata=None, cut=False, _rotdelay=None):
        """One block through the fused GPU demodulator.  `mtf_level` is the
        already-scaled MTF exponent, as in demodblock_cpu (core.py:755-879)."""
        dev_block = None
        if fftdata is not None:
            # the spectrum takes precedence, as in the reference; its real
            # inverse is made on the GPU (ldg_blocks_from_spectra)
            import torch
            X = np.ascontiguousarray(np.asarray(fftdata, dtype=np.complex128))
            if len(X) != self.blocklen:
                raise ValueError(f"demodblock needs {self.blocklen} spectrum bins, got {len(X)}")
            dev = torch.device("cuda", self.device)
            dX = torch.from_numpy(X.view(np.float64)).to(dev)
            dev_block = torch.empty(self.blocklen, dtype=torch.float32, device=dev)
            torch.cuda.current_stream(dev).synchronize()  # the context's stream reads them next
            L.check(self._ctx._lib.ldg_blocks_from_spectra(self._ctx.handle, dX.data_ptr(), 1,
                                                           dev_block.data_ptr(), None))
            x = None
        elif data is not None:
            x = np.asarray(data)[: self.blocklen]
            if len(x) != self.blocklen:
                raise ValueError(f"demodblock needs {self.blocklen} samples, got {len(x)}")
        else:
            raise Exception("demodblock called without raw or FFT data")
        if dev_block is not None:
            kind = L.LDG_IN_FLOAT32
        elif x.dtype == np.int16:
            kind = L.LDG_IN_INT16
            x = np.ascontiguousarray(x)
        else:
            kind = L.LDG_IN_FLOAT32
            x = np.ascontiguousarray(x, dtype=np.float32)
        self._load_mtf(mtf_level)
        sl = self.output_slices(cut, _rotdelay)
        vlen = sl["video"][1]
        out = {k: np.empty(vlen, dtype=np.float32) for k in ("demod", "demod_raw", "demod_05", "demod_burst")}
        if self.system == "PAL":
            out["demod_pilot"] = np.empty(vlen, dtype=np.float32)
        rfhpf = np.empty(sl["rfhpf"][1], dtype=np.float32)
        efm = np.empty(sl["efm"][1], dtype=np.int16) if self.decode_digital_audio else None
        alen = sl["audio"][1]
        al = np.empty(alen, dtype=np.float32) if self.decode_analog_audio else None
        ar = np.empty(alen, dtype=np.float32) if self.decode_analog_audio else None

        a = L.DemodArgs()
        a.in_ = dev_block.data_ptr() if dev_block is not None else x.ctypes.data
        a.in_kind = kind
        a.in_stride = self.blocklen
        a.nblocks = 1
        a.out_demod = out["demod"].ctypes.data if vlen else None
        a.out_raw = out["demod_raw"].ctypes.data if vlen else None
        a.out_05 = out["demod_05"].ctypes.data if vlen else None
        a.out_burst = out["demod_burst"].ctypes.data if vlen else None
        a.out_pilot = out["demod_pilot"].ctypes.data if (vlen and self.system == "PAL") else None
        a.out_rfhpf = rfhpf.ctypes.data if len(rfhpf) else None
        a.out_efm = efm.ctypes.data if (efm is not None and len(efm)) else None
        a.out_audio_left = al.ctypes.data if (al is not None and alen) else None
        a.out_audio_right = ar.ctypes.data if (ar is not None and alen) else None
        a.video = L.Slice(sl["video"][0], vlen, 0)
        a.roll_05 = int(self.Filters["F05_offset"])
        a.roll_burst = int(self.Filters["FVideoBurst_offset"])
        a.rfhpf = L.Slice(sl["rfhpf"][0], sl["rfhpf"][1], 0)
        a.efm = L.Slice(sl["efm"][0], sl["efm"][1] if efm is not None else 0, 0)
        a.audio = L.Slice(sl["audio"][0], alen if al is not None else 0, 0)
        a.stream = None
        L.check(self._ctx._lib.ldg_demod_blocks(self._ctx.handle, ctypes.byref(a)))

        rv = {"rfhpf": rfhpf}
        names = ["demod", "demod_raw", "demod_05", "demod_burst"]
        if self.system == "PAL":
            names.append("demod_pilot")
        rv["video"] = np.rec.fromarrays([out[k] for k in names], names=names)
        if efm is not None:
            rv["efm"] = efm
        if self.decode_analog_audio:
            rv["audio"] = np.rec.fromarrays([al, ar], names=["audio_left", "audio_right"])
        rv["setupcount"] = self.setupcount
        return rv

    def demod_args(self, in_ptr, nblocks, in_stride, outs, mtf_level=0, cut=True, in_kind=L.LDG_IN_INT16,
                   stream=None):
        """ldg_demod_args for a device batch (see demod_blocks_device); loads
        the filters of `mtf_level` into the context."""
        self._load_mtf(self.scaled_mtf(mtf_level))
        sl = self.output_slices(cut)
        a = L.DemodArgs()
        a.in_ = in_ptr
        a.in_kind = in_kind
        a.in_stride = int(in_stride)
        a.nblocks = int(nblocks)
        a.out_demod = outs.get("demod")
        a.out_raw = outs.get("demod_raw")
        a.out_05 = outs.get("demod_05")
        a.out_burst = outs.get("demod_burst")
        a.out_pilot = outs.get("demod_pilot")
        a.out_rfhpf = outs.get("rfhpf")
        a.out_efm = outs.get("efm")
        a.out_audio_left = outs.get("audio_left")
        a.out_audio_right = outs.get("audio_right")
        a.video = L.Slice(sl["video"][0], sl["video"][1], 0)
        a.roll_05 = int(self.Filters["F05_offset"])
        a.roll_burst = int(self.Filters["FVideoBurst_offset"])
        a.rfhpf = L.Slice(sl["rfhpf"][0], sl["rfhpf"][1] if outs.get("rfhpf") else 0, 0)
        a.efm = L.Slice(sl["efm"][0], sl["efm"][1] if outs.get("efm") else 0, 0)
        has_audio = outs.get("audio_left") or outs.get("audio_right")
        a.audio = L.Slice(sl["audio"][0], sl["audio"][1] if has_audio else 0, 0)
        a.stream = stream
        return a, sl

    def demod_blocks_device(self, in_ptr, nblocks, in_stride, outs, mtf_level=0, cut=True,
                            in_kind=L.LDG_IN_INT16, stream=None):
        """Batched form: demodulate `nblocks` blocks whose inputs and outputs
        already live in device memory.  `outs` maps output names (demod,
        demod_raw, demod_05, demod_burst, demod_pilot, rfhpf, efm,
        audio_left, audio_right) to device pointers laid out block after
        block; `mtf_level` is unscaled, as for demodblock.  Only enqueues."""
        a, sl = self.demod_args(in_ptr, nblocks, in_stride, outs, mtf_level, cut, in_kind, stream)
        L.check(self._ctx._lib.ldg_demod_blocks(self._ctx.handle, ctypes.byref(a)))
        return sl

    # ---- second-stage audio (per field, host FP64 as in the reference)

    def _phase2_segments(self, left, right, starts):
        """ldg_audio_phase2 over transforms of `blocklen` samples starting at
        `starts` (each clipped to the input); float32 results per start."""
        import torch
        dev = torch.device("cuda", self.device)
        n = len(left)
        tl = torch.from_numpy(np.ascontiguousarray(left, np.float32)).to(dev)
        tr = torch.from_numpy(np.ascontiguousarray(right, np.float32)).to(dev)
        lens = [min(self.blocklen, n - s0) for s0 in starts]
        outs = torch.empty((2, max(1, sum(lens))), dtype=torch.float32, device=dev)
        segs = (L.Audio2Segment * len(starts))()
        off = 0
        for i, (s0, ln) in enumerate(zip(starts, lens)):
            segs[i].left = tl.data_ptr() + 4 * s0
            segs[i].right = tr.data_ptr() + 4 * s0
            segs[i].len = ln
            segs[i].out_left = outs[0].data_ptr() + 4 * off
            segs[i].out_right = outs[1].data_ptr() + 4 * off
            off += ln
        torch.cuda.synchronize(dev)
        L.check(self._ctx._lib.ldg_audio_phase2(self._ctx.handle, segs, len(starts),
                                                float(self.SysParams["audio_lfreq"]),
                                                float(self.SysParams["audio_rfreq"]), 1))
        h = outs.cpu().numpy()
        res, off = [], 0
        for ln in lens:
            res.append((h[0, off:off + ln], h[1, off:off + ln]))
            off += ln
        return res

    def runfilter_audio_phase2(self, frame_audio, start):
        """core.py:884-915 on the GPU (ldg_audio_phase2): one transform of
        `blocklen` stage-1 samples from `start`."""
        left = np.asarray(frame_audio["audio_left"])
        right = np.asarray(frame_audio["audio_right"])
        (l, r), = self._phase2_segments(left, right, [start])
        return np.rec.array([l, r], names=["audio_left", "audio_right"])

    def audio_phase2(self, field_audio):
        """core.py:917-950: every transform of the stitching in one GPU
        launch, stitched as the reference does (512 samples dropped at each
        join)."""
        left = np.asarray(field_audio["audio_left"])
        right = np.asarray(field_audio["audio_right"])
        n = len(left)
        askip = 512
        sjump = self.blocklen - askip
        if n <= self.blocklen:
            starts = [0]
        else:
            starts = [0] + list(range(sjump, n - sjump, sjump)) + [n - self.blocklen - 1]
        segs = self._phase2_segments(left, right, starts)
        if len(segs[0][0]) >= n:
            # one transform: the reference returns its FP64 result as is
            return np.rec.array([segs[0][0][:n].astype(np.float64), segs[0][1][:n].astype(np.float64)],
                                names=["audio_left", "audio_right"])
        out = np.zeros(n, dtype=field_audio.dtype)
        out["audio_left"][:len(segs[0][0])] = segs[0][0]
        out["audio_right"][:len(segs[0][1])] = segs[0][1]
        ostart = len(segs[0][0])
        for l, r in segs[1:-1]:
            oend = ostart + len(l) - askip
            out["audio_left"][ostart:oend] = l[askip:]
            out["audio_right"][ostart:oend] = r[askip:]
            ostart += len(l) - askip
        l, r = segs[-1]
        out["audio_left"][n - (len(l) - askip):] = l[askip:]
        out["audio_right"][n - (len(r) - askip):] = r[askip:]
        return out.view(np.recarray)

    # ---- init-time delay calibration (core.py:952-1046), on the GPU

    def computedelays(self, mtf_level=0):
        """Demodulate a synthetic block (sync, burst, white, a 5-sample
        dropout) and measure the filter delays from it."""
        n = self.blocklen
        dp = self.DecoderParams
        fake = np.zeros(n, dtype=np.double)
        fake[:] = self.iretohz(0)
        synclen = int(4.7 * self.freq)
        fake[1500:1500 + synclen] = self.iretohz(dp["vsync_ire"])
        fake[2000:2000 + synclen] = self.iretohz(dp["vsync_ire"])
        porch_end = 2000 + synclen + int(0.6 * self.freq)
        burst_end = porch_end + int(1.2 * self.freq)
        fsc = self.SysParams["fsc_mhz"]
        fake[porch_end:burst_end] += fm_wave(np.full(burst_end - porch_end, fsc), self.freq / 2) * dp["hz_ire"] * 20
        fake[3000:3500] = self.iretohz(100)
        fake[4500:5000] = self.iretohz(100)
        fake[4200:5500] += fm_wave(np.full(5500 - 4200, fsc), self.freq / 2) * dp["hz_ire"] * 20
        fake[2000:2000 + synclen] = self.iretohz(dp["vsync_ire"]) + (
            fm_wave(np.full(synclen, fsc), self.freq / 2) * dp["hz_ire"] * dp["vsync_ire"])

        spec = np.fft.fft(fake) * self.Filters["Fvideo_lpf"] * self.Filters["Femp"]
        emp = np.fft.ifft(spec).real
        sig = fm_wave(emp, self.freq_hz / 2)
        sig *= 4096
        sig += 8192
        sig[6000:6005] = 0

        rotdelay = self.delays["video_rot"] if getattr(self, "delays", None) else 0
        dec = self.demodblock_gpu(sig, mtf_level=mtf_level, cut=False, _rotdelay=rotdelay)
        vdemod = dec["video"]["demod"]
        vraw = dec["video"]["demod_raw"]
        vsync_cross = self.iretohz(dp["vsync_ire"] / 2)
        self.delays = {
            "video_sync": calczc(vdemod, 1500, vsync_cross, count=512) - 1500,
            "video_white": calczc(vdemod, 3000, self.iretohz(50), count=512) - 3000,
            "video_rot": int(np.round(calczc(vdemod, 6000, self.iretohz(-10), count=512) - 6000)),
        }
        self.limits = {
            "sync": (np.min(vraw[1400:2800]), np.max(vraw[1400:2800])),
            "viewable": (np.min(vraw[2900:6000]), np.max(vraw[2900:6000])),
        }
        return dec, emp

    def demod_status(self):
        """Raise if a demodulator block was skipped since the last check
        (a wait for its scratch slot gave up); synchronous."""
        flags = ctypes.c_int32(0)
        L.check(self._ctx._lib.ldg_demod_status(self._ctx.handle, ctypes.byref(flags)))

    def synchronize(self):
        """Wait for the work queued on the context's own stream."""
        L.check(self._ctx._lib.ldg_synchronize(self._ctx.handle))

    def close(self):
        self._ctx.close()
