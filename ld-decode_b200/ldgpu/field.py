"""Field: per-field line locations and time-base correction.

Mirrors lddecode.core.Field / FieldNTSC / FieldPAL (lddecode/core.py:
1587-3495).  `downscale()` keeps the reference signature
(core.py:2626-2722) and returns (dsout, dsaudio, efmout); the resampling
(computewow_scaled + scale_field + hz_to_output_array) runs on the GPU
through ldg_tbc_fields, and the analog audio through ldg_audio_downscale.
process() runs the GPU line path on the field's read (sync-run scan,
native field chain, GPU refinement, field phase IDs); a read that needs the
previous field's refined line locations or the reference's level
re-calibration is decoded by the host restatement in ldgpu.linelocs, as in
the batched path.
"""

import ctypes

import numpy as np

from . import lib as L
from .linelocs import FieldLogic, FieldLogicNTSC, FieldLogicPAL


def tbc_descriptor(rf, buf, linelocs, lineoffset, outwidth, linesout, outlinecount, levels,
                   out_u16=None, out_f32=None, coord_f32=False, buf_len=None, nlines=None, wow_smoothing=0.0,
                   wow_interpolation_method="linear"):
    """Fill an ldg_tbc_field from numpy arrays or raw device pointers (ints;
    then buf_len / nlines must be given).

    `levels` = (ire0, hz_ire, vsync_ire, out_scale, output_zero);
    `wow_interpolation_method` "linear", "quadratic" or "cubic"."""
    if wow_interpolation_method not in L.WOW_METHODS:
        raise ValueError(f"unknown wow_interpolation_method {wow_interpolation_method!r}")
    d = L.TbcField()
    d.buf = buf if isinstance(buf, int) else buf.ctypes.data
    d.buf_len = int(buf_len if buf_len is not None else len(buf))
    d.linelocs = linelocs if isinstance(linelocs, int) else linelocs.ctypes.data
    d.nlines = int(nlines if nlines is not None else len(linelocs))
    d.lineoffset = int(lineoffset)
    d.outwidth = int(outwidth)
    d.linesout = int(linesout)
    d.outlinecount = int(outlinecount)
    d.coord_f32 = 1 if coord_f32 else 0
    d.inlinelen = float(rf.linelen)
    d.outlinelen = float(rf.SysParams["outlinelen"])
    d.ire0, d.hz_ire, d.vsync_ire, d.out_scale, d.output_zero = [float(v) for v in levels]
    d.out_f32 = None if out_f32 is None else (out_f32 if isinstance(out_f32, int) else out_f32.ctypes.data)
    d.out_u16 = None if out_u16 is None else (out_u16 if isinstance(out_u16, int) else out_u16.ctypes.data)
    d.wow_smoothing = float(wow_smoothing or 0.0)
    d.wow_interp = L.WOW_METHODS[wow_interpolation_method]
    return d


def tbc_fields(rf, descs, stream=None, asynchronous=False):
    """Run ldg_tbc_fields on a list (or prebuilt ctypes array) of descriptors;
    asynchronous=True: ldg_tbc_fields_async (device buffers only; errors come
    from tbc_status).  `stream`: a raw handle; None runs on torch's default
    stream (cudaStreamLegacy), so that device inputs written there (line
    locations, demodulator outputs) are complete first."""
    rf._load_lut()
    arr = descs if isinstance(descs, ctypes.Array) else (L.TbcField * len(descs))(*descs)
    fn = rf._ctx._lib.ldg_tbc_fields_async if asynchronous else rf._ctx._lib.ldg_tbc_fields
    L.check(fn(rf._ctx.handle, arr, len(arr), stream if stream else 1))


def tbc_status(rf):
    """Raise if an asynchronous TBC batch hit a tap outside its field buffer
    (or had too many lines) since the last check; synchronous."""
    flags = ctypes.c_int32(0)
    L.check(rf._ctx._lib.ldg_tbc_status(rf._ctx.handle, ctypes.byref(flags)))


class Field(FieldLogic):
    """A decoded field (core.py:1587-1635 constructor arguments)."""

    # coordinates rounded to float32 as the reference does (utils.py:160);
    # False keeps them in FP64 (the accuracy target)
    coord_f32 = False

    def levels(self):
        return (self.rf.DecoderParams["ire0"], self.rf.DecoderParams["hz_ire"],
                self.rf.DecoderParams["vsync_ire"], self.out_scale, self.rf.SysParams["outputZero"])

    def hz_to_output(self, input):
        """core.py:1714-1734 (array path: same arithmetic as the GPU)."""
        ire0, hz_ire, vsync_ire, out_scale, ozero = self.levels()
        if isinstance(input, np.ndarray):
            scale = out_scale / hz_ire
            offset = ozero - vsync_ire * out_scale - ire0 * scale
            v = input.astype(np.float64) * scale + offset + 0.5
            return np.clip(v, 0, 65535).astype(np.uint16)
        reduced = (input - ire0) / hz_ire
        reduced -= vsync_ire
        return np.uint16(np.clip((reduced * out_scale) + ozero, 0, 65535) + 0.5)

    def computewow_scaled(self):
        """Host FP64 restatement of core.py:2591-2623 (the GPU recomputes the
        same values internally; this is for callers that want the arrays).
        The quadratic / cubic forms call scipy's make_interp_spline with the
        reference's arguments."""
        act = np.asarray(self.linelocs, dtype=np.float64)
        n = len(act)
        exp = np.array([i * self.inlinelen for i in range(n)], dtype=np.float64)
        nout = self.outlinecount * self.outlinelen + (self.lineoffset + 1) * self.outlinelen
        x = np.arange(nout) * (self.inlinelen / self.outlinelen)
        if self.wow_interpolation_method != "linear":
            from scipy import interpolate
            k, bc = {"quadratic": (2, None), "cubic": (3, "natural")}[self.wow_interpolation_method]
            spl = interpolate.make_interp_spline(exp, act, k=k, bc_type=bc, check_finite=False)
            self.interpolated_pixel_locs = spl(x)
            self.wowfactors = spl(x, 1)
            return self.interpolated_pixel_locs, self.wowfactors
        seg = np.clip(np.searchsorted(exp, x, side="right") - 1, 0, n - 2)
        x0, x1 = exp[seg], exp[seg + 1]
        y0, y1 = act[seg], act[seg + 1]
        w = 1.0 / (x1 - x0)
        self.interpolated_pixel_locs = y0 * (w * (x1 - x)) + y1 * (w * (x - x0))
        self.wowfactors = y0 * (-w) + y1 * w
        return self.interpolated_pixel_locs, self.wowfactors

    def downscale(self, lineinfo=None, linesout=None, outwidth=None, channel="demod", audio=0,
                  final=False, lastfieldwritten=None):
        """core.py:2626-2722: resample to outwidth x linesout (float32, or
        uint16 levels if final) on the GPU; EFM slice; analog audio."""
        if lineinfo is None:
            lineinfo = self.linelocs
        if outwidth is None:
            outwidth = self.outlinelen
        if linesout is None:
            linesout = self.outlinecount
        buf = np.ascontiguousarray(self.data["video"][channel], dtype=np.float32)
        ll = np.ascontiguousarray(lineinfo, dtype=np.float64)
        nout = linesout * outwidth
        dsout = np.empty(nout, dtype=np.float32)
        pic = np.empty(nout, dtype=np.uint16) if final else None
        desc = tbc_descriptor(self.rf, buf, ll, self.lineoffset, outwidth, linesout, self.outlinecount,
                              self.levels(), out_u16=pic, out_f32=dsout, coord_f32=self.coord_f32,
                              wow_smoothing=self.wow_level_adjust_smoothing,
                              wow_interpolation_method=self.wow_interpolation_method)
        tbc_fields(self.rf, [desc])

        dsaudio = None
        if audio != 0 and self.rf.decode_analog_audio:
            from .audio import downscale_audio_gpu
            dsaudio, self.audio_next_offset = downscale_audio_gpu(
                self.data["audio"], lineinfo, self.rf, self.linecount, self.audio_offset(audio, lastfieldwritten),
                audio)
        self.dsaudio = dsaudio

        if self.rf.decode_digital_audio:
            self.efmout = self.data["efm"][int(self.linelocs[1]):int(self.linelocs[self.linecount + 1])]
        else:
            self.efmout = None
        if final:
            self.dspicture = pic
            return pic, self.dsaudio, self.efmout
        return dsout, self.dsaudio, self.efmout

    def rf_tbc(self, linelocs=None):
        """core.py:2724-2752 on the GPU: the TBC'd raw RF as int16."""
        from .rftbc import rf_tbc_host_field
        if linelocs is None:
            linelocs = self.linelocs
        return rf_tbc_host_field(self.rf, self.data["input"], linelocs, self.lineoffset, self.linecount)

    def dropout_detect(self):
        """core.py:2962-2983 on the GPU: (lines, starts, ends) of the field's
        dropouts, as LDdecode writes them into dropOuts."""
        from .dropouts import detect_host_field
        return detect_host_field(self.rf, self.data, self.linelocs, self.lineoffset, self.linecount,
                                 self.isFirstField, int(self.LT["hsync"][1]))

    def audio_offset(self, audio, lastfieldwritten):
        """A/V alignment offset of the first audio sample (core.py:2644-2670)."""
        from .audio import av_offset
        return av_offset(self.rf, self.readloc, self.isFirstField, audio, lastfieldwritten)


def _process(field, logic_cls):
    """Field.process(): the GPU line path for the field's read
    (LineLocator.process_field), else the host restatement (a read that
    needs the previous field's refined line locations or the level
    re-calibration, as in the batched path)."""
    loc = getattr(field.rf, "_field_locator", None)
    if loc is None:
        from .lines import LineLocator
        loc = field.rf._field_locator = LineLocator(field.rf)
    if not loc.process_field(field):
        logic_cls.process(field)
    field.out_scale = np.double(0xD300 - 0x0100) / (100 - field.rf.DecoderParams["vsync_ire"]) \
        if field.rf.system == "PAL" else np.double(0xC800 - 0x0400) / (100 - field.rf.DecoderParams["vsync_ire"])


class FieldNTSC(FieldLogicNTSC, Field):
    def process(self):
        """core.py:3471-3495 on the GPU (see _process)."""
        _process(self, FieldLogicNTSC)

    def downscale(self, lineoffset=0, final=False, *args, **kwargs):
        """core.py:3442-3451: audio only on the final pass."""
        if final is False and "audio" in kwargs:
            kwargs["audio"] = 0
        return Field.downscale(self, final=final, *args, **kwargs)


class FieldPAL(FieldLogicPAL, Field):
    def process(self):
        """core.py:3212-3239 on the GPU (see _process)."""
        _process(self, FieldLogicPAL)

    def downscale(self, final=False, *args, **kwargs):
        """core.py:3205-3207."""
        return Field.downscale(self, final=final, *args, **kwargs)
