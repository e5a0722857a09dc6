"""ctypes binding of the ldgpu C ABI (include/ldgpu.h).

The shared library is built in-tree (ld-decode_b200/build.py) next to this
file.  There is no CPU fallback: if the library is missing or cannot be
loaded, `load()` raises, and so does every GPU entry point of the package.
"""

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libldgpu.so")

LDG_OK = 0
LDG_NTSC, LDG_PAL = 0, 1
LDG_IN_INT16, LDG_IN_FLOAT32 = 0, 1
LDG_VARIANT_STOCKHAM, LDG_VARIANT_IN_PLACE = 0, 1
(LDG_F_RFHPF, LDG_F_VIDEO_G, LDG_F_DEMOD, LDG_F_05, LDG_F_BURST, LDG_F_PILOT,
 LDG_F_EFM, LDG_F_VIDEO_G_ODD, LDG_F_AUDIO2_LEFT, LDG_F_AUDIO2_RIGHT) = range(10)
LDG_NFILTERS = 10
LDG_ERR_ARG, LDG_ERR_CUDA, LDG_ERR_STATE, LDG_ERR_UNSUPPORTED, LDG_ERR_RANGE = -1, -2, -3, -4, -5

ERRORS = {-1: "argument", -2: "cuda", -3: "state", -4: "unsupported", -5: "range"}

# Every exported symbol with its (restype, argtypes); checked by the tests.
c_p = ctypes.c_void_p


class Slice(ctypes.Structure):
    _fields_ = [("start", ctypes.c_int32), ("len", ctypes.c_int32), ("roll", ctypes.c_int32)]


class DemodArgs(ctypes.Structure):
    _fields_ = [
        ("in_", c_p), ("in_kind", ctypes.c_int32), ("in_stride", ctypes.c_int64),
        ("nblocks", ctypes.c_int64),
        ("out_demod", c_p), ("out_raw", c_p), ("out_05", c_p), ("out_burst", c_p),
        ("out_pilot", c_p), ("out_rfhpf", c_p), ("out_efm", c_p),
        ("out_audio_left", c_p), ("out_audio_right", c_p),
        ("video", Slice), ("roll_05", ctypes.c_int32), ("roll_burst", ctypes.c_int32),
        ("rfhpf", Slice), ("efm", Slice), ("audio", Slice), ("stream", c_p),
    ]


class WorkItem(ctypes.Structure):
    _fields_ = [("ctx", c_p), ("args", DemodArgs)]


class TbcField(ctypes.Structure):
    _fields_ = [
        ("buf", c_p), ("buf_len", ctypes.c_int64), ("linelocs", c_p), ("nlines", ctypes.c_int32),
        ("lineoffset", ctypes.c_int32), ("outwidth", ctypes.c_int32), ("linesout", ctypes.c_int32),
        ("outlinecount", ctypes.c_int32), ("coord_f32", ctypes.c_int32),
        ("inlinelen", ctypes.c_double), ("outlinelen", ctypes.c_double),
        ("ire0", ctypes.c_double), ("hz_ire", ctypes.c_double), ("vsync_ire", ctypes.c_double),
        ("out_scale", ctypes.c_double), ("output_zero", ctypes.c_double),
        ("out_f32", c_p), ("out_u16", c_p), ("wow_smoothing", ctypes.c_double),
        ("wow_interp", ctypes.c_int32), ("pad1", ctypes.c_int32),
    ]


LDG_WOW_LINEAR, LDG_WOW_QUADRATIC, LDG_WOW_CUBIC = 1, 2, 3
WOW_METHODS = {"linear": LDG_WOW_LINEAR, "quadratic": LDG_WOW_QUADRATIC, "cubic": LDG_WOW_CUBIC}


LDG_CHAIN_MAX_LINES = 336
(LDG_CHAIN_STOP_END, LDG_CHAIN_STOP_FULL, LDG_CHAIN_STOP_PREV, LDG_CHAIN_STOP_LEVELS,
 LDG_CHAIN_STOP_ERROR) = range(5)
c_i32, c_i64, c_f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_double


class ChainParams(ctypes.Structure):
    _fields_ = [
        ("system", c_i32), ("num_pulses", c_i32), ("field_lines", c_i32 * 2), ("outlinecount", c_i32),
        ("proclines", c_i32), ("freq", c_f64), ("freq_hz", c_f64), ("linelen", c_f64), ("inlinelen", c_f64),
        ("linefreq0", c_f64), ("hsync_pulse_us", c_f64), ("eq_pulse_us", c_f64), ("vsync_pulse_us", c_f64),
        ("first_field_h", c_f64 * 2), ("hsync_tolerance", c_f64), ("ire0", c_f64), ("hz_ire", c_f64),
        ("vsync_ire", c_f64), ("max_pulse_len", c_i64), ("blocklen", c_i64), ("blockcut", c_i64),
        ("blockcut_end", c_i64), ("readlen", c_i64), ("nblocks", c_i64),
    ]


class ChainState(ctypes.Structure):
    _fields_ = [("start", c_f64), ("prev_valid", c_i32), ("prev_isfirst", c_i32), ("prev_startloc", c_i64),
                ("fields_written", c_i32), ("prev_known", c_i32), ("prev_line0", c_f64), ("prev_line0_hi", c_f64),
                ("prev_skip", c_i32), ("prev_conf", c_i32), ("prev_est", c_f64), ("prev_est_valid", c_i32),
                ("prev_est_conf", c_i32)]


class FieldPlan(ctypes.Structure):
    _fields_ = [
        ("start", c_f64), ("readloc", c_i64), ("first_block", c_i64), ("nblocks", c_i64), ("startloc", c_i64),
        ("length", c_i64), ("valid", c_i32), ("isfirst", c_i32), ("linecount", c_i32), ("proclines", c_i32),
        ("has_prev", c_i32), ("sync_confidence", c_i32), ("hsync_len", c_i32), ("prev_range", c_i32),
        ("nextfieldoffset", c_f64),
        ("linelocs1", c_f64 * LDG_CHAIN_MAX_LINES), ("linebad", ctypes.c_uint8 * LDG_CHAIN_MAX_LINES),
    ]


class Audio2Segment(ctypes.Structure):
    _fields_ = [("left", c_p), ("right", c_p), ("len", c_i64), ("out_left", c_p), ("out_right", c_p)]


class AudioField(ctypes.Structure):
    _fields_ = [("audio_left", c_p), ("audio_right", c_p), ("audio_len", c_i64), ("linelocs", c_p),
                ("nlines", ctypes.c_int32), ("nticks", ctypes.c_int32), ("timeoffset", ctypes.c_double),
                ("soundgap", ctypes.c_double), ("out", c_p)]


class AudioParams(ctypes.Structure):
    _fields_ = [("line_period", ctypes.c_double), ("linelen", ctypes.c_double), ("scale", ctypes.c_double),
                ("lfreq", ctypes.c_double), ("rfreq", ctypes.c_double)]


class RfTbcField(ctypes.Structure):
    _fields_ = [("input", c_p), ("len", c_i64), ("linelocs", c_p), ("nlines", c_i32), ("startline", c_i32),
                ("linecount", c_i32), ("linelen", c_i32), ("delay", c_f64), ("out", c_p)]


class EfmEdge(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_int32), ("prev", ctypes.c_int16), ("cur", ctypes.c_int16)]


EFM_EDGE_DTYPE = np.dtype([("pos", "<i4"), ("prev", "<i2"), ("cur", "<i2")])


class DropoutField(ctypes.Structure):
    _fields_ = [("demod", c_p), ("demod_05", c_p), ("demod_raw", c_p), ("rfhpf", c_p), ("len", c_i64),
                ("linelocs", c_p), ("nlines", c_i32), ("lineoffset", c_i32), ("linecount", c_i32),
                ("isfirst", c_i32), ("hsync_len", c_i32), ("pad", c_i32)]


class DropoutParams(ctypes.Structure):
    _fields_ = [("system", c_i32), ("video_rot", c_i32), ("outlinelen", c_i32), ("err_cap", c_i32),
                ("out_cap", c_i32), ("pad", c_i32), ("freq_mhz", c_f64), ("freq_hz_half", c_f64),
                ("ire0", c_f64), ("hz_ire", c_f64), ("vsync_ire", c_f64)]


class LinesConsts(ctypes.Structure):
    _fields_ = [("system", c_i32), ("pad", c_i32), ("freq", c_f64), ("linelen", c_f64), ("linefreq0", c_f64),
                ("samplesperline", c_f64), ("half_sync", c_f64), ("lo_ok", c_f64), ("hi_ok", c_f64),
                ("hz_ire", c_f64), ("fsc_mhz", c_f64), ("pilot_mhz", c_f64)]


class LinesArgs(ctypes.Structure):
    _fields_ = [
        ("k", LinesConsts), ("d05", c_p), ("demod", c_p), ("burst", c_p), ("pilot", c_p), ("capture_len", c_i64),
        ("nfields", c_i32), ("proclines", c_i32), ("startloc", c_p), ("wlen", c_p), ("isfirst", c_p),
        ("linecount", c_p), ("has_prev", c_p), ("linelocs1", c_p), ("linebad1", c_p),
        ("prev_phase_adjust", c_f64), ("linelocs", c_p), ("linebad", c_p), ("phase_adjust", c_p),
        ("field_phase", c_p), ("scratch", c_p), ("stream", c_p), ("prev_phase_adjust_dev", c_p),
        ("first_field", c_i32), ("count", c_i32), ("stages", c_i32), ("pad2", c_i32),
        ("prev_pal_adjust", c_f64 * 4), ("prev_pal_adjust_dev", c_p), ("prev_field_phase_dev", c_p),
        ("prev_field_phase", c_i32), ("pad3", c_i32), ("linelocs2", c_p),
    ]


SIGNATURES = {
    "ldg_abi_version": (ctypes.c_int, []),
    "ldg_last_error": (ctypes.c_char_p, []),
    "ldg_device_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    "ldg_ctx_create": (ctypes.c_int, [ctypes.POINTER(c_p), ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_int32, ctypes.c_double]),
    "ldg_ctx_destroy": (None, [c_p]),
    "ldg_set_filter": (ctypes.c_int, [c_p, ctypes.c_int32, c_p, ctypes.c_int64]),
    "ldg_set_audio": (ctypes.c_int, [c_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_p,
                                     ctypes.c_double, ctypes.c_double]),
    "ldg_set_sinc_lut": (ctypes.c_int, [c_p, c_p, ctypes.c_int32, ctypes.c_int32]),
    "ldg_demod_blocks": (ctypes.c_int, [c_p, ctypes.POINTER(DemodArgs)]),
    "ldg_set_notch": (ctypes.c_int, [c_p, ctypes.c_int32, ctypes.c_int32]),
    "ldg_copy_async": (ctypes.c_int, [c_p, c_p, ctypes.c_int64, c_p]),
    "ldg_unpack_lds": (ctypes.c_int, [c_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, c_p, c_p]),
    "ldg_audio_phase2": (ctypes.c_int, [c_p, ctypes.POINTER(Audio2Segment), ctypes.c_int32, ctypes.c_double,
                                        ctypes.c_double, c_p]),
    "ldg_rf_tbc": (ctypes.c_int, [c_p, ctypes.POINTER(RfTbcField), ctypes.c_int32, c_p]),
    "ldg_audio_downscale": (ctypes.c_int, [c_p, ctypes.POINTER(AudioField), ctypes.c_int32,
                                           ctypes.POINTER(AudioParams), c_p, c_p]),
    "ldg_dropouts": (ctypes.c_int, [c_p, ctypes.POINTER(DropoutParams), ctypes.POINTER(DropoutField),
                                    ctypes.c_int32, c_p, c_p, c_p, c_p]),
    "ldg_queue_create": (ctypes.c_int, [ctypes.POINTER(c_p), ctypes.c_int32]),
    "ldg_queue_destroy": (None, [c_p]),
    "ldg_queue_submit": (ctypes.c_int, [c_p, ctypes.POINTER(WorkItem), ctypes.c_int32]),
    "ldg_queue_set_schedule": (ctypes.c_int, [c_p, ctypes.c_int32, ctypes.c_int32]),
    "ldg_queue_info": (ctypes.c_int, [c_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)]),
    "ldg_queue_run": (ctypes.c_int, [c_p, c_p, ctypes.c_int32]),
    "ldg_tbc_fields": (ctypes.c_int, [c_p, ctypes.POINTER(TbcField), ctypes.c_int32, c_p]),
    "ldg_synchronize": (ctypes.c_int, [c_p]),
    "ldg_demod_scratch_bytes": (ctypes.c_int, [c_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "ldg_demod_blocks_noalloc": (ctypes.c_int, [c_p, ctypes.POINTER(DemodArgs), ctypes.c_int32]),
    "ldg_sync_runs": (ctypes.c_int, [c_p, c_p, c_i64, c_f64, c_i64, c_i64, c_i64, c_p, c_p, c_p, c_i64,
                                     ctypes.POINTER(c_i64), c_p]),
    "ldg_field_chain": (ctypes.c_int, [ctypes.POINTER(ChainParams), c_p, c_p, c_p, c_i64,
                                       ctypes.POINTER(ChainState), ctypes.POINTER(ChainState), c_p, c_i32,
                                       ctypes.POINTER(c_i32), ctypes.POINTER(c_i32)]),
    "ldg_chain_last_error": (ctypes.c_char_p, []),
    "ldg_field_chain_mt": (ctypes.c_int, [ctypes.POINTER(ChainParams), c_p, c_p, c_p, c_i64,
                                          ctypes.POINTER(ChainState), ctypes.POINTER(ChainState), c_p, c_i32,
                                          ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), c_i32, c_i64, c_i64]),
    "ldg_lines_scratch_bytes": (c_i64, [c_i32]),
    "ldg_abi_sizeof": (c_i64, [ctypes.c_char_p]),
    "ldg_demod_status": (ctypes.c_int, [c_p, ctypes.POINTER(c_i32)]),
    "ldg_tbc_fields_async": (ctypes.c_int, [c_p, c_p, c_i32, c_p]),
    "ldg_tbc_status": (ctypes.c_int, [c_p, ctypes.POINTER(c_i32)]),
    "ldg_lines_refine": (ctypes.c_int, [c_p, ctypes.POINTER(LinesArgs)]),
    "ldg_ac3_last_error": (ctypes.c_char_p, []),
    "ldg_ac3_create": (ctypes.c_int, [ctypes.POINTER(c_p), ctypes.c_int32, c_p, ctypes.c_int32, c_p,
                                      ctypes.c_int32, c_p, ctypes.c_int32, ctypes.c_int32, c_p, c_p,
                                      ctypes.c_int32]),
    "ldg_ac3_destroy": (None, [c_p]),
    "ldg_ac3_frontend": (ctypes.c_int, [c_p, c_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                        ctypes.c_int64, ctypes.c_int64, c_p, c_p, c_p]),
    "ldg_ac3_dpll_create": (ctypes.c_int, [ctypes.POINTER(c_p), ctypes.c_double]),
    "ldg_ac3_dpll_destroy": (None, [c_p]),
    "ldg_ac3_dpll_reclock": (ctypes.c_int, [c_p, c_p, c_p, ctypes.c_int64, c_p, ctypes.POINTER(ctypes.c_int64)]),
    "ldg_set_demod_variant": (ctypes.c_int, [c_p, c_i32]),
    "ldg_get_demod_variant": (ctypes.c_int, [c_p, ctypes.POINTER(c_i32)]),
    "ldg_set_demod_schedule": (ctypes.c_int, [c_p, c_i32]),
    "ldg_blocks_from_spectra": (ctypes.c_int, [c_p, c_p, c_i64, c_p, c_p]),
    "ldg_queue_set_variant": (ctypes.c_int, [c_p, c_i32]),
    "ldg_efm_pll_create": (ctypes.c_int, [ctypes.POINTER(c_p)]),
    "ldg_efm_pll_destroy": (ctypes.c_int, [c_p]),
    "ldg_efm_pll_process": (ctypes.c_int, [c_p, c_p, c_i64, c_p, c_i64, ctypes.POINTER(c_i64)]),
    "ldg_efm_pll_state": (ctypes.c_int, [c_p, c_p, c_p]),
    "ldg_efm_pll_process_edges": (ctypes.c_int, [c_p, c_p, c_i64, c_i64, c_i64, ctypes.c_int16, ctypes.c_int16, c_p,
                                                 c_i64, ctypes.POINTER(c_i64)]),
    "ldg_efm_edges_scratch_bytes": (c_i64, [c_i64]),
    "ldg_efm_field_slices": (ctypes.c_int, [c_p, c_p, c_p, c_i32, c_p, c_i64, c_p, c_p, c_p]),
    "ldg_efm_edges": (ctypes.c_int, [c_p, c_i64, c_i32, c_i64, c_p, c_i64, c_p, c_p, c_p]),
}

# ABI of the library this binding is written for (LDG_ABI_VERSION in
# include/ldgpu.h) and the structures whose layout it mirrors
ABI_VERSION = 3
ABI_STRUCTS = [("ldg_chain_params", ChainParams), ("ldg_chain_state", ChainState),
               ("ldg_field_plan", FieldPlan), ("ldg_lines_consts", LinesConsts),
               ("ldg_lines_args", LinesArgs), ("ldg_tbc_field", TbcField),
               ("ldg_demod_args", DemodArgs), ("ldg_slice", Slice), ("ldg_work_item", WorkItem),
               ("ldg_dropout_field", DropoutField), ("ldg_dropout_params", DropoutParams),
               ("ldg_rftbc_field", RfTbcField), ("ldg_audio2_segment", Audio2Segment),
               ("ldg_audio_field", AudioField), ("ldg_audio_params", AudioParams), ("ldg_efm_edge", EfmEdge)]

_lib = None
_lock = threading.Lock()


class LdgError(RuntimeError):
    """A failed ldgpu C-ABI call (code and message from ldg_last_error)."""

    def __init__(self, code, msg):
        super().__init__(f"ldgpu error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


def load(path=None):
    """Load (once) and return the ctypes handle of libldgpu.so."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or LIBPATH
        if not os.path.exists(p):
            raise ImportError(f"ldgpu CUDA library not built: {p} is missing "
                              "(run python ld-decode_b200/build.py)")
        lib = ctypes.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        # a library built from other sources than this binding would misread
        # every descriptor: refuse it
        if lib.ldg_abi_version() != ABI_VERSION:
            raise ImportError(f"{p}: ABI version {lib.ldg_abi_version()}, this binding needs {ABI_VERSION} "
                              "(rebuild with python ld-decode_b200/build.py)")
        for sname, t in ABI_STRUCTS:
            if lib.ldg_abi_sizeof(sname.encode()) != ctypes.sizeof(t):
                raise ImportError(f"{p}: {sname} is {lib.ldg_abi_sizeof(sname.encode())} bytes, "
                                  f"the binding's {ctypes.sizeof(t)} (rebuild the library)")
        _lib = lib
        return lib


def check(rc):
    if rc != LDG_OK:
        msg = load().ldg_last_error()
        raise LdgError(rc, msg.decode() if msg else "")
    return rc


def device_count():
    n = ctypes.c_int32(0)
    check(load().ldg_device_count(ctypes.byref(n)))
    return n.value


class Context:
    """Owns one ldg_ctx (device filters, twiddles, scratch, staging)."""

    def __init__(self, system, blocklen, fs_hz, device=0):
        lib = load()
        self._lib = lib
        h = c_p()
        check(lib.ldg_ctx_create(ctypes.byref(h), int(device), LDG_PAL if system == "PAL" else LDG_NTSC,
                                 int(blocklen), float(fs_hz)))
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self._lib.ldg_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
