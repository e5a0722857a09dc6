"""Host restatement of the reference's field sync / line-location logic.

Field.process() and its helpers (lddecode/core.py:1636-2589, 2998-3047,
3053-3239, 3349-3495): sync-pulse detection on demod_05, the vertical
blanking state machine, line 0, per-line H-sync zero crossings, colour
burst (NTSC) / pilot (PAL) phase refinement and bad-line repair.  It runs on
the host in FP64 over the GPU-demodulated field arrays; integer results
(pulse indices, line count, field order) follow the reference's rules.
"""

import numpy as np


class FieldLogic:
    """Constructor and shared state of a field (core.py:1587-1634)."""

    def __init__(self, rf, decode, prevfield=None, initphase=False, fields_written=0, readloc=0,
                 use_threads=True, wow_level_adjust_smoothing=0, wow_interpolation_method="linear"):
        self.rawdata = decode.get("input")
        self.data = decode
        self.initphase = initphase
        self.readloc = readloc
        self.prevfield = prevfield
        self.fields_written = fields_written
        self.rf = rf
        self.freq = rf.freq
        self.inlinelen = rf.linelen
        self.outlinelen = rf.SysParams["outlinelen"]
        self.lineoffset = 0
        self.needrerun = False
        self.valid = False
        self.sync_confidence = 100
        self.dspicture = None
        self.dsaudio = None
        self.interpolated_pixel_locs = None
        self.wowfactors = None
        self.outlinecount = (rf.SysParams["frame_lines"] // 2) + 1
        self.linecount = None
        self.use_threads = use_threads
        self.wow_level_adjust_smoothing = wow_level_adjust_smoothing
        self.wow_interpolation_method = wow_interpolation_method


class FieldLogicNTSC(FieldLogic):
    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.phase_adjust_median = 0
        self.out_scale = np.double(0xC800 - 0x0400) / (100 - self.rf.DecoderParams["vsync_ire"])


class FieldLogicPAL(FieldLogic):
    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.out_scale = np.double(0xD300 - 0x0100) / (100 - self.rf.DecoderParams["vsync_ire"])
