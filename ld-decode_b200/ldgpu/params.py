"""System and decoder parameter tables for NTSC and PAL LaserDisc RF.

These numbers define the television systems and the decoder's filter
settings; they must equal the reference decoder's tables value for value,
because every filter, line length and output level is derived from them
(lddecode/core.py:66-251).  They are rebuilt here by two small factory
functions instead of module-level dict literals, and the derived entries
(line period, outlinelen, ...) are computed the same way the reference
derives them (core.py:111-127, 166-170).
"""

import copy

import numpy as np

# FFT block length of the overlap-save demodulator (core.py:66).
BLOCKSIZE = 32 * 1024
# Samples dropped at the start of every demodulated block (core.py:321).
BLOCKCUT = 1024


def _round_int(x):
    """int(np.round(x)): round-half-even, as the reference's nb_round
    (lddecode/utils.py:1238-1239)."""
    return int(np.round(x))


def calclinelen(sysparams, mult, mhz):
    """Exact line length in samples for a clock of `mhz` * `mult`
    (core.py:111-115)."""
    if isinstance(mhz, str):
        mhz = sysparams[mhz]
    return _round_int(sysparams["line_period"] * mhz * mult)


def _ntsc():
    fsc = 315.0 / np.double(88.0)
    linerate = 1e6 * 315 / 88 / 227.5
    sp = {
        "fsc_mhz": fsc,
        "pilot_mhz": fsc,  # NTSC discs carry no pilot; the burst stands in
        "frame_lines": 525,
        "field_lines": (263, 262),
        "ire0": 8100000,
        "hz_ire": 1700000 / 140.0,
        "vsync_ire": -40,
        "analog_audio": True,
        "audio_lfreq": linerate * 146.25,
        "audio_rfreq": linerate * 178.75,
        "audio_rfreq_AC3": 2880000,
        "colorBurstUS": (5.3, 7.8),
        "blacksnr_slice": (1, 10, 20),
        "firstFieldH": (0.5, 1),
        "numPulses": 6,
        "hsyncPulseUS": 4.7,
        "eqPulseUS": 2.3,
        "vsyncPulseUS": 27.1,
        "outputZero": 1024,
        "fieldPhases": 4,
        "LD_VITS_whitelocs": [(20, 14, 12), (20, 52, 8), (13, 13, 15), (11, 12, 45)],
        "LD_VITS_code_slices": [(16, 12, 48, 85), (17, 12, 48, 85), (10, 13, 39, 85)],
    }
    sp["line_period"] = 1 / (sp["fsc_mhz"] / np.double(227.5))
    sp["activeVideoUS"] = (9.45, sp["line_period"] - 1.0)
    sp["FPS"] = 1000000 / (525 * sp["line_period"])
    sp["outlinelen"] = calclinelen(sp, 4, "fsc_mhz")
    sp["outfreq"] = 4 * sp["fsc_mhz"]
    return sp


def _pal():
    sp = {
        "FPS": 25,
        "fsc_mhz": ((1 / 64) * 283.75) + (25 / 1000000),
        "pilot_mhz": 3.75,
        "frame_lines": 625,
        "field_lines": (312, 313),
        "line_period": 64,
        "ire0": 7100000,
        "hz_ire": 800000 / 100.0,
        "analog_audio": True,
        "audio_lfreq": (1000000 / 64) * 43.75,
        "audio_rfreq": (1000000 / 64) * 68.25,
        "colorBurstUS": (5.6, 7.85),
        "activeVideoUS": (10.5, 64 - 1.5),
        "firstFieldH": (1, 0.5),
        "blacksnr_slice": (22, 12, 50),
        "numPulses": 5,
        "hsyncPulseUS": 4.7,
        "eqPulseUS": 2.35,
        "vsyncPulseUS": 27.3,
        "outputZero": 256,
        "fieldPhases": 8,
        "LD_VITS_whitelocs": [(19, 12, 8)],
        "LD_VITS_code_slices": [(16, 11, 49, 85), (17, 11, 49, 85)],
    }
    sp["outlinelen"] = calclinelen(sp, 4, "fsc_mhz")
    sp["outlinelen_pilot"] = calclinelen(sp, 4, "pilot_mhz")
    sp["outfreq"] = 4 * sp["fsc_mhz"]
    sp["vsync_ire"] = -0.3 * (100 / 0.7)
    return sp


def _filters(system, lowband):
    """Decoder (filter) parameters (core.py:172-251)."""
    if system == "NTSC":
        fp = {
            "audio_notchwidth": 200000,
            "audio_notchorder": 2,
            "video_deemp": (120e-9, 320e-9),
            "video_bpf_low": 3700000,
            "video_bpf_low_order": 2,
            "video_bpf_high": 13800000,
            "video_bpf_high_order": 3,
            "video_bpf_order": 4,
            "video_lpf_freq": 4500000,
            "video_lpf_order": 6,
            "MTF_basemult": 0.4,
            "MTF_poledist": 0.9,
            "MTF_freq": 12.2,
            "video_hpf_freq": 10000000,
            "video_hpf_order": 4,
            "audio_filterwidth": 150000,
            "audio_filterorder": 512,
        }
        if lowband:
            fp.update(video_bpf_low=3800000, video_bpf_high=12500000,
                      video_lpf_freq=4200000)
    elif system == "PAL":
        fp = {
            "audio_notchwidth": 200000,
            "audio_notchorder": 2,
            "video_deemp": (100e-9, 400e-9),
            "video_bpf_low": 2300000,
            "video_bpf_low_order": 2,
            "video_bpf_high": 14000000,
            "video_bpf_high_order": 3,
            "video_bpf_order": 2,
            "video_lpf_freq": 5800000,
            "video_lpf_order": 7,
            "MTF_basemult": 1.0,
            "MTF_poledist": 0.70,
            "MTF_freq": 10,
            "video_hpf_freq": 10000000,
            "video_hpf_order": 4,
            "audio_filterwidth": 100000,
            "audio_filterorder": 900,
        }
        if lowband:
            fp.update(video_bpf_low=3200000, video_bpf_high=13000000,
                      video_bpf_order=2, video_lpf_freq=4800000)
    else:
        raise ValueError(f"unknown system {system!r}")
    return fp


_SYS = {"NTSC": _ntsc(), "PAL": _pal()}

SysParams_NTSC = _SYS["NTSC"]
SysParams_PAL = _SYS["PAL"]


def sysparams(system):
    """A private deep copy of the system table for `system`."""
    if system not in _SYS:
        raise ValueError(f"unknown system {system!r}")
    return copy.deepcopy(_SYS[system])


def filterparams(system, lowband=False):
    """A private copy of the decoder/filter table for `system`."""
    return copy.deepcopy(_filters(system, lowband))
