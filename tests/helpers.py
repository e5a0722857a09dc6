"""Shared helpers for the parity tests (oracle runs, error metrics)."""

import numpy as np

from oracle import demod as odemod

VIDEO_KEYS = ("demod", "demod_raw", "demod_05", "demod_burst")


def video_keys(system):
    return VIDEO_KEYS + (("demod_pilot",) if system == "PAL" else ())


def oracle_block(rf, block, mtf_scaled, cut=True, rot=None):
    """The CPU oracle on one block with rf's filters and geometry."""
    rot = rf.delays["video_rot"] if rot is None else rot
    return odemod.demodblock(block, rf.Filters, system=rf.system, freq_hz=rf.freq_hz,
                             blocklen=rf.blocklen, blockcut=rf.blockcut,
                             blockcut_end=rf.blockcut_end, video_rot=rot, mtf_level=mtf_scaled,
                             cut=cut, efm=bool(rf.decode_digital_audio),
                             audio=rf.audio if rf.decode_analog_audio else None)


def oracle_capture(rf, cap, first_block, nblocks, mtf_scaled, keys=("demod",)):
    """Concatenated cut oracle outputs of blocks [first, first+n)."""
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    outs = {k: [] for k in keys}
    for b in range(first_block, first_block + nblocks):
        rv = odemod.demodblock(cap[b * U:b * U + rf.blocklen], rf.Filters, system=rf.system,
                               freq_hz=rf.freq_hz, blocklen=rf.blocklen, blockcut=rf.blockcut,
                               blockcut_end=rf.blockcut_end, video_rot=rf.delays["video_rot"],
                               mtf_level=mtf_scaled, cut=True)
        for k in keys:
            outs[k].append(rv["video"][k])
    return {k: np.concatenate(v) for k, v in outs.items()}


def err_stats(gpu, ref):
    d = gpu.astype(np.float64) - ref.astype(np.float64)
    return float(np.sqrt(np.mean(d * d))), float(np.abs(d).max())
