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


class OracleBlocks:
    """Cut oracle outputs of a capture's blocks, computed on demand by a
    thread pool (numpy's transforms release the GIL) and cached, joined into
    field read windows the way DemodCache.read joins them."""

    def __init__(self, rf, cap, mtf_scaled, keys, threads=8):
        self.rf, self.cap, self.mtf, self.keys = rf, cap, mtf_scaled, keys
        self.U = rf.blocklen - rf.blockcut - rf.blockcut_end
        self.threads = threads
        self.cache = {}

    def _one(self, b):
        rf = self.rf
        rv = odemod.demodblock(self.cap[b * self.U:b * self.U + rf.blocklen], rf.Filters, system=rf.system,
                               freq_hz=rf.freq_hz, blocklen=rf.blocklen, blockcut=rf.blockcut,
                               blockcut_end=rf.blockcut_end, video_rot=rf.delays["video_rot"],
                               mtf_level=self.mtf, cut=True)
        return {k: rv["video"][k] for k in self.keys}

    def window(self, first_block, nblocks):
        from concurrent.futures import ThreadPoolExecutor
        need = [b for b in range(first_block, first_block + nblocks) if b not in self.cache]
        if need:
            with ThreadPoolExecutor(self.threads) as ex:
                for b, rv in zip(need, ex.map(self._one, need)):
                    self.cache[b] = rv
        bl = range(first_block, first_block + nblocks)
        return {k: np.concatenate([self.cache[b][k] for b in bl]) for k in self.keys}


def efm_crossings(x, before=None):
    """Zero crossings of int16 array x as EFM_PLL.process tests them
    (efm_pll.py:148-151): i with sign(x[i-1]) != sign(x[i]), x[-1] = before
    (no crossing at 0 without it); an EFM_EDGE_DTYPE array."""
    from ldgpu import lib as L
    x = np.asarray(x, np.int16)
    prev = np.concatenate([[before if before is not None else 0], x[:-1]]).astype(np.int16)
    i = np.nonzero((prev.astype(np.int32) ^ x.astype(np.int32)) < 0)[0]
    e = np.empty(len(i), L.EFM_EDGE_DTYPE)
    e["pos"], e["prev"], e["cur"] = i, prev[i], x[i]
    return e
