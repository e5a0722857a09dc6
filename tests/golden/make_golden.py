#!/usr/bin/env python3
"""Regenerate the golden fixtures in this folder from the unmodified reference.

Runs happycube/ld-decode's own Python code (imported from /root/reference,
read-only, in the development container only) on seeded synthetic inputs made
by ldgpu.synth, and saves small .npz fixtures:

  filters_<cfg>.npz  -- RFDecode filter bank summaries (sampled bins, sums),
                        audio slice geometry, computedelays results;
  demod_<cfg>.npz    -- one input block and the reference demodblock outputs
                        (subsampled video/rfhpf/efm, full audio) at two MTF levels;
  tbc_smoothing_<sys>.npz -- the first golden field through the reference's
                        TBC with wow_level_adjust_smoothing = 2 (utils.py:
                        141-149): line locations and the uint16 picture;
  wow_interp_<sys>.npz -- the first golden field through the reference's
                        TBC with wow_interpolation_method quadratic / cubic
                        (core.py:2591-2623), on its own line locations and on
                        line locations with added sinusoidal wow and two
                        displaced lines (with and without level smoothing):
                        coordinates, wow factors, their median / MAD and
                        every PIC_STRIDE-th sample of the uint16 picture;
  audio2_<sys>.npz   -- analog audio stage 2 (RFDecode.audio_phase2,
                        core.py:884-950) on seeded field-length stage-1
                        audio with spikes (blanked by its peak finder), one
                        field-length and one longer (several transforms);
  demod_pal_notch.npz -- a PAL block with spurious 8.5 MHz tones through the
                        reference demodblock with PAL_V4300D_NotchFilter on
                        (core.py:774-798): outputs and the zeroed bins;
  field_<sys>.npz    -- a capture, and for two consecutive fields the
                        reference's sync pulses, line locations, field flags,
                        TBC coordinates summary and the final uint16 picture;
  sinc_lut_rows.npz  -- sampled rows of the reference's shipped sinc table;
  audio_downscale.npz -- analog audio downscale (core.py:1423-1580) for a set of
                        seeded line-location / audio cases: locs, wow factors,
                        int16 output, next-field offset, mute flag;
  ac3_loopback.npz   -- AC3-RF demodulator (lddecode/ac3rf.py) on a seeded
                        DQPSK signal: baseband I/Q windows and the symbols of
                        a clean (streamed in uneven blocks) and a noisy run;
  lds_unpack.npz     -- the reference's .lds unpacker (unpack_data_4_40,
                        utils.py:371-391) on seeded random packed bytes at
                        several offsets and lengths;
  rftbc_<sys>.npz    -- RF TBC (Field.rf_tbc, core.py:2724-2752, cubic scale
                        utils.py:37-70) of two fields: SHA-256 of each int16
                        output, a subsample and two whole lines;
  dropouts_<sys>.npz -- dropout detection (Field.dropout_detect,
                        core.py:2829-2996) on a capture with seeded dropouts:
                        per field the line locations, flags, hsync length,
                        rfhpf standard deviation, error sample indices, the
                        merged error list and the final dropout lines/ranges.

  fields_<case>.npz  -- line location over 10-12 consecutive fields of a
                        capture per case of tests/golden/field_cases.py (clean,
                        30 dB SNR, seeded dropouts, 0.8-sample wow, dropouts
                        on vertical sync, PAL through its 8-field sequence):
                        per field the reference's sync pulses, valid-pulse
                        classes, line locations, bad lines, flags (field order,
                        line count, line offset, phase ID, sync confidence),
                        next-field offset and a picture digest;
  efm_pll.npz        -- the reference's EFM_PLL (efm_pll.py:80-244) over seeded
                        EFM-like signals (tests/golden/efm_cases.py) fed in
                        buffers of uneven length: every call's T-values and
                        the loop state at the end;
  audio_slices.npz   -- the reference's _downscale_audio_to_output (core.py:
                        1493-1533) on hand-made run boundaries that start
                        before the audio buffer (both bounds negative, and a
                        start below -len that numpy clamps to 0).

Nothing at test time reads the reference; only this script does.
Usage: python tests/golden/make_golden.py --ref <ld-decode checkout> [fixture]
(or set LDDECODE_REF to the checkout instead of --ref).
"""

import hashlib
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _take_ref(argv):
    """The reference checkout: --ref PATH (removed from argv) or $LDDECODE_REF."""
    if "--ref" in argv:
        i = argv.index("--ref")
        path = argv[i + 1]
        del argv[i:i + 2]
        return path
    return os.environ.get("LDDECODE_REF")


REF = _take_ref(sys.argv)
if not REF or not os.path.isdir(os.path.join(REF, "lddecode")):
    sys.exit("usage: make_golden.py --ref <ld-decode checkout> [fixture]  (or LDDECODE_REF=<checkout>)")

os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
sys.dont_write_bytecode = True
sys.path.insert(0, os.path.join(REPO, "ld-decode_b200"))
sys.path.insert(0, REF)

import numpy as np  # noqa: E402

from lddecode import core as refcore  # noqa: E402
from ldgpu.synth import inject_dropouts, synth_capture  # noqa: E402

sys.path.insert(0, HERE)
from audio_cases import AUDIO_CASES, audio_case_inputs  # noqa: E402

STRIDE = 9
COORD_STRIDE = 101
CAPTURE_START = 123457
FILTER_STEP = 61

CONFIGS = {
    "ntsc": dict(system="NTSC", decode_analog_audio=44100, decode_digital_audio=True),
    "pal": dict(system="PAL", decode_analog_audio=44100, decode_digital_audio=True),
    "ntsc_lowband": dict(system="NTSC", decode_analog_audio=44100, decode_digital_audio=True,
                         extra_options={"lowband": True, "deemp_str": 1.5,
                                        "NTSC_ColorNotchFilter": True, "MTF_level": 0.7,
                                        "MTF_offset": 0.1}),
    "pal_lowband": dict(system="PAL", decode_analog_audio=44100, decode_digital_audio=True,
                        extra_options={"lowband": True, "deemp_coeff": (2.0, 7.0)}),
}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def filters_fixture(name, kw):
    rf = refcore.RFDecode(**kw)
    out = {}
    idx = np.arange(0, rf.blocklen, FILTER_STEP)
    for k, v in rf.Filters.items():
        if isinstance(v, np.ndarray):
            out["F_" + k] = v[idx]
            out["Fsum_" + k] = np.array([np.sum(v), np.sum(np.abs(v) ** 2)])
        else:
            out["S_" + k] = np.array(v)
    for ch in ("left", "right"):
        a = rf.audio[ch]
        out[f"A_{ch}_geom"] = np.array([a.lowbin, a.nbins, a.a1_freq, a.low_freq], dtype=np.float64)
        out[f"A_{ch}_filt1"] = a.filt1
        out[f"A_{ch}_audio2"] = a.audio2_filter[idx]
    out["delays"] = np.array([rf.delays["video_sync"], rf.delays["video_white"],
                              rf.delays["video_rot"]], dtype=np.float64)
    out["limits"] = np.array([*rf.limits["sync"], *rf.limits["viewable"]], dtype=np.float64)
    out["blockcut_end"] = np.array(rf.blockcut_end)
    out["bin_idx"] = idx
    np.savez_compressed(os.path.join(HERE, f"filters_{name}.npz"), **out)
    return rf


def demod_fixture(name, rf, kw, seed):
    cap = synth_capture(kw["system"], rf.blocklen + 4096, seed=seed).numpy()
    block = cap[1000:1000 + rf.blocklen].copy()
    out = {"block": block}
    for tag, mtf in (("m0", 0), ("m1", 1)):
        rv = rf.demodblock(data=block, mtf_level=mtf, cut=True)
        for k in rv["video"].dtype.names:
            v = np.asarray(rv["video"][k])
            out[f"{tag}_{k}"] = v[::STRIDE]
            out[f"{tag}_{k}_sum"] = np.array([np.sum(v.astype(np.float64)),
                                              np.sum(v.astype(np.float64) ** 2)])
        out[f"{tag}_rfhpf"] = rv["rfhpf"][::STRIDE]
        out[f"{tag}_efm"] = rv["efm"][::STRIDE]
        out[f"{tag}_efm_sum"] = np.array([np.sum(rv["efm"].astype(np.int64))])
        out[f"{tag}_audio_left"] = np.asarray(rv["audio"]["audio_left"])
        out[f"{tag}_audio_right"] = np.asarray(rv["audio"]["audio_right"])
    # uncut form, video only
    rv = rf.demodblock(data=block, mtf_level=1, cut=False)
    for k in rv["video"].dtype.names:
        out[f"full_{k}"] = np.asarray(rv["video"][k])[::STRIDE]
    out["full_audio_left"] = np.asarray(rv["audio"]["audio_left"])
    out["full_efm"] = rv["efm"][::STRIDE]
    out["mtf_scaled"] = np.array([((1 * rf.mtf_mult) + rf.mtf_offset) * rf.DecoderParams["MTF_basemult"]])
    np.savez_compressed(os.path.join(HERE, f"demod_{name}.npz"), **out)


class BlockSource:
    """Per-block demod outputs over a capture, assembled into field reads the
    way DemodCache.read + LDdecode.decodefield do (core.py:1343-1413,
    4030-4042)."""

    def __init__(self, rf, cap, mtf):
        self.rf, self.cap, self.mtf = rf, cap, mtf
        self.U = rf.blocklen - rf.blockcut - rf.blockcut_end
        self.cache = {}

    def block(self, b):
        if b not in self.cache:
            raw = self.cap[b * self.U:b * self.U + self.rf.blocklen]
            if len(raw) < self.rf.blocklen:
                return None
            rv = self.rf.demodblock(data=raw, mtf_level=self.mtf, cut=True)
            rv["input"] = raw[self.rf.blockcut:-self.rf.blockcut_end]
            self.cache[b] = rv
        return self.cache[b]

    def read_field(self, start):
        readloc = max(int(start - self.rf.blockcut), 0)
        bs = self.rf.blocklen
        begin = (readloc // bs) * bs
        length = ((self.readlen // bs) + 2) * bs
        end = begin + length
        blocks = range(begin // self.U, end // self.U + 1)
        parts = [self.block(b) for b in blocks]
        if any(p is None for p in parts):
            return None
        rv = {
            "input": np.concatenate([p["input"] for p in parts]),
            "video": np.concatenate([p["video"] for p in parts]).view(np.recarray),
            "rfhpf": np.concatenate([p["rfhpf"] for p in parts]),
            "startloc": (begin // self.U) * self.U,
        }
        return rv, readloc


def field_fixture(system, seed, nfields=2):
    kw = dict(system=system, decode_analog_audio=0, decode_digital_audio=False)
    rf = refcore.RFDecode(**kw)
    src = BlockSource(rf, None, 1)
    fieldcls = refcore.FieldPAL if system == "PAL" else refcore.FieldNTSC
    if system == "PAL":
        src.readlen = rf.linelen * 400
    else:
        src.readlen = ((rf.linelen * 350) // 16384) * 16384
    fieldlen = int(rf.freq_hz / (rf.SysParams["FPS"] * 2))
    ncap = nfields * fieldlen + src.readlen + 8 * rf.blocklen
    cap = synth_capture(system, ncap, seed=seed, start=CAPTURE_START).numpy()
    src.cap = cap
    out = {"capture_sha256": np.array(sha(cap)), "capture_len": np.array(ncap),
           "capture_seed": np.array(seed), "capture_start": np.array(CAPTURE_START),
           "mtf_level": np.array(1.0)}
    prev = None
    start = 0
    i = 0
    skipped = []
    while i < nfields:
        rd = src.read_field(start)
        assert rd is not None
        decode, readloc = rd
        f = fieldcls(rf, decode, prevfield=prev, initphase=(i == 0), fields_written=i,
                     readloc=decode["startloc"])
        f.process()
        if not f.valid:
            # readfield moves on by nextfieldoffset after an invalid field
            skipped.append(start)
            start = start + f.nextfieldoffset
            prev = None
            assert len(skipped) < 4
            continue
        dsout, _, _ = f.downscale(linesout=f.outlinecount, final=True)
        p = f"f{i}_"
        out[p + "start"] = np.array(start)
        out[p + "readloc"] = np.array(readloc)
        out[p + "startloc"] = np.array(decode["startloc"])
        out[p + "pulse_start"] = np.array([q.start for q in f.rawpulses], dtype=np.int64)
        out[p + "pulse_len"] = np.array([q.len for q in f.rawpulses], dtype=np.int64)
        out[p + "valid_type"] = np.array([v[0] for v in f.validpulses], dtype=np.int64)
        out[p + "valid_start"] = np.array([v[1].start for v in f.validpulses], dtype=np.int64)
        out[p + "valid_good"] = np.array([bool(v[2]) for v in f.validpulses])
        out[p + "linelocs1"] = np.array(f.linelocs1, dtype=np.float64)
        out[p + "linelocs2"] = np.array(f.linelocs2, dtype=np.float64)
        out[p + "linelocs"] = np.array(f.linelocs, dtype=np.float64)
        out[p + "linebad"] = np.array(f.linebad, dtype=bool)
        out[p + "flags"] = np.array([int(f.isFirstField), f.linecount, f.lineoffset,
                                     f.fieldPhaseID, f.sync_confidence], dtype=np.int64)
        out[p + "nextfieldoffset"] = np.array(f.nextfieldoffset, dtype=np.float64)
        out[p + "burstmedian"] = np.array(f.burstmedian, dtype=np.float64)
        out[p + "coords"] = f.interpolated_pixel_locs[::COORD_STRIDE]
        out[p + "wow"] = f.wowfactors[::COORD_STRIDE]
        out[p + "wow_stats"] = np.array([len(f.wowfactors), np.median(f.wowfactors)])
        out[p + "dspicture"] = np.asarray(f.dspicture)
        out[p + "levels"] = np.array([rf.DecoderParams["ire0"], rf.DecoderParams["hz_ire"],
                                      rf.DecoderParams["vsync_ire"], f.out_scale,
                                      rf.SysParams["outputZero"]], dtype=np.float64)
        # where the next field read starts (decodefield/readfield offset logic)
        offset = f.nextfieldoffset - (readloc - decode["startloc"])
        start = start + offset
        prev = f
        i += 1
    out["skipped_starts"] = np.array(skipped, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, f"field_{system.lower()}.npz"), **out)


FIELDS_PIC_STRIDE = 97


def fields_fixture(case):
    """Consecutive fields of one capture through the reference's readfield
    walk (decodefield offsets, invalid fields skipped as readfield skips
    them)."""
    from field_cases import field_case_capture
    name, system, nfields = case[0], case[1], case[2]
    kw = dict(system=system, decode_analog_audio=0, decode_digital_audio=False)
    rf = refcore.RFDecode(**kw)
    src = BlockSource(rf, None, 1)
    fieldcls = refcore.FieldPAL if system == "PAL" else refcore.FieldNTSC
    if system == "PAL":
        src.readlen = rf.linelen * 400
    else:
        src.readlen = ((rf.linelen * 350) // 16384) * 16384
    cap, meta = field_case_capture(case, rf.blocklen, src.readlen)
    src.cap = cap
    out = {"capture_sha256": np.array(sha(cap)), "capture_len": np.array(len(cap)), "mtf_level": np.array(1.0)}
    prev = None
    start = 0
    i = 0
    tries = 0
    skipped = []
    while i < nfields:
        rd = src.read_field(start)
        assert rd is not None, (name, i)
        decode, readloc = rd
        f = fieldcls(rf, decode, prevfield=prev, initphase=(i == 0), fields_written=i,
                     readloc=decode["startloc"])
        f.process()
        tries += 1
        assert tries < nfields + 6, name
        if not f.valid:
            skipped.append(start)
            start = start + f.nextfieldoffset
            prev = None
            continue
        dsout, _, _ = f.downscale(linesout=f.outlinecount, final=True)
        p = f"f{i}_"
        out[p + "start"] = np.array(start, dtype=np.float64)
        out[p + "readloc"] = np.array(readloc)
        out[p + "startloc"] = np.array(decode["startloc"])
        out[p + "pulse_start"] = np.array([q.start for q in f.rawpulses], dtype=np.int64)
        out[p + "pulse_len"] = np.array([q.len for q in f.rawpulses], dtype=np.int64)
        out[p + "valid_type"] = np.array([v[0] for v in f.validpulses], dtype=np.int64)
        out[p + "valid_start"] = np.array([v[1].start for v in f.validpulses], dtype=np.int64)
        out[p + "valid_good"] = np.array([bool(v[2]) for v in f.validpulses])
        out[p + "linelocs1"] = np.array(f.linelocs1, dtype=np.float64)
        out[p + "linelocs"] = np.array(f.linelocs, dtype=np.float64)
        out[p + "linebad"] = np.array(f.linebad, dtype=bool)
        out[p + "flags"] = np.array([int(f.isFirstField), f.linecount, f.lineoffset,
                                     f.fieldPhaseID, f.sync_confidence], dtype=np.int64)
        out[p + "nextfieldoffset"] = np.array(f.nextfieldoffset, dtype=np.float64)
        pic = np.asarray(f.dspicture)
        out[p + "dspicture_sha256"] = np.array(sha(pic))
        out[p + "dspicture_sub"] = pic[::FIELDS_PIC_STRIDE]
        start = start + f.nextfieldoffset - (readloc - decode["startloc"])
        prev = f
        i += 1
    out["nfields"] = np.array(nfields)
    out["skipped_starts"] = np.array(skipped, dtype=np.float64)
    for k, v in meta.items():
        out["meta_" + k] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, f"fields_{name}.npz"), **out)


def dropout_fixture(system, seed, nfields=3, ndrop=60):
    kw = dict(system=system, decode_analog_audio=0, decode_digital_audio=False)
    rf = refcore.RFDecode(**kw)
    src = BlockSource(rf, None, 1)
    fieldcls = refcore.FieldPAL if system == "PAL" else refcore.FieldNTSC
    if system == "PAL":
        src.readlen = rf.linelen * 400
    else:
        src.readlen = ((rf.linelen * 350) // 16384) * 16384
    fieldlen = int(rf.freq_hz / (rf.SysParams["FPS"] * 2))
    ncap = (nfields + 3) * fieldlen + src.readlen + 8 * rf.blocklen
    cap = synth_capture(system, ncap, seed=seed, start=CAPTURE_START, snr_db=38.0).numpy()
    spans = inject_dropouts(cap, seed + 1000, ndrop)
    src.cap = cap
    out = {"capture_sha256": np.array(sha(cap)), "capture_len": np.array(ncap),
           "capture_seed": np.array(seed), "capture_start": np.array(CAPTURE_START), "snr_db": np.array(38.0),
           "drop_seed": np.array(seed + 1000), "drop_count": np.array(ndrop),
           "drop_spans": np.array(spans, dtype=np.int64), "mtf_level": np.array(1.0)}
    prev = None
    start = 0
    i = 0
    tries = 0
    while i < nfields:
        rd = src.read_field(start)
        assert rd is not None
        decode, readloc = rd
        f = fieldcls(rf, decode, prevfield=prev, initphase=(i == 0), fields_written=i,
                     readloc=decode["startloc"])
        f.process()
        tries += 1
        assert tries < nfields + 4
        if not f.valid:
            start = start + f.nextfieldoffset
            prev = None
            continue
        iserr = f.dropout_detect_demod()
        errmap = np.nonzero(iserr)[0]
        errlist = f.build_errlist(errmap) if len(errmap) and errmap[-1] > f.linelocs[f.lineoffset] else []
        lines, starts, ends = f.dropout_detect()
        p = f"f{i}_"
        out[p + "startloc"] = np.array(decode["startloc"])
        out[p + "length"] = np.array(len(decode["video"]))
        out[p + "linelocs"] = np.array(f.linelocs, dtype=np.float64)
        out[p + "flags"] = np.array([int(f.isFirstField), f.linecount, f.lineoffset], dtype=np.int64)
        out[p + "hsync_len"] = np.array(int(f.LT["hsync"][1]))
        out[p + "rfstd"] = np.array(float(refcore.nb_std(f.data["rfhpf"])))
        out[p + "errmap"] = errmap.astype(np.int64)
        out[p + "errlist"] = np.array(errlist, dtype=np.float64).reshape(-1, 2)
        out[p + "dropouts"] = np.array([lines, starts, ends], dtype=np.int64).reshape(3, -1)
        start = start + f.nextfieldoffset - (readloc - decode["startloc"])
        prev = f
        i += 1
    out["nfields"] = np.array(nfields)
    np.savez_compressed(os.path.join(HERE, f"dropouts_{system.lower()}.npz"), **out)


def rftbc_fixture(system, seed, nfields=2):
    kw = dict(system=system, decode_analog_audio=0, decode_digital_audio=False)
    rf = refcore.RFDecode(**kw)
    src = BlockSource(rf, None, 1)
    fieldcls = refcore.FieldPAL if system == "PAL" else refcore.FieldNTSC
    if system == "PAL":
        src.readlen = rf.linelen * 400
    else:
        src.readlen = ((rf.linelen * 350) // 16384) * 16384
    fieldlen = int(rf.freq_hz / (rf.SysParams["FPS"] * 2))
    ncap = (nfields + 2) * fieldlen + src.readlen + 8 * rf.blocklen
    cap = synth_capture(system, ncap, seed=seed, start=CAPTURE_START).numpy()
    src.cap = cap
    out = {"capture_sha256": np.array(sha(cap)), "capture_len": np.array(ncap), "capture_seed": np.array(seed),
           "capture_start": np.array(CAPTURE_START), "mtf_level": np.array(1.0),
           "video_white": np.array(float(rf.delays["video_white"])), "inlinelen": np.array(float(rf.linelen))}
    prev = None
    start = 0
    i = 0
    while i < nfields:
        decode, readloc = src.read_field(start)
        f = fieldcls(rf, decode, prevfield=prev, initphase=(i == 0), fields_written=i,
                     readloc=decode["startloc"])
        f.process()
        if not f.valid:
            start = start + f.nextfieldoffset
            prev = None
            continue
        rt = np.asarray(f.rf_tbc())
        linelen = int(round(f.inlinelen))
        p = f"f{i}_"
        out[p + "startloc"] = np.array(decode["startloc"])
        out[p + "length"] = np.array(len(decode["input"]))
        out[p + "linelocs"] = np.array(f.linelocs, dtype=np.float64)
        out[p + "flags"] = np.array([int(f.isFirstField), f.linecount, f.lineoffset], dtype=np.int64)
        out[p + "sha256"] = np.array(sha(rt.astype(np.int16)))
        out[p + "n"] = np.array(len(rt))
        out[p + "sub"] = rt[::13].astype(np.int16)
        out[p + "lines"] = np.stack([rt[20 * linelen:21 * linelen], rt[150 * linelen:151 * linelen]]).astype(np.int16)
        start = start + f.nextfieldoffset - (readloc - decode["startloc"])
        prev = f
        i += 1
    out["nfields"] = np.array(nfields)
    np.savez_compressed(os.path.join(HERE, f"rftbc_{system.lower()}.npz"), **out)


def lds_fixture():
    import io
    from lddecode import utils as refutils
    rng = np.random.default_rng(71)
    data = rng.integers(0, 256, 5 * 1200, dtype=np.uint8)
    out = {"packed": data}
    # (first sample, samples): the reference's file loader on an in-memory .lds (it needs
    # multiples of 4 samples, as the decoder reads them)
    cases = [(0, 4000), (401, 4000), (0, 4096), (2, 4096), (5, 1000), (8, 1), (3, 2048), (3001, 1024)]
    f = io.BytesIO(data.tobytes())
    for k, (sample, readlen) in enumerate(cases):
        out[f"case{k}"] = np.array([sample, readlen])
        out[f"out{k}"] = np.asarray(refutils.load_packed_data_4_40(f, sample, readlen))
    out["ncases"] = np.array(len(cases))
    np.savez_compressed(os.path.join(HERE, "lds_unpack.npz"), **out)


def notch_fixture(seed=33):
    kw = dict(system="PAL", decode_analog_audio=44100, decode_digital_audio=True,
              extra_options={"PAL_V4300D_NotchFilter": True})
    rf = refcore.RFDecode(**kw)
    cap = synth_capture("PAL", rf.blocklen + 4096, seed=seed).numpy()
    t = np.arange(len(cap), dtype=np.float64)
    # spurious carriers inside the notch search band (8.42-8.6 MHz), as the
    # LD-V4300D players add them
    tone = 300.0 * np.cos(2 * np.pi * 8.52e6 / 40e6 * t) + 120.0 * np.cos(2 * np.pi * 8.471e6 / 40e6 * t + 1.0)
    cap = np.clip(np.round(cap + tone), -32768, 32767).astype(np.int16)
    block = cap[1000:1000 + rf.blocklen].copy()
    out = {"block": block}
    rv = rf.demodblock(data=block, mtf_level=1, cut=True)
    for k in rv["video"].dtype.names:
        v = np.asarray(rv["video"][k])
        out[f"m1_{k}"] = v[::STRIDE]
        out[f"m1_{k}_sum"] = np.array([np.sum(v.astype(np.float64)), np.sum(v.astype(np.float64) ** 2)])
    out["m1_rfhpf"] = rv["rfhpf"][::STRIDE]
    out["m1_efm"] = rv["efm"][::STRIDE]
    out["m1_audio_left"] = np.asarray(rv["audio"]["audio_left"])
    # the bins the reference zeroes (its own rule, on the block's spectrum)
    X = np.fft.fft(block.astype(np.float64))
    sl = slice(int(rf.blocklen * (8.42 / rf.freq)), int(1 + (rf.blocklen * (8.6 / rf.freq))))
    sq = np.sqrt(X[sl].real ** 2 + X[sl].imag ** 2)
    m = np.mean(sq) + np.std(sq) * 3
    zero = sorted({sl.start + i + d for i in np.where(sq > m)[0] for d in (-1, 0, 1)})
    out["notch_bins"] = np.array(zero, dtype=np.int64)
    out["notch_slice"] = np.array([sl.start, sl.stop])
    out["mtf_scaled"] = np.array([((1 * rf.mtf_mult) + rf.mtf_offset) * rf.DecoderParams["MTF_basemult"]])
    # the same block without the notch, to show that it acts
    rf2 = refcore.RFDecode(system="PAL", decode_analog_audio=44100, decode_digital_audio=True)
    rv2 = rf2.demodblock(data=block, mtf_level=1, cut=True)
    out["plain_demod"] = np.asarray(rv2["video"]["demod"])[::STRIDE]
    np.savez_compressed(os.path.join(HERE, "demod_pal_notch.npz"), **out)


def smoothing_fixture(system, seed, smoothing=2.0):
    kw = dict(system=system, decode_analog_audio=0, decode_digital_audio=False)
    rf = refcore.RFDecode(**kw)
    src = BlockSource(rf, None, 1)
    fieldcls = refcore.FieldPAL if system == "PAL" else refcore.FieldNTSC
    src.readlen = rf.linelen * 400 if system == "PAL" else ((rf.linelen * 350) // 16384) * 16384
    fieldlen = int(rf.freq_hz / (rf.SysParams["FPS"] * 2))
    ncap = 2 * fieldlen + src.readlen + 8 * rf.blocklen
    cap = synth_capture(system, ncap, seed=seed, start=CAPTURE_START).numpy()
    src.cap = cap
    start = 0
    while True:
        decode, readloc = src.read_field(start)
        f = fieldcls(rf, decode, prevfield=None, initphase=True, fields_written=0, readloc=decode["startloc"],
                     wow_level_adjust_smoothing=smoothing)
        f.process()
        if f.valid:
            break
        start += f.nextfieldoffset
    f.downscale(linesout=f.outlinecount, final=True)
    np.savez_compressed(os.path.join(HERE, f"tbc_smoothing_{system.lower()}.npz"),
                        capture_sha256=np.array(sha(cap)), capture_len=np.array(ncap), capture_seed=np.array(seed),
                        capture_start=np.array(CAPTURE_START), mtf_level=np.array(1.0), smoothing=np.array(smoothing),
                        start=np.array(start), startloc=np.array(decode["startloc"]),
                        linelocs=np.array(f.linelocs, dtype=np.float64),
                        flags=np.array([int(f.isFirstField), f.linecount, f.lineoffset], dtype=np.int64),
                        levels=np.array([rf.DecoderParams["ire0"], rf.DecoderParams["hz_ire"],
                                         rf.DecoderParams["vsync_ire"], f.out_scale, rf.SysParams["outputZero"]]),
                        dspicture=np.asarray(f.dspicture))


PIC_STRIDE = 11
# (method, perturbed line locations, level smoothing)
WOW_CASES = (("cubic", False, 0.0), ("quadratic", True, 0.0), ("cubic", True, 0.0), ("cubic", True, 2.0))


def perturb_linelocs(ll, lineoffset):
    """Sinusoidal wow of 0.8 samples (period 37 lines) plus two lines moved
    by +4 / -5 samples (H-sync errors that the 15*MAD rule catches)."""
    ll = np.asarray(ll, dtype=np.float64)
    out = ll + 0.8 * np.sin(2 * np.pi * np.arange(len(ll)) / 37.0)
    out[lineoffset + 60] += 4.0
    out[lineoffset + 140] -= 5.0
    return out


def wow_interp_fixture(system, seed):
    kw = dict(system=system, decode_analog_audio=0, decode_digital_audio=False)
    rf = refcore.RFDecode(**kw)
    src = BlockSource(rf, None, 1)
    fieldcls = refcore.FieldPAL if system == "PAL" else refcore.FieldNTSC
    src.readlen = rf.linelen * 400 if system == "PAL" else ((rf.linelen * 350) // 16384) * 16384
    fieldlen = int(rf.freq_hz / (rf.SysParams["FPS"] * 2))
    ncap = 2 * fieldlen + src.readlen + 8 * rf.blocklen
    cap = synth_capture(system, ncap, seed=seed, start=CAPTURE_START).numpy()
    src.cap = cap
    start = 0
    while True:
        decode, readloc = src.read_field(start)
        f = fieldcls(rf, decode, prevfield=None, initphase=True, fields_written=0, readloc=decode["startloc"])
        f.process()
        if f.valid:
            break
        start += f.nextfieldoffset
    base = np.array(f.linelocs, dtype=np.float64)
    out = dict(capture_sha256=np.array(sha(cap)), capture_len=np.array(ncap), capture_seed=np.array(seed),
               capture_start=np.array(CAPTURE_START), mtf_level=np.array(1.0), start=np.array(start),
               startloc=np.array(decode["startloc"]), pic_stride=np.array(PIC_STRIDE),
               flags=np.array([int(f.isFirstField), f.linecount, f.lineoffset], dtype=np.int64),
               levels=np.array([rf.DecoderParams["ire0"], rf.DecoderParams["hz_ire"],
                                rf.DecoderParams["vsync_ire"], f.out_scale, rf.SysParams["outputZero"]]))
    for i, (method, perturbed, smoothing) in enumerate(WOW_CASES):
        ll = perturb_linelocs(base, f.lineoffset) if perturbed else base.copy()
        f.linelocs = ll
        f.wow_interpolation_method = method
        f.wow_level_adjust_smoothing = smoothing
        f.downscale(linesout=f.outlinecount, final=True)
        wow = f.wowfactors
        med = np.median(wow)
        p = f"c{i}_"
        out[p + "case"] = np.array([method, str(perturbed), str(smoothing)])
        out[p + "smoothing"] = np.array(smoothing)
        out[p + "linelocs"] = ll
        out[p + "coords"] = f.interpolated_pixel_locs[::COORD_STRIDE]
        out[p + "wow"] = wow[::COORD_STRIDE]
        out[p + "wow_stats"] = np.array([len(wow), med, np.median(np.abs(wow - med))])
        out[p + "picture"] = np.asarray(f.dspicture)[::PIC_STRIDE]
        out[p + "picture_sha256"] = np.array(sha(np.asarray(f.dspicture)))
    np.savez_compressed(os.path.join(HERE, f"wow_interp_{system.lower()}.npz"), **out)


def audio2_fixture(system, seed):
    from audio_cases import AUDIO2_CASES, AUDIO2_STRIDE, audio2_inputs
    rf = refcore.RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=False)
    out = {"seed": np.array(seed)}
    for tag, n in AUDIO2_CASES:
        left, right = audio2_inputs((rf.SysParams["audio_lfreq"], rf.SysParams["audio_rfreq"]), seed, n)
        out[f"{tag}_in_sha256"] = np.array(sha(np.concatenate([left, right])))
        res = rf.audio_phase2(np.rec.fromarrays([left, right], names=["audio_left", "audio_right"]))
        for ch in ("left", "right"):
            v = np.asarray(res["audio_" + ch], dtype=np.float64)
            out[f"{tag}_{ch}_out"] = v[::AUDIO2_STRIDE]
            out[f"{tag}_{ch}_sum"] = np.array([np.sum(v), np.sum((v - v.mean()) ** 2)])
            out[f"{tag}_{ch}_len"] = np.array(len(v))
    np.savez_compressed(os.path.join(HERE, f"audio2_{system.lower()}.npz"), **out)


def lut_fixture():
    lut = np.load(os.path.join(REF, "lddecode", "sinc_lut.npz"))["downscale_sinc_lut"]
    rows = np.concatenate([np.arange(0, 65537, 997), [32767, 32768, 65535, 65536]])
    np.savez_compressed(os.path.join(HERE, "sinc_lut_rows.npz"), rows=rows, values=lut[rows],
                        sha256=np.array(sha(lut)))


def audio_fixture():
    out = {}
    for k, (name, system, linecount, freq, toff, dtype, alen, glitch) in enumerate(AUDIO_CASES):
        sp = refcore.SysParams_NTSC if system == "NTSC" else refcore.SysParams_PAL
        lineinfo, left, right, linelen = audio_case_inputs(
            system, linecount, dtype, alen, glitch, 500 + k, sp["line_period"],
            (sp["audio_lfreq"], sp["audio_rfreq"]))
        locs, swow, arange, frametime = refcore._downscale_audio_compute_locs_and_swow(
            lineinfo, sp["line_period"], linelen, linecount, toff, freq, 32)
        o16, failed = refcore._downscale_audio_to_output(arange, locs, swow, left, right,
                                                         sp["audio_lfreq"], sp["audio_rfreq"])
        out[name + "_locs"] = locs
        out[name + "_swow"] = swow
        out[name + "_out"] = o16
        out[name + "_next"] = np.array(arange[-1] - frametime)
        out[name + "_failed"] = np.array(failed)
    np.savez_compressed(os.path.join(HERE, "audio_downscale.npz"), **out)


# (name, audio length, locs): run boundaries before the buffer's start
AUDIO_SLICE_CASES = [
    ("both_negative", 28800, [-90.4, -61.7, -33.2, -4.9]),
    ("below_minus_len", 28800, [-40000.2, 7.9, 35.3, 63.6]),
    ("below_minus_len_neg_end", 28800, [-40000.6, -100.2, -71.9]),
]


def audio_slices_fixture():
    out = {}
    sp = refcore.SysParams_NTSC
    rng = np.random.default_rng(77)
    for name, alen, locs in AUDIO_SLICE_CASES:
        left = (sp["audio_lfreq"] + rng.integers(-150000, 150000, alen)).astype(np.float32)
        right = (sp["audio_rfreq"] + rng.integers(-150000, 150000, alen)).astype(np.float32)
        locs = np.array(locs, dtype=np.float64)
        swow = 1.0 + 0.001 * np.arange(len(locs), dtype=np.float64)
        arange = np.arange(len(locs), dtype=np.float64)
        o16, failed = refcore._downscale_audio_to_output(arange, locs, swow, left, right,
                                                         sp["audio_lfreq"], sp["audio_rfreq"])
        out[name + "_left"] = left
        out[name + "_right"] = right
        out[name + "_locs"] = locs
        out[name + "_swow"] = swow
        out[name + "_out"] = o16
        out[name + "_failed"] = np.array(failed)
    np.savez_compressed(os.path.join(HERE, "audio_slices.npz"), **out)


def efm_pll_fixture():
    from lddecode import efm_pll
    from efm_cases import EFM_CASES, efm_case, split
    out = {}
    for c in EFM_CASES:
        name = c[0]
        x, bufs = efm_case(name)
        pll = efm_pll.EFM_PLL()
        res = [np.array(pll.process(b), dtype=np.int8) for b in split(x, bufs)]
        out[name + "_in_sha256"] = np.array(sha(x))
        out[name + "_t"] = np.concatenate(res)
        out[name + "_counts"] = np.array([len(r) for r in res], dtype=np.int64)
        out[name + "_state_f"] = np.array([pll.delta, pll.currentPeriod, pll.phaseAdjust, pll.refClockTime])
        out[name + "_state_i"] = np.array([pll.zcPreviousInput, pll.frequencyHysteresis, pll.tCounter],
                                          dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "efm_pll.npz"), **out)


def ac3_fixture():
    from lddecode import ac3rf
    sys.path.insert(0, REPO)
    from oracle.ac3 import dqpsk_signal

    tx = np.random.default_rng(4242).integers(0, 4, 6000).astype(np.uint8)
    table = np.cos(2 * np.pi * np.arange(1000) / 1000).astype(np.float32)
    clean = dqpsk_signal(tx, cos_table=table)
    noisy = dqpsk_signal(tx, noise_int=64, noise_scale=0.25 / 74.5, seed=99, cos_table=table)

    # baseband I/Q through the reference's own stages (demodulate_to_symbols
    # without its DPLL, ac3rf.py:372-394)
    d = ac3rf.Ac3RfDemodulator(40e6)
    data = clean
    for st in d.pre_mix_filters:
        data = st.process(data)
    ph = (d._phase_step * np.arange(len(data))) & ((1 << d._PHASE_ACCUM_BITS) - 1)
    re, im = data * d._cos_lut[ph], data * d._sin_lut[ph]
    for st in d.post_mix_filters:
        re, im = st.process(re, im)
    windows = np.array([[0, 3000], [20000, 23000], [len(re) - 3000, len(re)]])
    iq_i = np.concatenate([re[a:b] for a, b in windows])
    iq_q = np.concatenate([im[a:b] for a, b in windows])

    d = ac3rf.Ac3RfDemodulator(40e6)
    blocks = [100001, 65536, 999999]
    rx, pos, k = b"", 0, 0
    while pos < len(clean):
        n = blocks[k % 3]
        rx += d.demodulate_to_symbols(clean[pos:pos + n])
        pos += n
        k += 1
    rx_noisy = ac3rf.Ac3RfDemodulator(40e6).demodulate_to_symbols(noisy)
    np.savez_compressed(os.path.join(HERE, "ac3_loopback.npz"), tx=tx, cos_table=table,
                        n_iq=np.array(len(re)), windows=windows, iq_i=iq_i, iq_q=iq_q,
                        rx_clean=np.frombuffer(rx, np.uint8), rx_noisy=np.frombuffer(rx_noisy, np.uint8),
                        blocks=np.array(blocks), clean_sha256=np.array(sha(clean)),
                        hb19=ac3rf.halfband_kaiser(19), hb23=ac3rf.halfband_kaiser(23),
                        rrc=ac3rf.rrc_filter(55, 2.5e6 / ac3rf.SYMBOL_RATE, 0.7),
                        noisy_sha256=np.array(sha(noisy)))


def main():
    if sys.argv[1:] == ["dropouts"]:
        dropout_fixture("NTSC", seed=41)
        dropout_fixture("PAL", seed=42)
        return
    if sys.argv[1:] == ["audio2"]:
        audio2_fixture("NTSC", seed=81)
        audio2_fixture("PAL", seed=82)
        return
    if sys.argv[1:] == ["smoothing"]:
        smoothing_fixture("NTSC", seed=21)
        smoothing_fixture("PAL", seed=22)
        return
    if sys.argv[1:] == ["wow"]:
        wow_interp_fixture("NTSC", seed=21)
        wow_interp_fixture("PAL", seed=22)
        return
    if sys.argv[1:] == ["notch"]:
        notch_fixture()
        return
    if sys.argv[1:2] == ["fields"]:
        from field_cases import FIELD_CASES
        for case in FIELD_CASES:
            if len(sys.argv) < 3 or case[0] in sys.argv[2:]:
                fields_fixture(case)
        return
    if sys.argv[1:] == ["efm_pll"]:
        efm_pll_fixture()
        return
    if sys.argv[1:] == ["audio_slices"]:
        audio_slices_fixture()
        return
    if sys.argv[1:] == ["lds"]:
        lds_fixture()
        return
    if sys.argv[1:] == ["rftbc"]:
        rftbc_fixture("NTSC", seed=21)
        rftbc_fixture("PAL", seed=22)
        return
    audio_fixture()
    audio_slices_fixture()
    efm_pll_fixture()
    from field_cases import FIELD_CASES
    for case in FIELD_CASES:
        fields_fixture(case)
    ac3_fixture()
    lut_fixture()
    for i, (name, kw) in enumerate(CONFIGS.items()):
        rf = filters_fixture(name, kw)
        if name in ("ntsc", "pal"):
            demod_fixture(name, rf, kw, seed=11 + i)
    field_fixture("NTSC", seed=21)
    field_fixture("PAL", seed=22)
    dropout_fixture("NTSC", seed=41)
    dropout_fixture("PAL", seed=42)
    rftbc_fixture("NTSC", seed=21)
    rftbc_fixture("PAL", seed=22)
    lds_fixture()
    notch_fixture()
    smoothing_fixture("NTSC", seed=21)
    smoothing_fixture("PAL", seed=22)
    audio2_fixture("NTSC", seed=81)
    audio2_fixture("PAL", seed=82)
    wow_interp_fixture("NTSC", seed=21)
    wow_interp_fixture("PAL", seed=22)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
