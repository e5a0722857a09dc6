"""Analog audio downscale (ldgpu.audio) against the reference's outputs on
seeded cases (tests/golden/audio_downscale.npz), and the sample-count pins of
the reference's own tests/test_audio_rate.py."""

import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, golden

sys.path.insert(0, GOLDEN)
from audio_cases import AUDIO_CASES, audio_case_inputs  # noqa: E402

from ldgpu import audio as A  # noqa: E402
from ldgpu.params import sysparams  # noqa: E402


@pytest.mark.parametrize("case", AUDIO_CASES, ids=[c[0] for c in AUDIO_CASES])
def test_downscale_audio_matches_reference(case):
    g = golden("audio_downscale")
    name, system, linecount, freq, toff, dtype, alen, glitch = case
    k = AUDIO_CASES.index(case)
    sp = sysparams(system)
    lineinfo, left, right, linelen = audio_case_inputs(
        system, linecount, dtype, alen, glitch, 500 + k, sp["line_period"], (sp["audio_lfreq"], sp["audio_rfreq"]))
    locs, swow, arange, frametime = A.compute_locs_and_swow(lineinfo, sp["line_period"], linelen, linecount,
                                                            toff, freq, 32)
    np.testing.assert_array_equal(locs, g[name + "_locs"])
    np.testing.assert_array_equal(swow, g[name + "_swow"])
    assert arange[-1] - frametime == float(g[name + "_next"])
    out, failed = A.to_output(arange, locs, swow, left, right, sp["audio_lfreq"], sp["audio_rfreq"])
    np.testing.assert_array_equal(out, g[name + "_out"])
    assert failed == bool(g[name + "_failed"])


def test_downscale_audio_entry_point_and_warning(caplog):
    """downscale_audio(audio, lineinfo, rf, ...) with an RFDecode-like object,
    the rv dict, and the mute warning of a capture too short for the field."""
    from ldgpu.rfdecode import RFParams
    rf = RFParams(system="NTSC", decode_analog_audio=44100)
    g = golden("audio_downscale")
    name, system, linecount, freq, toff, dtype, alen, glitch = AUDIO_CASES[3]
    sp = rf.SysParams
    lineinfo, left, right, linelen = audio_case_inputs(
        system, linecount, dtype, alen, glitch, 503, sp["line_period"], (sp["audio_lfreq"], sp["audio_rfreq"]))
    assert linelen == rf.linelen and rf.Filters["audio_fdiv"] == 32
    audio = np.rec.array([left, right], names=["audio_left", "audio_right"])
    rv = {}
    with caplog.at_level("WARNING"):
        out, nxt = A.downscale_audio(audio, lineinfo, rf, linecount, toff, freq, rv)
    assert "muting samples" in caplog.text
    np.testing.assert_array_equal(out, g[name + "_out"])
    assert rv["audio_next_offset"] == nxt == float(g[name + "_next"])


def _count(freq, linecount=525, linelen=910):
    lineinfo = np.arange(0, (linecount + 4) * linelen, linelen, dtype=np.double)
    _, swow, arange, _ = A.compute_locs_and_swow(lineinfo, sysparams("NTSC")["line_period"], linelen,
                                                 linecount, 0.0, freq, 32)
    return len(arange) - 1, swow


def test_ntsc_locked_rate_sample_counts():
    """Pins of the reference's tests/test_audio_rate.py: -2.8 gives exactly
    1470 samples per 525-line frame with unity wow; 44100 gives 1471."""
    n, swow = _count(-2.8)
    assert n == 1470
    np.testing.assert_allclose(swow, 1.0, atol=1e-9)
    assert 1_000_000 / sysparams("NTSC")["line_period"] * 2.8 == 44055.944055944055
    assert _count(44100)[0] == 1471


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
@pytest.mark.parametrize("freq", [44100, 48000, 8000, -4])
def test_field_clocks_vectorised_equals_scalar(system, freq):
    """The batched path's per-field output clocks (ldgpu.audio.field_clocks)
    equal Field.downscale's scalar av_offset + compute_locs_and_swow set-up
    field by field, including the first field (no lastfieldwritten)."""
    from ldgpu.audio import av_offset, field_clock, field_clocks
    from ldgpu.rfdecode import RFParams
    rf = RFParams(system=system)
    rng = np.random.default_rng(4)
    n = 40
    per_field = rf.freq_hz / rf.SysParams["FPS"] / 2
    startloc = (np.arange(n) * per_field + rng.integers(-3000, 3000, n)).astype(np.int64) // 31712 * 31712
    isfirst = (np.arange(n) % 2 == 0)
    linecount = np.where(isfirst, 262 if system == "NTSC" else 312, 263 if system == "NTSC" else 313)
    for first, count in ((0, n), (7, 13)):
        off, gap, nt, nxt = field_clocks(rf, startloc, isfirst, linecount, first, count, freq)
        for j in range(count):
            i = first + j
            lfw = None if i == 0 else (i, int(startloc[i - 1]))
            o = av_offset(rf, int(startloc[i]), bool(isfirst[i]), freq, lfw)
            t0, sg, ntk, nx = field_clock(rf.SysParams["line_period"], int(linecount[i]), o, freq)
            assert (off[j], gap, nt[j], nxt[j]) == (t0, sg, ntk, nx), (i, off[j], t0)


@pytest.mark.parametrize("name", ["both_negative", "below_minus_len", "below_minus_len_neg_end"])
def test_runs_before_buffer_follow_reference_slices(name):
    """Runs that start before the audio buffer (tests/golden/audio_slices.npz,
    the reference's _downscale_audio_to_output on hand-made boundaries): both
    bounds negative wrap to the buffer's end, a start below -len clamps to 0,
    and each mean divides by the slice's own length."""
    g = golden("audio_slices")
    sp = sysparams("NTSC")
    locs = g[name + "_locs"]
    arange = np.arange(len(locs), dtype=np.float64)
    out, failed = A.to_output(arange, locs, g[name + "_swow"], g[name + "_left"], g[name + "_right"],
                              sp["audio_lfreq"], sp["audio_rfreq"])
    np.testing.assert_array_equal(out, g[name + "_out"])
    assert failed == bool(g[name + "_failed"])


def test_run_across_buffer_start_is_muted():
    """A run from before the buffer's start to after it is an empty numpy
    slice, whose mean makes the reference raise ZeroDivisionError; the
    restatement mutes that sample and reports it."""
    sp = sysparams("NTSC")
    a = np.full(1000, sp["audio_lfreq"], dtype=np.float32)
    locs = np.array([-14.3, 13.7, 41.2])
    out, failed = A.to_output(np.arange(3.0), locs, np.ones(3), a, a, sp["audio_lfreq"], sp["audio_rfreq"])
    assert failed and out[0] == 0 and out[1] == 0
