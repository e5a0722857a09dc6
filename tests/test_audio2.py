"""Analog audio stage 2 (RFDecode.audio_phase2, lddecode/core.py:884-950):
the oracle pinned to the reference's outputs on seeded stage-1 audio with
dropout spikes (tests/golden/audio2_*.npz), one field-length input and one
longer input stitched from overlapping transforms; and on the B200 the GPU
form (ldg_audio_phase2) against the oracle and the reference."""

import hashlib
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, golden
from ldgpu.rfdecode import RFParams
from oracle import audio2 as oa2

sys.path.insert(0, GOLDEN)
from audio_cases import AUDIO2_CASES, AUDIO2_STRIDE, audio2_inputs  # noqa: E402

SYSTEMS = ["NTSC", "PAL"]


def _case(system):
    g = golden("audio2_" + system.lower())
    rf = RFParams(system=system, decode_analog_audio=44100)
    centers = (rf.SysParams["audio_lfreq"], rf.SysParams["audio_rfreq"])
    filters = (rf.audio["left"].audio2_filter, rf.audio["right"].audio2_filter)
    return g, rf, centers, filters


def _inputs(g, centers, tag, n):
    left, right = audio2_inputs(centers, int(g["seed"]), n)
    assert hashlib.sha256(np.concatenate([left, right]).tobytes()).hexdigest() == str(g[f"{tag}_in_sha256"])
    return left, right


@pytest.mark.parametrize("system", SYSTEMS)
def test_oracle_matches_reference(system):
    g, rf, centers, filters = _case(system)
    for tag, n in AUDIO2_CASES:
        left, right = _inputs(g, centers, tag, n)
        outs = oa2.audio_phase2(left, right, rf.blocklen, centers, filters)
        for ch, v in zip(("left", "right"), outs):
            assert len(v) == int(g[f"{tag}_{ch}_len"])
            np.testing.assert_allclose(np.asarray(v, np.float64)[::AUDIO2_STRIDE], g[f"{tag}_{ch}_out"],
                                       rtol=0, atol=0.25)


@pytest.mark.gpu
@pytest.mark.parametrize("system", SYSTEMS)
def test_gpu_matches_oracle_and_reference(cuda_ok, system):
    from ldgpu import RFDecode
    g, _, centers, filters = _case(system)
    rf = RFDecode(system=system, decode_analog_audio=44100)
    for tag, n in AUDIO2_CASES:
        left, right = _inputs(g, centers, tag, n)
        got = rf.audio_phase2(np.rec.fromarrays([left, right], names=["audio_left", "audio_right"]))
        want = oa2.audio_phase2(left, right, rf.blocklen, centers, filters)
        for ch, w in zip(("left", "right"), want):
            v = np.asarray(got["audio_" + ch], np.float64)
            d = v - np.asarray(w, np.float64)
            rms, mx = float(np.sqrt(np.mean(d * d))), float(np.abs(d).max())
            print(system, tag, ch, "GPU vs oracle Hz: rms", rms, "max", mx)
            assert len(v) == n and rms < 2.0 and mx < 20.0
            assert np.abs(v[::AUDIO2_STRIDE] - g[f"{tag}_{ch}_out"]).max() < 20.0
    rf.close()
