"""Pin the host line-location logic (ldgpu.linelocs, Field.process) against
the reference's golden fields.  Input: the oracle's demodulated field arrays
for the golden captures; integers (sync pulses, valid-pulse classes, line
count, field order, phase ID) must be identical and FP64 line locations
equal to well below a thousandth of a sample."""

import numpy as np
import pytest

from conftest import golden
from helpers import oracle_capture
from ldgpu.fieldread import field_window
from ldgpu.linelocs import FieldLogicNTSC, FieldLogicPAL, find_pulses
from ldgpu.rfdecode import RFParams
from ldgpu.synth import synth_capture


def _decode(rf, cap, start, mtf):
    w = field_window(rf, start)
    keys = ("demod", "demod_05", "demod_burst") + (("demod_pilot",) if rf.system == "PAL" else ())
    v = oracle_capture(rf, cap, w.first_block, w.nblocks, mtf, keys=keys)
    return {"video": v, "startloc": w.startloc}, w


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_field_process_matches_reference(system):
    g = golden("field_" + system.lower())
    rf = RFParams(system=system)
    rf.delays = {"video_rot": 3}
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    mtf = rf.scaled_mtf(float(g["mtf_level"]))
    cls = FieldLogicPAL if system == "PAL" else FieldLogicNTSC
    prev = None
    start = float(g["f0_start"])
    for i in range(2):
        p = f"f{i}_"
        assert start == pytest.approx(float(g[p + "start"]), abs=1e-6)
        decode, w = _decode(rf, cap, start, mtf)
        f = cls(rf, decode, prevfield=prev, initphase=(i == 0), fields_written=i, readloc=w.startloc)
        f.process()
        assert f.valid
        np.testing.assert_array_equal([q.start for q in f.rawpulses], g[p + "pulse_start"])
        np.testing.assert_array_equal([q.len for q in f.rawpulses], g[p + "pulse_len"])
        np.testing.assert_array_equal([v[0] for v in f.validpulses], g[p + "valid_type"])
        np.testing.assert_array_equal([v[1].start for v in f.validpulses], g[p + "valid_start"])
        np.testing.assert_array_equal([bool(v[2]) for v in f.validpulses], g[p + "valid_good"])
        np.testing.assert_allclose(f.linelocs1, g[p + "linelocs1"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(f.linelocs2, g[p + "linelocs2"], rtol=0, atol=1e-4)
        np.testing.assert_allclose(f.linelocs, g[p + "linelocs"], rtol=0, atol=1e-3)
        np.testing.assert_array_equal(f.linebad, g[p + "linebad"])
        flags = [int(f.isFirstField), f.linecount, f.lineoffset, f.fieldPhaseID, f.sync_confidence]
        np.testing.assert_array_equal(flags, g[p + "flags"])
        assert f.nextfieldoffset == pytest.approx(float(g[p + "nextfieldoffset"]), abs=1e-6)
        assert f.burstmedian == pytest.approx(float(g[p + "burstmedian"]), rel=1e-5)
        readloc = max(int(start - rf.blockcut), 0)
        start = start + f.nextfieldoffset - (readloc - w.startloc)
        prev = f


def test_find_pulses_edges():
    """Run detection: a leading run is dropped, a trailing run is dropped,
    lengths above 5000 are dropped (utils.py:1101-1140)."""
    x = np.full(20000, 10.0, np.float32)
    x[:5] = 0          # leading run (start 0): dropped
    x[100:150] = 0     # kept
    x[200:201] = 0     # length 1: kept
    x[1000:7000] = 0   # length 6000 > 5000: dropped
    x[19990:] = 0      # trailing: dropped
    p = find_pulses(x, 5.0)
    assert [(q.start, q.len) for q in p] == [(100, 50), (200, 1)]
    assert find_pulses(np.zeros(10, np.float32), 5.0) == []
    assert find_pulses(np.full(10, 9.0, np.float32), 5.0) == []


def _field_cases():
    import sys
    from conftest import GOLDEN
    if GOLDEN not in sys.path:
        sys.path.insert(0, GOLDEN)
    from field_cases import FIELD_CASES
    return FIELD_CASES


@pytest.mark.parametrize("case", _field_cases(), ids=[c[0] for c in _field_cases()])
def test_consecutive_fields_match_reference(case):
    """Ten or more consecutive fields per case (tests/golden/fields_<case>.npz:
    clean, 30 dB SNR, seeded dropouts, 0.8-sample wow, dropouts on vertical
    sync, PAL through its 8-field sequence), walked as LDdecode.readfield
    walks them (invalid reads skipped, the next read at the reference's
    offsets): the host restatement on the oracle's outputs gives the
    reference's integers exactly -- sync pulses, pulse classes, field order,
    line count, line offset, phase ID, sync confidence, bad lines -- and its
    line locations to a thousandth of a sample."""
    from field_cases import field_case_capture
    from helpers import OracleBlocks
    from ldgpu.fieldread import readlen_for
    name, system = case[0], case[1]
    g = golden("fields_" + name)
    rf = RFParams(system=system)
    rf.delays = {"video_rot": 3}
    cap, _ = field_case_capture(case, rf.blocklen, readlen_for(rf))
    assert len(cap) == int(g["capture_len"])
    keys = ("demod", "demod_05", "demod_burst") + (("demod_pilot",) if system == "PAL" else ())
    src = OracleBlocks(rf, cap, rf.scaled_mtf(float(g["mtf_level"])), keys)
    cls = FieldLogicPAL if system == "PAL" else FieldLogicNTSC
    prev, start, i, skipped = None, 0.0, 0, []
    while i < int(g["nfields"]):
        w = field_window(rf, start)
        f = cls(rf, {"video": src.window(w.first_block, w.nblocks), "startloc": w.startloc}, prevfield=prev,
                initphase=(i == 0), fields_written=i, readloc=w.startloc)
        f.process()
        if not f.valid:
            skipped.append(start)
            start = start + f.nextfieldoffset
            prev = None
            continue
        p = f"f{i}_"
        assert start == pytest.approx(float(g[p + "start"]), abs=1e-6), (name, i)
        np.testing.assert_array_equal([q.start for q in f.rawpulses], g[p + "pulse_start"])
        np.testing.assert_array_equal([q.len for q in f.rawpulses], g[p + "pulse_len"])
        np.testing.assert_array_equal([v[0] for v in f.validpulses], g[p + "valid_type"])
        np.testing.assert_array_equal([v[1].start for v in f.validpulses], g[p + "valid_start"])
        np.testing.assert_array_equal([bool(v[2]) for v in f.validpulses], g[p + "valid_good"])
        flags = [int(f.isFirstField), f.linecount, f.lineoffset, f.fieldPhaseID, f.sync_confidence]
        np.testing.assert_array_equal(flags, g[p + "flags"], err_msg=f"{name} field {i}")
        np.testing.assert_array_equal(f.linebad, g[p + "linebad"])
        np.testing.assert_allclose(f.linelocs1, g[p + "linelocs1"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(f.linelocs, g[p + "linelocs"], rtol=0, atol=1e-3)
        assert f.nextfieldoffset == pytest.approx(float(g[p + "nextfieldoffset"]), abs=1e-6)
        readloc = max(int(start - rf.blockcut), 0)
        start = start + f.nextfieldoffset - (readloc - w.startloc)
        prev = f
        i += 1
    np.testing.assert_allclose(skipped, g["skipped_starts"], atol=1e-6)
