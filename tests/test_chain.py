"""The native field chain (ldg_field_chain) against the host restatement of
Field.process(): same reads, same validity, same windows, identical
pulse-level line locations and bad-line flags, field parity and next-field
offsets, on oracle-demodulated multi-field NTSC and PAL captures read from
sample 0 (the first reads land mid-field and are invalid, as in the
reference).  Host code only: runs without a GPU."""

import ctypes

import numpy as np
import pytest

from helpers import oracle_capture
from ldgpu import lib as L
from ldgpu.fieldread import blocks_in_capture
from ldgpu.lines import host_field_chain, host_sync_runs, run_chain
from ldgpu.rfdecode import RFParams
from ldgpu.synth import synth_capture

NSAMPLES = {"NTSC": 5_200_000, "PAL": 6_000_000}


@pytest.fixture(scope="module", params=["NTSC", "PAL"])
def capture(request):
    system = request.param
    rf = RFParams(system=system)
    rf.delays = {"video_rot": 3}
    cap = synth_capture(system, NSAMPLES[system], seed=31, start=7777).numpy()
    nb = blocks_in_capture(rf, len(cap))
    keys = ("demod", "demod_05", "demod_burst") + (("demod_pilot",) if system == "PAL" else ())
    arrays = oracle_capture(rf, cap, 0, nb, rf.scaled_mtf(1.0), keys=keys)
    return rf, arrays, nb


def test_chain_matches_host_process(capture, monkeypatch):
    from ldgpu.linelocs import FieldLogic
    rf, arrays, nb = capture
    orig = FieldLogic.compute_linelocs

    def recording(self):
        rv = orig(self)
        ll1, err, nxt = rv
        self._pulse_level = (None if ll1 is None else np.array(ll1, np.float64),
                             None if err is None else np.array(err), nxt)
        return rv

    monkeypatch.setattr(FieldLogic, "compute_linelocs", recording)
    reads, _ = host_field_chain(rf, arrays, nb)
    runs = host_sync_runs(rf, arrays["demod_05"])
    plans, stop, st = run_chain(rf, runs, nb)
    assert stop == L.LDG_CHAIN_STOP_END
    assert len(plans) == len(reads)
    nvalid = 0
    for p, (w, f) in zip(plans, reads):
        assert (p.startloc, p.length, p.readloc) == (w.startloc, w.length, w.readloc)
        assert bool(p.valid) == bool(f.valid)
        if not f.valid:
            assert p.nextfieldoffset == pytest.approx(f.nextfieldoffset, abs=0)
            continue
        nvalid += 1
        ll1, err, nxt = f._pulse_level
        bad = f.compute_deriv_error(ll1, err)
        n = p.proclines
        np.testing.assert_array_equal(np.frombuffer(p.linelocs1, np.float64)[:n], np.asarray(ll1, np.float64))
        np.testing.assert_array_equal(np.frombuffer(p.linebad, np.uint8)[:n].astype(bool), bad)
        assert bool(p.isfirst) == bool(f.isFirstField)
        assert p.linecount == (263 if f.isFirstField else 262)
        assert p.nextfieldoffset == nxt
        assert p.sync_confidence == f.sync_confidence
        assert p.hsync_len == int(f.LT["hsync"][1])
    assert nvalid >= 5
    print(rf.system, "reads", len(plans), "valid", nvalid)


def test_chain_resumes_from_state(capture):
    """Walking in pieces (max_plans) gives the same plans as one walk."""
    rf, arrays, nb = capture
    runs = host_sync_runs(rf, arrays["demod_05"])
    whole, _, _ = run_chain(rf, runs, nb)
    st = None
    parts = []
    while True:
        plans, stop, st = run_chain(rf, runs, nb, st, max_plans=2)
        parts.extend(plans)
        if stop != L.LDG_CHAIN_STOP_FULL:
            break
    assert len(parts) == len(whole)
    for a, b in zip(parts, whole):
        assert a.tobytes() == b.tobytes()


def test_chain_stops_on_level_recalibration():
    """No pulses in the very first read: the reference re-levels ire0 from
    the field's data, so the chain stops there (LDG_CHAIN_STOP_LEVELS)."""
    rf = RFParams(system="NTSC")
    z = np.zeros(0, np.int64)
    plans, stop, _ = run_chain(rf, (z, z, np.zeros(0)), 200)
    assert stop == L.LDG_CHAIN_STOP_LEVELS and len(plans) == 0


def test_abi_struct_sizes():
    h = L.load()
    assert len(L.ABI_STRUCTS) == 16
    for name, t in L.ABI_STRUCTS:
        assert h.ldg_abi_sizeof(name.encode()) == ctypes.sizeof(t), name


def test_parallel_chain_equals_serial(capture):
    """The chain walked in pieces joined at common states equals one walk."""
    from ldgpu.lines import parallel_chain
    rf, arrays, nb = capture
    runs = host_sync_runs(rf, arrays["demod_05"])
    whole, stop, st = run_chain(rf, runs, nb)
    for nthreads in (2, 3):
        got, stop2, st2 = parallel_chain(rf, runs, nb, None, nthreads, margin_blocks=100, min_seg_blocks=30)
        assert got.tobytes() == whole.tobytes()
        # a margin too short to reach a common state falls back to walking on
        got, stop2, st2 = parallel_chain(rf, runs, nb, None, nthreads, margin_blocks=0, min_seg_blocks=30)
        assert stop2 == stop and st2.start == st.start
        assert len(got) == len(whole)
        assert got.tobytes() == whole.tobytes()


def test_parallel_chain_concurrent_callers(capture):
    """Several host threads walking captures at once share the chain's
    thread pool; each gets the plans of its own sequential walk."""
    from concurrent.futures import ThreadPoolExecutor
    from ldgpu.lines import parallel_chain
    rf, arrays, nb = capture
    runs = host_sync_runs(rf, arrays["demod_05"])
    whole, _, _ = run_chain(rf, runs, nb)

    def one(k):
        got, _, _ = parallel_chain(rf, runs, nb, None, 2 + k % 3, margin_blocks=100, min_seg_blocks=30)
        return got.tobytes()

    with ThreadPoolExecutor(6) as ex:
        outs = list(ex.map(one, range(24)))
    assert all(o == whole.tobytes() for o in outs)


def test_chain_takes_previous_field_inputs(monkeypatch):
    """Seeded dropouts that hide a field's vertical interval make its line 0
    depend on the previous field's refined line locations (getLine0,
    core.py:2156-2239).  The chain first retries such a field with the range
    of +-32 samples around the previous field's pulse-level estimate and
    skip_check unknown: a plan made so (prev_range) is byte for byte the plan
    the exact inputs give.  Where the range leaves the field open it stops;
    given what getLine0 reads of the previous field (skip_check() >= 50,
    line0loc_prev, its sync confidence; here from the host restatement's
    previous field) it goes on.  Every plan equals the host restatement."""
    from ldgpu.fieldread import field_window
    from ldgpu.linelocs import FieldLogic
    from ldgpu.synth import inject_dropouts
    rf = RFParams(system="NTSC")
    rf.delays = {"video_rot": 3}
    fieldlen = int(40e6 / (rf.SysParams["FPS"] * 2))
    cap = synth_capture("NTSC", 12 * fieldlen, seed=5, start=1004, snr_db=36).numpy()
    inject_dropouts(cap, 6, 240)
    nb = blocks_in_capture(rf, len(cap))
    from helpers import OracleBlocks
    arrays = OracleBlocks(rf, cap, rf.scaled_mtf(1.0), ("demod", "demod_05", "demod_burst")).window(0, nb)
    orig = FieldLogic.compute_linelocs

    def recording(self):
        rv = orig(self)
        ll1, err, nxt = rv
        self._pulse_level = (None if ll1 is None else np.array(ll1, np.float64),
                             None if err is None else np.array(err), nxt)
        return rv

    monkeypatch.setattr(FieldLogic, "compute_linelocs", recording)
    reads, _ = host_field_chain(rf, arrays, nb)
    runs = host_sync_runs(rf, arrays["demod_05"])

    def with_exact_inputs(st):
        w_prev, prev = [r for r in reads[:len(plans)] if r[1].valid][-1]
        w = field_window(rf, st.start)
        x = L.ChainState.from_buffer_copy(st)
        x.prev_known, x.prev_conf = 1, int(prev.sync_confidence)
        x.prev_skip = 1 if prev.skip_check() >= 50 else 0
        x.prev_line0 = x.prev_line0_hi = float(np.asarray(prev.linelocs, np.float64)[prev.linecount]
                                               - (w.startloc - w_prev.startloc))
        return x

    st, plans, resolved, ranged = None, [], 0, 0
    while True:
        got, stop, st_next = run_chain(rf, runs, nb, st, max_plans=1)
        if len(got):
            if got[0].prev_range:
                ranged += 1
                one_x, _, _ = run_chain(rf, runs, nb, with_exact_inputs(st), max_plans=1)
                a = got.copy()
                a.prev_range = 0
                assert len(one_x) == 1 and a.tobytes() == one_x.tobytes()
            plans.extend(got)
            st = st_next
            continue
        if stop == L.LDG_CHAIN_STOP_END:
            break
        assert stop == L.LDG_CHAIN_STOP_PREV and not st_next.prev_known
        one_x, _, st = run_chain(rf, runs, nb, with_exact_inputs(st_next), max_plans=1)
        assert len(one_x) == 1
        plans.extend(one_x)
        resolved += 1
    assert resolved + ranged >= 1
    assert len(plans) == len(reads)
    for p, (w, f) in zip(plans, reads):
        assert (p.startloc, p.readloc) == (w.startloc, w.readloc)
        assert bool(p.valid) == bool(f.valid)
        if not f.valid:
            continue
        ll1, err, nxt = f._pulse_level
        n = p.proclines
        np.testing.assert_array_equal(np.frombuffer(p.linelocs1, np.float64)[:n], np.asarray(ll1, np.float64))
        np.testing.assert_array_equal(np.frombuffer(p.linebad, np.uint8)[:n].astype(bool),
                                      f.compute_deriv_error(ll1, err))
        assert bool(p.isfirst) == bool(f.isFirstField)
        assert p.nextfieldoffset == nxt
        assert p.sync_confidence == f.sync_confidence
    print(len(plans), "reads;", ranged, "decided from the previous field's estimate,", resolved, "with exact inputs")
