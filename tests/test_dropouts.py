"""Dropout detection (Field.dropout_detect, lddecode/core.py:2829-2983):
the oracle pinned against the reference's golden fields (captures with
seeded dropouts, tests/golden/dropouts_*.npz).

* The sequential stages (error-span merge, spans to TBC line ranges) run on
  the reference's own error samples and must give its spans and dropouts
  exactly.
* The per-sample mask runs on the oracle's demodulation of the same capture
  (float32 outputs within an ulp of the reference's): the rfhpf standard
  deviation agrees to 1e-5 and the error samples to a few in thousands; the
  final dropouts are the same."""

import hashlib

import numpy as np
import pytest

from conftest import golden
from helpers import oracle_capture
from ldgpu.rfdecode import RFParams
from ldgpu.synth import inject_dropouts, synth_capture
from oracle import demod as odemod
from oracle import dropouts as odrop

SYSTEMS = ["NTSC", "PAL"]


def _field(g, i):
    p = f"f{i}_"
    isfirst, linecount, lineoffset = (int(x) for x in g[p + "flags"])
    return dict(ll=g[p + "linelocs"], isfirst=bool(isfirst), linecount=linecount, lineoffset=lineoffset,
                hsync_len=int(g[p + "hsync_len"]), errmap=g[p + "errmap"], errlist=g[p + "errlist"],
                drops=g[p + "dropouts"], rfstd=float(g[p + "rfstd"]), startloc=int(g[p + "startloc"]),
                length=int(g[p + "length"]))


@pytest.mark.parametrize("system", SYSTEMS)
def test_oracle_merge_and_lines_match_reference(system):
    g = golden("dropouts_" + system.lower())
    rf = RFParams(system=system)
    outw = rf.SysParams["outlinelen"]
    total = 0
    for i in range(int(g["nfields"])):
        f = _field(g, i)
        el = odrop.build_errlist(f["errmap"], f["ll"], f["lineoffset"], rf.freq)
        np.testing.assert_array_equal(np.array(el, np.float64).reshape(-1, 2), f["errlist"])
        iserr = np.zeros(int(f["errmap"][-1]) + 1, bool)
        iserr[f["errmap"]] = True
        lines, starts, ends = odrop.detect(iserr, f["ll"], f["lineoffset"], f["linecount"], rf.freq, outw)
        np.testing.assert_array_equal(np.array([lines, starts, ends], np.int64).reshape(3, -1), f["drops"])
        total += len(lines)
    assert total > 20


def test_oracle_merge_edge_cases():
    ll = np.arange(0, 300 * 2500, 2500, dtype=np.float64)
    # one isolated error sample: a single span, not padded
    assert odrop.build_errlist([5000], ll, 1, 40.0) == [(5000, 5000)]
    # the span grows by 1.7x the distance to its start; a gap of more than
    # 20 samples past its end closes it (padded by -8 / +4)
    el = odrop.build_errlist([5000, 5010, 5030, 5100, 9000], ll, 1, 40.0)
    assert el == [(4992, 5000 + 30 * 1.7 + 4), (5092, 5104), (9000, 9000)]
    # the growth stops at 12 samples per MHz (480 at 40 MHz)
    el = odrop.build_errlist(list(range(5000, 5601, 10)), ll, 1, 40.0)
    assert el == [(4992, 5000 + 480.0 + 4), (5510, 5510 + 90 * 1.7)]  # the last span is not padded
    # a span across line ends is split into one dropout per line
    drops = odrop.errlist_to_tbc([(2500 * 3 + 100, 2500 * 5 + 50)], ll, 1, 262, 910)
    assert [d[0] for d in drops] == [3, 4, 5] and drops[1] == (4, 0, 910)
    assert odrop.errlist_to_tbc([], ll, 1, 262, 910) == []


@pytest.mark.parametrize("system", SYSTEMS)
def test_oracle_mask_matches_reference(system):
    g = golden("dropouts_" + system.lower())
    rf = RFParams(system=system)
    rf.delays = {"video_rot": 3}
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"]), snr_db=float(g["snr_db"])).numpy()
    inject_dropouts(cap, int(g["drop_seed"]), int(g["drop_count"]))
    assert hashlib.sha256(cap.tobytes()).hexdigest() == str(g["capture_sha256"])
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    mtf = rf.scaled_mtf(float(g["mtf_level"]))
    f = _field(g, 0)
    nb = f["length"] // U
    v = oracle_capture(rf, cap, f["startloc"] // U, nb, mtf, keys=("demod", "demod_05", "demod_raw"))
    hp = np.concatenate([odemod.demodblock(cap[b * U:b * U + rf.blocklen], rf.Filters, system=system,
                                           freq_hz=rf.freq_hz, video_rot=3, mtf_level=mtf, cut=True)["rfhpf"]
                         for b in range(f["startloc"] // U, f["startloc"] // U + nb)])
    lim = odrop.limits(system, rf.DecoderParams["ire0"], rf.DecoderParams["hz_ire"],
                       rf.SysParams["vsync_ire"])
    iserr, rfstd = odrop.mask(v["demod"], v["demod_05"], v["demod_raw"], hp, f["ll"], f["lineoffset"],
                              f["linecount"], f["isfirst"], f["hsync_len"], system, 3, rf.freq_hz / 2, lim)
    assert rfstd == pytest.approx(f["rfstd"], rel=1e-5)
    got = set(np.nonzero(iserr)[0].tolist())
    want = set(f["errmap"].tolist())
    assert len(got ^ want) <= max(4, len(want) // 200), (len(got ^ want), len(want))
    lines, starts, ends = odrop.detect(iserr, f["ll"], f["lineoffset"], f["linecount"], rf.freq,
                                       rf.SysParams["outlinelen"])
    np.testing.assert_array_equal(np.array([lines, starts, ends], np.int64).reshape(3, -1), f["drops"])
