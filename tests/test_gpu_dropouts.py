"""Dropout detection on the B200 (ldg_dropouts, ldgpu.dropouts) against the
oracle (oracle/dropouts.py, pinned to the reference's golden fields) on the
same inputs: GPU demodulator outputs of captures with seeded dropouts and
the batched line locations.  Every field's dropout list must be identical;
the rfhpf standard deviation equal to 1e-12.  The per-field API
(Field.dropout_detect form, host buffers) gives the same lists, and the
reference's own golden field gives its dropouts."""

import numpy as np
import pytest

from conftest import golden
from ldgpu import lib as L
from ldgpu.fieldread import blocks_in_capture
from ldgpu.synth import inject_dropouts, synth_capture
from oracle import dropouts as odrop

pytestmark = pytest.mark.gpu

NSAMPLES = {"NTSC": 4_000_000, "PAL": 4_800_000}


@pytest.fixture(scope="module", params=["NTSC", "PAL"])
def capture(request, cuda_ok):
    import torch
    from ldgpu import RFDecode
    from ldgpu.lines import LineLocator
    system = request.param
    rf = RFDecode(system=system)
    cap = synth_capture(system, NSAMPLES[system], seed=51, start=999, snr_db=36.0).numpy()
    spans = inject_dropouts(cap, 77, 90)
    nb = blocks_in_capture(rf, len(cap))
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    keys = ["demod", "demod_raw", "demod_05", "demod_burst", "rfhpf"] + (["demod_pilot"] if system == "PAL" else [])
    outs = {k: torch.empty(nb * U, dtype=torch.float32, device="cuda") for k in keys}
    dcap = torch.from_numpy(cap).cuda()
    torch.cuda.synchronize()
    rf.demod_blocks_device(dcap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in outs.items()}, mtf_level=1)
    rf.synchronize()
    loc = LineLocator(rf)
    fields = loc.locate({k: outs[k] for k in ("demod", "demod_05", "demod_burst", "demod_pilot") if k in outs}, nb)
    torch.cuda.synchronize()
    host = {k: v.cpu().numpy() for k, v in outs.items()}
    yield rf, outs, host, fields, spans
    rf.close()


def _oracle(rf, host, fl):
    w = fl.window
    sl = slice(w.startloc, w.startloc + w.length)
    ll = fl.host_linelocs()
    lim = odrop.limits(rf.system, rf.DecoderParams["ire0"], rf.DecoderParams["hz_ire"], rf.SysParams["vsync_ire"])
    iserr, rfstd = odrop.mask(host["demod"][sl], host["demod_05"][sl], host["demod_raw"][sl], host["rfhpf"][sl], ll,
                              fl.lineoffset, fl.linecount, fl.isFirstField, fl.hsync_len, rf.system,
                              int(rf.delays["video_rot"]), rf.freq_hz_half, lim)
    lines, starts, ends = odrop.detect(iserr, ll, fl.lineoffset, fl.linecount, rf.freq, rf.SysParams["outlinelen"])
    return (lines, starts, ends), rfstd, int(iserr.sum())


def test_batch_equals_oracle(capture):
    from ldgpu.dropouts import detect_located
    rf, outs, host, fields, _ = capture
    got, sd = detect_located(rf, fields, outs, rfstd=True)
    assert len(got) == len(fields) >= 4
    total = 0
    for i, fl in enumerate(fields):
        want, rfstd, nerr = _oracle(rf, host, fl)
        assert got[i] == want, i
        assert sd[i] == pytest.approx(rfstd, rel=1e-12)
        total += len(want[0])
    print(rf.system, "fields", len(fields), "dropouts", total)
    assert total >= 20


def test_host_field_api_equals_batch(capture):
    from ldgpu.dropouts import detect_host_field, detect_located
    rf, outs, host, fields, _ = capture
    batch = detect_located(rf, fields, outs, first=1, count=2)
    for j, i in enumerate((1, 2)):
        fl = fields[i]
        w = fl.window
        sl = slice(w.startloc, w.startloc + w.length)
        data = {"video": {k: host[k][sl] for k in ("demod", "demod_05", "demod_raw")}, "rfhpf": host["rfhpf"][sl]}
        one = detect_host_field(rf, data, fl.host_linelocs(), fl.lineoffset, fl.linecount, fl.isFirstField,
                                fl.hsync_len)
        assert one == batch[j]


def test_caps_and_bad_fields_raise(capture):
    import torch
    from ldgpu.dropouts import _field, detect_located, run
    rf, outs, host, fields, _ = capture
    with pytest.raises(L.LdgError, match="error samples"):
        detect_located(rf, fields, outs, err_cap=4)
    with pytest.raises(L.LdgError, match="dropouts"):
        detect_located(rf, fields, outs, out_cap=1)
    # a vertical-sync line beyond the line locations: the reference raises
    # IndexError there; here the call raises
    ll = torch.tensor([100.0, 3000.0, 5600.0, 8200.0, 10800.0], dtype=torch.float64, device="cuda")
    p = [outs[k].data_ptr() for k in ("demod", "demod_05", "demod_raw", "rfhpf")]
    with pytest.raises(L.LdgError, match="vertical-sync"):
        run(rf, [_field(*p, 20000, ll.data_ptr(), 5, 0, 2, 1, 200)])
    torch.cuda.synchronize()


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_reference_golden_fields(cuda_ok, system):
    """The reference's own fields (its line locations and hsync length) on
    the GPU demodulation of the golden capture: the dropout lists match the
    reference's one to one -- same line, each edge within one pixel (the
    GPU's float32 demodulation may move a sample across a limit) -- with no
    dropout missing or extra."""
    import torch
    from ldgpu import RFDecode
    from ldgpu.dropouts import detect_host_field
    g = golden("dropouts_" + system.lower())
    rf = RFDecode(system=system)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"]), snr_db=float(g["snr_db"])).numpy()
    inject_dropouts(cap, int(g["drop_seed"]), int(g["drop_count"]))
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    same = total = 0
    for i in range(int(g["nfields"])):
        p = f"f{i}_"
        startloc, length = int(g[p + "startloc"]), int(g[p + "length"])
        nb = length // U
        raw = torch.from_numpy(np.ascontiguousarray(cap[startloc:startloc + (nb - 1) * U + rf.blocklen])).cuda()
        o = {k: torch.empty(nb * U, dtype=torch.float32, device="cuda")
             for k in ("demod", "demod_05", "demod_raw", "rfhpf")}
        torch.cuda.synchronize()
        rf.demod_blocks_device(raw.data_ptr(), nb, U, {k: v.data_ptr() for k, v in o.items()}, mtf_level=1)
        rf.synchronize()
        data = {"video": {k: o[k].cpu().numpy() for k in ("demod", "demod_05", "demod_raw")},
                "rfhpf": o["rfhpf"].cpu().numpy()}
        isfirst, linecount, lineoffset = (int(x) for x in g[p + "flags"])
        lines, starts, ends = detect_host_field(rf, data, g[p + "linelocs"], lineoffset, linecount, bool(isfirst),
                                                int(g[p + "hsync_len"]))
        want = sorted(map(tuple, g[p + "dropouts"].T.tolist()))
        got = sorted(zip(lines, starts, ends))
        free = list(got)
        unmatched = []
        for w in want:
            m = [x for x in free if x[0] == w[0] and abs(x[1] - w[1]) <= 1 and abs(x[2] - w[2]) <= 1]
            if m:
                best = min(m, key=lambda x: abs(x[1] - w[1]) + abs(x[2] - w[2]))
                free.remove(best)
                same += best == w
            else:
                unmatched.append(w)
        total += len(want)
        assert not unmatched and not free, (system, i, "reference only", unmatched, "GPU only", free)
    print(system, "dropouts", total, "identical", same)
    assert total > 20
    rf.close()
