"""RF TBC (Field.rf_tbc, lddecode/core.py:2724-2752): the oracle pinned
bit for bit to the reference's output on the golden fields (SHA-256 of each
field's int16 output, a subsample and two whole lines), and the GPU kernel
(ldg_rf_tbc) bit-identical to both."""

import hashlib

import numpy as np
import pytest

from conftest import golden
from ldgpu.rfdecode import RFParams
from ldgpu.synth import synth_capture
from oracle import rftbc as ortbc

SYSTEMS = ["NTSC", "PAL"]


def _inputs(system):
    g = golden("rftbc_" + system.lower())
    rf = RFParams(system=system)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    assert hashlib.sha256(cap.tobytes()).hexdigest() == str(g["capture_sha256"])
    fields = []
    for i in range(int(g["nfields"])):
        p = f"f{i}_"
        s0, n = int(g[p + "startloc"]), int(g[p + "length"])
        isfirst, linecount, lineoffset = (int(x) for x in g[p + "flags"])
        fields.append(dict(inp=cap[s0 + rf.blockcut:s0 + rf.blockcut + n], ll=g[p + "linelocs"],
                           linecount=linecount, lineoffset=lineoffset, sha=str(g[p + "sha256"]), n=int(g[p + "n"]),
                           sub=g[p + "sub"], lines=g[p + "lines"]))
    return g, rf, fields


def _check(rf, f, out):
    ll = int(round(rf.linelen))
    assert len(out) == f["n"]
    np.testing.assert_array_equal(out[::13], f["sub"])
    np.testing.assert_array_equal(out[20 * ll:21 * ll], f["lines"][0])
    np.testing.assert_array_equal(out[150 * ll:151 * ll], f["lines"][1])
    assert hashlib.sha256(out.astype(np.int16).tobytes()).hexdigest() == f["sha"]


@pytest.mark.parametrize("system", SYSTEMS)
def test_oracle_equals_reference(system):
    g, rf, fields = _inputs(system)
    for f in fields:
        out = ortbc.rf_tbc(f["inp"], f["ll"], float(g["video_white"]), float(g["inlinelen"]), system,
                           f["lineoffset"], f["linecount"])
        _check(rf, f, out)


def test_oracle_scale_edges():
    buf = np.arange(100, dtype=np.float64) * 3.0
    # a straight line is reproduced exactly by the cubic
    np.testing.assert_array_equal(ortbc.scale(buf, 10.0, 20.0, 10), np.arange(10, 20) * 3.0)
    with pytest.raises(IndexError):
        ortbc.scale(buf, 0.5, 10.0, 5)


@pytest.mark.gpu
@pytest.mark.parametrize("system", SYSTEMS)
def test_gpu_equals_reference(cuda_ok, system):
    from ldgpu import RFDecode
    from ldgpu.rftbc import rf_tbc_host_field
    g, _, fields = _inputs(system)
    rf = RFDecode(system=system)
    for f in fields:
        out = rf_tbc_host_field(rf, f["inp"], f["ll"], f["lineoffset"], f["linecount"],
                                delay=float(g["video_white"]))
        _check(rf, f, out)
    # the context's own video delay (computedelays on the GPU) is the reference's to 0.01 sample
    assert abs(rf.delays["video_white"] - float(g["video_white"])) < 0.01
    rf.close()


@pytest.mark.gpu
def test_gpu_batch_equals_oracle(cuda_ok):
    """Every field of a capture in one launch from the batched line
    locations, against the oracle on the same inputs."""
    import torch
    from ldgpu import RFDecode
    from ldgpu.fieldread import blocks_in_capture
    from ldgpu.lines import LineLocator
    from ldgpu.rftbc import rf_tbc_located
    rf = RFDecode(system="NTSC")
    cap = synth_capture("NTSC", 4_500_000, seed=61, start=4321).numpy()
    nb = blocks_in_capture(rf, len(cap))
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    outs = {k: torch.empty(nb * U, dtype=torch.float32, device="cuda") for k in ("demod", "demod_05", "demod_burst")}
    dcap = torch.from_numpy(cap).cuda()
    torch.cuda.synchronize()
    rf.demod_blocks_device(dcap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in outs.items()}, mtf_level=1)
    rf.synchronize()
    fields = LineLocator(rf).locate(outs, nb)
    out, offs = rf_tbc_located(rf, fields, dcap)
    got = out.cpu().numpy()
    a = fields.arrays()
    assert len(fields) >= 4
    for i, fl in enumerate(fields):
        s0 = int(a["startloc"][i]) + rf.blockcut
        want = ortbc.rf_tbc(cap[s0:s0 + int(a["length"][i])], fl.host_linelocs(), rf.delays["video_white"],
                            rf.linelen, "NTSC", fl.lineoffset, fl.linecount)
        np.testing.assert_array_equal(got[offs[i]:offs[i + 1]], want)
    rf.close()
