"""GPU parity of the time-base corrector (Field.downscale on the B200).

Line locations come from the reference's golden fields; the demodulated
field buffer is the oracle's (FP64) or the GPU's own.  Bars:
  * compat mode (float32 coordinates, as the reference) vs the reference's
    picture: within 1 LSB, >= 99 % exact;
  * FP64 mode vs the FP64 oracle on the same buffer: within 1 LSB on
    >= 99.99 % of samples;
  * GPU demod + GPU TBC vs the FP64 oracle end to end: within 1 LSB on
    >= 99.99 % of samples.
"""

import numpy as np
import pytest

from conftest import golden
from helpers import oracle_capture
from oracle import tbc as otbc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["NTSC", "PAL"])
def case(request, cuda_ok):
    from ldgpu import RFDecode
    from ldgpu.fieldread import field_window
    from ldgpu.synth import synth_capture
    system = request.param
    g = golden("field_" + system.lower())
    rf = RFDecode(system=system)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    w = field_window(rf, float(g["f0_start"]))
    mtf = rf.scaled_mtf(float(g["mtf_level"]))
    buf = oracle_capture(rf, cap, w.first_block, w.nblocks, mtf)["demod"]
    yield rf, g, cap, w, buf
    rf.close()


def _field(rf, g, buf, coord_f32):
    from ldgpu.field import FieldNTSC, FieldPAL
    cls = FieldPAL if rf.system == "PAL" else FieldNTSC
    isfirst, linecount, lineoffset = (int(v) for v in g["f0_flags"][:3])
    f = cls(rf, {"video": {"demod": buf}, "startloc": int(g["f0_startloc"])})
    f.linelocs = g["f0_linelocs"]
    f.lineoffset = lineoffset
    f.linecount = linecount
    f.isFirstField = bool(isfirst)
    f.coord_f32 = coord_f32
    ire0, hz_ire, vsync_ire, out_scale, ozero = g["f0_levels"]
    f.out_scale = out_scale
    return f


def _oracle_picture(rf, g, buf, coord_f32):
    outw = rf.SysParams["outlinelen"]
    outlines = rf.SysParams["frame_lines"] // 2 + 1
    lineoffset = int(g["f0_flags"][2])
    coords, wow = otbc.pixel_coords(g["f0_linelocs"], rf.linelen, outw, outlines, lineoffset)
    ds = otbc.scale_field(buf, coords, wow, rf.downscale_sinc_lut, lineoffset, outw, outlines * outw,
                          coord_f32=coord_f32)
    ire0, hz_ire, vsync_ire, out_scale, ozero = g["f0_levels"]
    return ds, otbc.hz_to_output(ds, ire0, hz_ire, ozero, vsync_ire, out_scale)


def test_tbc_compat_matches_reference_picture(case):
    rf, g, cap, w, buf = case
    f = _field(rf, g, buf, coord_f32=True)
    pic, _, _ = f.downscale(linesout=f.outlinecount, final=True)
    d = np.abs(pic.astype(int) - g["f0_dspicture"].astype(int))
    print(rf.system, "compat vs reference: max", d.max(), "exact", np.mean(d == 0))
    assert d.max() <= 1 and np.mean(d == 0) >= 0.99


def test_tbc_fp64_matches_oracle(case):
    rf, g, cap, w, buf = case
    f = _field(rf, g, buf, coord_f32=False)
    ds, _, _ = f.downscale(linesout=f.outlinecount, final=False)
    pic, _, _ = f.downscale(linesout=f.outlinecount, final=True)
    ods, opic = _oracle_picture(rf, g, buf, coord_f32=False)
    assert np.abs(ds.astype(np.float64) - ods).max() < 2.0  # Hz
    d = np.abs(pic.astype(int) - opic.astype(int))
    print(rf.system, "fp64 vs oracle: max", d.max(), "within1", np.mean(d <= 1))
    assert d.max() <= 1 and np.mean(d <= 1) >= 0.9999


def test_tbc_wide_first_taps(case):
    """A field whose line 100 spans 2.4 M samples: 32 consecutive pixels of
    that line start their taps more than 65535 samples apart, which the
    gather handles by its separate path (first taps and phases shuffled one
    by one); the picture still equals the FP64 oracle's."""
    rf, g, cap, w, buf = case
    stretch = 2_400_000
    long_buf = np.concatenate([buf, np.tile(buf, stretch // len(buf) + 2)]).astype(np.float32)
    ll = np.array(g["f0_linelocs"], dtype=np.float64)
    ll[101:] += stretch
    g2 = dict(g)
    g2["f0_linelocs"] = ll
    f = _field(rf, g2, long_buf, coord_f32=False)
    pic, _, _ = f.downscale(linesout=f.outlinecount, final=True)
    _, opic = _oracle_picture(rf, g2, long_buf, coord_f32=False)
    d = np.abs(pic.astype(int) - opic.astype(int))
    print(rf.system, "wide first taps vs oracle: max", d.max(), "within1", np.mean(d <= 1))
    assert d.max() <= 1 and np.mean(d <= 1) >= 0.9999


def test_demod_plus_tbc_end_to_end(case):
    """GPU demod of the field's blocks, then GPU TBC, vs the FP64 oracle."""
    import torch
    rf, g, cap, w, buf = case
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    dcap = torch.from_numpy(cap).cuda()
    dem = torch.empty(w.nblocks * U, dtype=torch.float32, device="cuda")
    rf.demod_blocks_device(dcap.data_ptr() + 2 * w.first_block * U, w.nblocks, U,
                           {"demod": dem.data_ptr()}, mtf_level=float(g["mtf_level"]))
    rf.synchronize()
    gbuf = dem.cpu().numpy()
    rms = float(np.sqrt(np.mean((gbuf.astype(np.float64) - buf) ** 2)))
    print(rf.system, "field demod rms Hz", rms)
    assert rms < 1000.0
    f = _field(rf, g, gbuf, coord_f32=False)
    pic, _, _ = f.downscale(linesout=f.outlinecount, final=True)
    _, opic = _oracle_picture(rf, g, buf, coord_f32=False)
    d = np.abs(pic.astype(int) - opic.astype(int))
    print(rf.system, "e2e vs oracle: max", d.max(), "within1", np.mean(d <= 1), "exact", np.mean(d == 0))
    assert np.mean(d <= 1) >= 0.9999


def test_tbc_batched_fields(case):
    """Several fields in one launch give the same pictures as one by one."""
    from ldgpu.field import tbc_descriptor, tbc_fields
    rf, g, cap, w, buf = case
    f = _field(rf, g, buf, coord_f32=False)
    single, _, _ = f.downscale(linesout=f.outlinecount, final=True)
    outs = []
    descs = []
    for shift in (0.0, 0.25, -0.5):
        ll = np.ascontiguousarray(g["f0_linelocs"] + shift)
        o = np.empty(f.outlinecount * f.outlinelen, dtype=np.uint16)
        outs.append((ll, o))
        descs.append(tbc_descriptor(rf, buf, ll, f.lineoffset, f.outlinelen, f.outlinecount,
                                    f.outlinecount, f.levels(), out_u16=o))
    tbc_fields(rf, descs)
    np.testing.assert_array_equal(outs[0][1], single)
    assert not np.array_equal(outs[1][1], single)


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_tbc_level_smoothing(cuda_ok, system):
    """wow_level_adjust_smoothing = 2: the GPU picture against the
    reference's (compat mode) and against the FP64 oracle with the same IIR
    (FP64 coordinates)."""
    from ldgpu import RFDecode
    from ldgpu.field import FieldNTSC, FieldPAL
    from ldgpu.fieldread import field_window
    from ldgpu.synth import synth_capture
    g = golden("tbc_smoothing_" + system.lower())
    rf = RFDecode(system=system)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    w = field_window(rf, float(g["start"]))
    buf = oracle_capture(rf, cap, w.first_block, w.nblocks, rf.scaled_mtf(float(g["mtf_level"])))["demod"]
    isfirst, linecount, lineoffset = (int(v) for v in g["flags"])
    ire0, hz_ire, vsync_ire, out_scale, ozero = g["levels"]
    smoothing = float(g["smoothing"])
    cls = FieldPAL if system == "PAL" else FieldNTSC
    outw = rf.SysParams["outlinelen"]
    outlines = rf.SysParams["frame_lines"] // 2 + 1
    coords, wow = otbc.pixel_coords(g["linelocs"], rf.linelen, outw, outlines, lineoffset)
    for coord_f32 in (True, False):
        f = cls(rf, {"video": {"demod": buf}, "startloc": int(g["startloc"])}, wow_level_adjust_smoothing=smoothing)
        f.linelocs = g["linelocs"]
        f.lineoffset, f.linecount, f.isFirstField = lineoffset, linecount, bool(isfirst)
        f.coord_f32 = coord_f32
        f.out_scale = out_scale
        pic, _, _ = f.downscale(linesout=f.outlinecount, final=True)
        if coord_f32:
            d = np.abs(pic.astype(int) - g["dspicture"].astype(int))
            print(system, "smoothing, compat vs reference: max", d.max(), "exact", np.mean(d == 0))
            assert d.max() <= 1 and np.mean(d == 0) >= 0.99
        else:
            ds = otbc.scale_field(buf, coords, wow, rf.downscale_sinc_lut, lineoffset, outw, outlines * outw,
                                  smoothing=smoothing)
            opic = otbc.hz_to_output(ds, ire0, hz_ire, ozero, vsync_ire, out_scale)
            d = np.abs(pic.astype(int) - opic.astype(int))
            print(system, "smoothing, fp64 vs oracle: max", d.max(), "within 1", np.mean(d <= 1))
            assert np.mean(d <= 1) >= 0.9999 and d.max() <= 2
    rf.close()


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_tbc_wow_interpolation(cuda_ok, system):
    """wow_interpolation_method quadratic / cubic (core.py:2602-2613), with
    and without level smoothing, on the reference's line locations and on
    line locations with added wow and two displaced lines: the GPU picture
    against the reference's (compat mode, every pic_stride-th sample) and
    against the FP64 oracle with the same spline (FP64 coordinates); a batch
    mixing spline and linear fields through the asynchronous entry point
    gives each field's single-call picture."""
    import torch
    from ldgpu import RFDecode
    from ldgpu.field import FieldNTSC, FieldPAL, tbc_descriptor, tbc_fields, tbc_status
    from ldgpu.fieldread import field_window
    from ldgpu.synth import synth_capture
    g = golden("wow_interp_" + system.lower())
    rf = RFDecode(system=system)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    w = field_window(rf, float(g["start"]))
    buf = oracle_capture(rf, cap, w.first_block, w.nblocks, rf.scaled_mtf(float(g["mtf_level"])))["demod"]
    isfirst, linecount, lineoffset = (int(v) for v in g["flags"])
    levels = g["levels"]
    ire0, hz_ire, vsync_ire, out_scale, ozero = levels
    stride = int(g["pic_stride"])
    cls = FieldPAL if system == "PAL" else FieldNTSC
    outw = rf.SysParams["outlinelen"]
    outlines = rf.SysParams["frame_lines"] // 2 + 1
    singles = {}
    for i in range(4):
        p = f"c{i}_"
        method, smoothing = str(g[p + "case"][0]), float(g[p + "smoothing"])
        ll = g[p + "linelocs"]
        coords, wow = otbc.pixel_coords(ll, rf.linelen, outw, outlines, lineoffset, method=method)
        for coord_f32 in (True, False):
            f = cls(rf, {"video": {"demod": buf}, "startloc": int(g["startloc"])},
                    wow_level_adjust_smoothing=smoothing, wow_interpolation_method=method)
            f.linelocs = ll
            f.lineoffset, f.linecount, f.isFirstField = lineoffset, linecount, bool(isfirst)
            f.coord_f32 = coord_f32
            f.out_scale = out_scale
            pic, _, _ = f.downscale(linesout=f.outlinecount, final=True)
            if coord_f32:
                d = np.abs(pic[::stride].astype(int) - g[p + "picture"].astype(int))
                print(system, method, smoothing, "compat vs reference: max", d.max(), "exact", np.mean(d == 0))
                assert d.max() <= 1 and np.mean(d == 0) >= 0.99
            else:
                singles[i] = pic
                ds = otbc.scale_field(buf, coords, wow, rf.downscale_sinc_lut, lineoffset, outw, outlines * outw,
                                      smoothing=smoothing)
                opic = otbc.hz_to_output(ds, ire0, hz_ire, ozero, vsync_ire, out_scale)
                d = np.abs(pic.astype(int) - opic.astype(int))
                print(system, method, smoothing, "fp64 vs oracle: max", d.max(), "within 1", np.mean(d <= 1))
                assert np.mean(d <= 1) >= 0.9999 and d.max() <= 2
    # one asynchronous batch: the four spline cases and a linear field
    nout = outlines * outw
    dbuf = torch.from_numpy(np.ascontiguousarray(buf, np.float32)).cuda()
    dll = [torch.from_numpy(np.ascontiguousarray(g[f"c{i}_linelocs"])).cuda() for i in range(4)]
    dll.append(dll[2])
    meths = [str(g[f"c{i}_case"][0]) for i in range(4)] + ["linear"]
    smooth = [float(g[f"c{i}_smoothing"]) for i in range(4)] + [2.0]
    out = torch.zeros(5 * nout, dtype=torch.int16, device="cuda")
    descs = [tbc_descriptor(rf, dbuf.data_ptr(), dll[k].data_ptr(), lineoffset, outw, outlines, outlines,
                            levels, out_u16=out.data_ptr() + 2 * k * nout, buf_len=len(buf), nlines=len(dll[k]),
                            wow_smoothing=smooth[k], wow_interpolation_method=meths[k]) for k in range(5)]
    torch.cuda.synchronize()
    tbc_fields(rf, descs, asynchronous=True)
    torch.cuda.synchronize()
    tbc_status(rf)
    got = out.cpu().numpy().view(np.uint16).reshape(5, nout)
    for k in range(4):
        assert np.array_equal(got[k], singles[k]), k
    f = cls(rf, {"video": {"demod": buf}, "startloc": int(g["startloc"])}, wow_level_adjust_smoothing=2.0)
    f.linelocs = g["c2_linelocs"]
    f.lineoffset, f.linecount, f.isFirstField = lineoffset, linecount, bool(isfirst)
    f.out_scale = out_scale
    lin, _, _ = f.downscale(linesout=f.outlinecount, final=True)
    assert np.array_equal(got[4], lin)
    assert not np.array_equal(lin, singles[3])
    rf.close()


def test_tbc_argument_checks(cuda_ok):
    """ldg_tbc_fields rejects, before any launch: an unknown wow_interp, a
    quadratic / cubic field with fewer than 4 line locations, and a field
    buffer of 2^31 samples or more."""
    from ldgpu import RFDecode
    from ldgpu import lib as L
    from ldgpu.field import tbc_descriptor, tbc_fields
    rf = RFDecode(system="NTSC")
    try:
        outw = rf.SysParams["outlinelen"]
        buf = np.zeros(200000, np.float32)
        ll = np.arange(60, dtype=np.float64) * rf.linelen + 100.0
        pic = np.zeros(20 * outw, np.uint16)
        levels = (8.1e6, 12142.86, -40.0, 1.0, 1024.0)

        def desc(lls, **kw):
            return tbc_descriptor(rf, buf, lls, 0, outw, 20, 20, levels, out_u16=pic, **kw)

        tbc_fields(rf, [desc(ll, wow_interpolation_method="cubic")])  # valid
        d = desc(ll)
        d.wow_interp = 7
        with pytest.raises(L.LdgError) as e:
            tbc_fields(rf, [d])
        assert e.value.code == L.LDG_ERR_ARG
        with pytest.raises(L.LdgError) as e:
            tbc_fields(rf, [desc(ll[:3], wow_interpolation_method="quadratic")])
        assert e.value.code == L.LDG_ERR_ARG
        d = desc(ll)
        d.buf_len = 1 << 31
        with pytest.raises(L.LdgError) as e:
            tbc_fields(rf, [d])
        assert e.value.code == L.LDG_ERR_ARG
        with pytest.raises(ValueError):
            desc(ll, wow_interpolation_method="spline")
    finally:
        rf.close()
