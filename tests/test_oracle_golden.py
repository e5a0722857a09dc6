"""Pin the CPU oracle (oracle/) against the reference's own outputs.

The golden fixtures were produced by running the unmodified reference on
the same inputs (tests/golden/make_golden.py).  The oracle uses the
product's host filter design, which test_host.py pins separately.
"""

import numpy as np
import pytest

from conftest import golden
from ldgpu.fieldread import field_window
from ldgpu.rfdecode import RFParams
from ldgpu.synth import synth_capture
from oracle import demod as odemod
from oracle import tbc as otbc

STRIDE = 9


def _rf(system, **kw):
    rf = RFParams(system=system, decode_analog_audio=44100, decode_digital_audio=True, **kw)
    rf.delays = {"video_rot": 3}
    return rf


def oracle_block(rf, block, mtf_scaled, cut=True):
    return odemod.demodblock(block, rf.Filters, system=rf.system, freq_hz=rf.freq_hz,
                             blocklen=rf.blocklen, blockcut=rf.blockcut, blockcut_end=rf.blockcut_end,
                             video_rot=rf.delays["video_rot"], mtf_level=mtf_scaled, cut=cut,
                             efm=True, audio=rf.audio)


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_oracle_demod_matches_reference(system):
    g = golden("demod_" + system.lower())
    rf = _rf(system)
    for tag, mtf in (("m0", 0.0), ("m1", rf.scaled_mtf(1))):
        rv = oracle_block(rf, g["block"], mtf)
        names = ["demod", "demod_raw", "demod_05", "demod_burst"] + (["demod_pilot"] if system == "PAL" else [])
        for k in names:
            mine = rv["video"][k][::STRIDE]
            ref = g[f"{tag}_{k}"]
            # both are float32 casts of FP64 results; allow one float32 ulp (~1 Hz)
            assert np.abs(mine.astype(np.float64) - ref).max() <= 2.0, (tag, k)
            assert np.mean(mine == ref) > 0.99, (tag, k)
        np.testing.assert_allclose(rv["rfhpf"][::STRIDE], g[f"{tag}_rfhpf"], rtol=0, atol=1e-3)
        assert np.abs(rv["efm"][::STRIDE].astype(int) - g[f"{tag}_efm"]).max() <= 1
        for ch in ("audio_left", "audio_right"):
            assert np.abs(rv["audio"][ch].astype(np.float64) - g[f"{tag}_{ch}"]).max() <= 1.0
    rv = oracle_block(rf, g["block"], rf.scaled_mtf(1), cut=False)
    for k in ("demod", "demod_05", "demod_burst"):
        assert np.abs(rv["video"][k][::STRIDE].astype(np.float64) - g[f"full_{k}"]).max() <= 2.0
    assert np.abs(rv["efm"][::STRIDE].astype(int) - g["full_efm"]).max() <= 1
    assert len(rv["audio"]["audio_left"]) == 1024


def test_oracle_pal_notch_matches_reference():
    """PAL_V4300D_NotchFilter (core.py:774-798) on a block with spurious
    8.5 MHz carriers: the oracle zeroes the reference's bins and its outputs
    match the reference's; without the notch they do not."""
    g = golden("demod_pal_notch")
    rf = _rf("PAL")
    X = np.fft.fft(g["block"].astype(np.float64))
    Xn = odemod.notch_v4300d(X, rf.blocklen, rf.freq)
    zeroed = np.nonzero((Xn == 0) & (X != 0))[0]
    want = g["notch_bins"]
    np.testing.assert_array_equal(zeroed[zeroed < rf.blocklen // 2], want)
    np.testing.assert_array_equal(zeroed[zeroed >= rf.blocklen // 2], np.sort(rf.blocklen - want))
    rv = odemod.demodblock(g["block"], rf.Filters, system="PAL", freq_hz=rf.freq_hz, blocklen=rf.blocklen,
                           blockcut=rf.blockcut, blockcut_end=rf.blockcut_end, video_rot=3,
                           mtf_level=float(g["mtf_scaled"][0]), cut=True, efm=True, audio=rf.audio, pal_notch=True)
    for k in ("demod", "demod_raw", "demod_05", "demod_burst", "demod_pilot"):
        mine = rv["video"][k][::STRIDE].astype(np.float64)
        assert np.abs(mine - g[f"m1_{k}"]).max() <= 2.0, k
    np.testing.assert_allclose(rv["rfhpf"][::STRIDE], g["m1_rfhpf"], rtol=0, atol=1e-3)
    assert np.abs(rv["efm"][::STRIDE].astype(int) - g["m1_efm"]).max() <= 1
    assert np.abs(rv["audio"]["audio_left"].astype(np.float64) - g["m1_audio_left"]).max() <= 1.0
    assert np.abs(g["m1_demod"].astype(np.float64) - g["plain_demod"]).max() > 1000.0


def field_demod_oracle(rf, cap, window, mtf_scaled, keys=("demod",)):
    """Capture-wide concatenated oracle outputs for one field window."""
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    outs = {k: [] for k in keys}
    for b in range(window.first_block, window.first_block + window.nblocks):
        raw = cap[b * U:b * U + rf.blocklen]
        rv = odemod.demodblock(raw, rf.Filters, system=rf.system, freq_hz=rf.freq_hz,
                               blocklen=rf.blocklen, blockcut=rf.blockcut,
                               blockcut_end=rf.blockcut_end, video_rot=3,
                               mtf_level=mtf_scaled, cut=True)
        for k in keys:
            outs[k].append(rv["video"][k])
    return {k: np.concatenate(v) for k, v in outs.items()}


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_oracle_tbc_matches_reference(system):
    """Oracle coordinates, wow and the uint16 picture (compat mode: the
    reference's float32 coordinate cast) against the reference's fields."""
    g = golden("field_" + system.lower())
    rf = RFParams(system=system)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    lut = rf.downscale_sinc_lut
    outw = rf.SysParams["outlinelen"]
    outlines = rf.SysParams["frame_lines"] // 2 + 1
    for i in range(2):
        p = f"f{i}_"
        w = field_window(rf, float(g[p + "start"]))
        assert w.startloc == int(g[p + "startloc"])
        buf = field_demod_oracle(rf, cap, w, rf.scaled_mtf(float(g["mtf_level"])))["demod"]
        ll = g[p + "linelocs"]
        isfirst, linecount, lineoffset = g[p + "flags"][:3]
        coords, wow = otbc.pixel_coords(ll, rf.linelen, outw, outlines, int(lineoffset))
        np.testing.assert_allclose(coords[::101], g[p + "coords"], rtol=0, atol=1e-8)
        np.testing.assert_allclose(wow[::101], g[p + "wow"], rtol=1e-12)
        assert len(wow) == int(g[p + "wow_stats"][0])
        assert np.median(wow) == g[p + "wow_stats"][1]
        ds = otbc.scale_field(buf, coords, wow, lut, int(lineoffset), outw, outlines * outw,
                              coord_f32=True)
        ire0, hz_ire, vsync_ire, out_scale, ozero = g[p + "levels"]
        pic = otbc.hz_to_output(ds, ire0, hz_ire, ozero, vsync_ire, out_scale)
        ref = g[p + "dspicture"]
        d = np.abs(pic.astype(int) - ref.astype(int))
        assert d.max() <= 1, (i, d.max())
        assert np.mean(d == 0) > 0.99, (i, np.mean(d == 0))


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_oracle_tbc_smoothing_matches_reference(system):
    """wow_level_adjust_smoothing = 2 (the level-adjust IIR, utils.py:141-149):
    the oracle's picture (compat mode) against the reference's."""
    g = golden("tbc_smoothing_" + system.lower())
    rf = RFParams(system=system)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    outw = rf.SysParams["outlinelen"]
    outlines = rf.SysParams["frame_lines"] // 2 + 1
    w = field_window(rf, float(g["start"]))
    assert w.startloc == int(g["startloc"])
    buf = field_demod_oracle(rf, cap, w, rf.scaled_mtf(float(g["mtf_level"])))["demod"]
    lineoffset = int(g["flags"][2])
    coords, wow = otbc.pixel_coords(g["linelocs"], rf.linelen, outw, outlines, lineoffset)
    ire0, hz_ire, vsync_ire, out_scale, ozero = g["levels"]
    ds = otbc.scale_field(buf, coords, wow, rf.downscale_sinc_lut, lineoffset, outw, outlines * outw,
                          coord_f32=True, smoothing=float(g["smoothing"]))
    pic = otbc.hz_to_output(ds, ire0, hz_ire, ozero, vsync_ire, out_scale)
    d = np.abs(pic.astype(int) - g["dspicture"].astype(int))
    assert d.max() <= 1 and np.mean(d == 0) > 0.99, (d.max(), np.mean(d == 0))
    # the smoothing acts: without it the picture differs by more
    ds0 = otbc.scale_field(buf, coords, wow, rf.downscale_sinc_lut, lineoffset, outw, outlines * outw,
                           coord_f32=True)
    pic0 = otbc.hz_to_output(ds0, ire0, hz_ire, ozero, vsync_ire, out_scale)
    assert np.abs(pic0.astype(int) - g["dspicture"].astype(int)).max() > 1


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_oracle_wow_interpolation_matches_reference(system):
    """wow_interpolation_method quadratic / cubic (core.py:2602-2613) on the
    reference's line locations and on line locations with added wow and two
    displaced lines, with and without level smoothing: the oracle's
    coordinates, wow factors, their median / MAD and the picture (compat
    mode, every pic_stride-th sample) against the reference's."""
    g = golden("wow_interp_" + system.lower())
    rf = RFParams(system=system)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    outw = rf.SysParams["outlinelen"]
    outlines = rf.SysParams["frame_lines"] // 2 + 1
    w = field_window(rf, float(g["start"]))
    assert w.startloc == int(g["startloc"])
    buf = field_demod_oracle(rf, cap, w, rf.scaled_mtf(float(g["mtf_level"])))["demod"]
    lineoffset = int(g["flags"][2])
    ire0, hz_ire, vsync_ire, out_scale, ozero = g["levels"]
    stride = int(g["pic_stride"])
    ncase = len([k for k in g.files if k.endswith("_case")])
    assert ncase == 4
    for i in range(ncase):
        p = f"c{i}_"
        method = str(g[p + "case"][0])
        coords, wow = otbc.pixel_coords(g[p + "linelocs"], rf.linelen, outw, outlines, lineoffset, method=method)
        np.testing.assert_allclose(coords[::101], g[p + "coords"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(wow[::101], g[p + "wow"], rtol=1e-13)
        n, med, mad = g[p + "wow_stats"]
        assert len(wow) == int(n) and np.median(wow) == med
        assert np.median(np.abs(wow - med)) == mad
        ds = otbc.scale_field(buf, coords, wow, rf.downscale_sinc_lut, lineoffset, outw, outlines * outw,
                              coord_f32=True, smoothing=float(g[p + "smoothing"]))
        pic = otbc.hz_to_output(ds, ire0, hz_ire, ozero, vsync_ire, out_scale)[::stride]
        d = np.abs(pic.astype(int) - g[p + "picture"].astype(int))
        assert d.max() <= 1 and np.mean(d == 0) > 0.99, (i, d.max(), np.mean(d == 0))
    # the spline forms differ from the linear one (and the displaced lines trip the 15*MAD rule)
    c_lin, w_lin = otbc.pixel_coords(g["c2_linelocs"], rf.linelen, outw, outlines, lineoffset)
    c_cub, w_cub = otbc.pixel_coords(g["c2_linelocs"], rf.linelen, outw, outlines, lineoffset, method="cubic")
    assert np.abs(c_lin - c_cub).max() > 0.05
    med = np.median(w_cub)
    assert np.any(np.abs(w_cub - med) > 15 * np.median(np.abs(w_cub - med)))
