"""CPU tests of the host side: filter design, sinc table, parameters, block
geometry, the synthetic generator and the C-ABI library's exports."""

import hashlib
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from ldgpu import params
from ldgpu.lut import build_sinc_lut
from ldgpu.rfdecode import RFParams

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


@pytest.mark.parametrize("name", list(CONFIGS))
def test_filter_design_matches_reference(name):
    """Every FP64 filter of RFDecode (core.py:544-737, 422-465) equals the
    reference's, sampled every 61 bins plus whole-array sums."""
    g = golden("filters_" + name)
    rf = RFParams(**CONFIGS[name])
    idx = g["bin_idx"]
    keys = [k[2:] for k in g.files if k.startswith("F_")]
    assert sorted(keys) == sorted(k for k, v in rf.Filters.items() if isinstance(v, np.ndarray))
    for k in keys:
        ref = g["F_" + k]
        mine = rf.Filters[k][idx]
        scale = max(1.0, np.abs(ref).max())
        assert np.abs(mine - ref).max() <= 1e-12 * scale, k
        s = g["Fsum_" + k]
        v = rf.Filters[k]
        assert abs(np.sum(v) - s[0]) <= 1e-9 * max(1.0, abs(s[0])), k
        assert abs(np.sum(np.abs(v) ** 2) - s[1]) <= 1e-9 * max(1.0, s[1]), k
    for k in [k for k in g.files if k.startswith("S_")]:
        assert rf.Filters[k[2:]] == g[k]
    for ch in ("left", "right"):
        a = rf.audio[ch]
        np.testing.assert_allclose([a.lowbin, a.nbins, a.a1_freq, a.low_freq], g[f"A_{ch}_geom"], rtol=0)
        np.testing.assert_allclose(a.filt1, g[f"A_{ch}_filt1"], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(a.audio2_filter[idx], g[f"A_{ch}_audio2"], rtol=1e-10, atol=1e-14)
    assert int(g["blockcut_end"]) == rf.blockcut_end


def test_sinc_lut_bit_exact():
    """The regenerated table equals the reference's shipped sinc_lut.npz."""
    g = golden("sinc_lut_rows")
    lut = build_sinc_lut()
    assert lut.shape == (65537, 16) and lut.dtype == np.float32
    assert np.array_equal(lut[g["rows"]], g["values"])
    assert hashlib.sha256(lut.tobytes()).hexdigest() == str(g["sha256"])


def test_system_tables():
    """Derived system constants (core.py:109-170)."""
    n, p = params.sysparams("NTSC"), params.sysparams("PAL")
    assert n["outlinelen"] == 910 and p["outlinelen"] == 1135 and p["outlinelen_pilot"] == 960
    assert abs(n["line_period"] - 63.5555555) < 1e-6
    assert abs(n["FPS"] - 29.97002997) < 1e-6
    assert RFParams(system="NTSC").linelen == 2542
    assert RFParams(system="PAL").linelen == 2560
    with pytest.raises(ValueError):
        params.sysparams("SECAM")


def test_output_slices_follow_reference_semantics():
    """cut=True keeps [1024, N-32) of video/efm, rfhpf is [1021, N-35),
    audio [32, 1023) (core.py:769-772, 843-875)."""
    rf = RFParams(system="NTSC")
    rf.delays = {"video_rot": 3}
    s = rf.output_slices(True)
    assert s["video"] == (1024, 31712) and s["efm"] == (1024, 31712)
    assert s["rfhpf"] == (1021, 31712) and s["audio"] == (32, 991)
    s = rf.output_slices(False)
    assert s["video"] == (0, 32768) and s["audio"] == (0, 1024)
    rf.blockcut_end = 0
    rf.delays = {"video_rot": 0}
    assert rf.output_slices(True)["rfhpf"][1] == 0  # [1024:0] is empty in the reference too


def test_synth_reproducible():
    """The seeded generator reproduces the golden field captures bit for bit."""
    from ldgpu.synth import synth_capture
    for sysname in ("ntsc", "pal"):
        g = golden("field_" + sysname)
        cap = synth_capture(sysname.upper(), int(g["capture_len"]), seed=int(g["capture_seed"]),
                            start=int(g["capture_start"])).numpy()
        assert hashlib.sha256(cap.tobytes()).hexdigest() == str(g["capture_sha256"]), sysname


def _header_symbols():
    src = open(os.path.join(ROOT, "include", "ldgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ldg_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    """libldgpu.so loads without a GPU and exports every function that
    include/ldgpu.h declares, with a binding in ldgpu.lib."""
    from ldgpu import lib
    h = lib.load()
    syms = _header_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(h, s), s
        assert s in lib.SIGNATURES, s
    assert h.ldg_abi_version() == lib.ABI_VERSION == 3


def test_library_without_gpu_fails_cleanly():
    """On a machine without a GPU the context constructor returns an error
    code (no crash, no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ldgpu import lib
    assert lib.device_count() == 0
    with pytest.raises(lib.LdgError):
        lib.Context("NTSC", 32768, 40e6)
