"""GPU parity of the fused demodulator (RFDecode.demodblock on the B200)
against the CPU oracle and the reference's golden outputs.

Tolerances: the demodulated frequency outputs are FP32 on the GPU against
an FP64 oracle; the bar is <= 1 kHz RMS (the target), checked per output,
with a max-error bound; EFM int16 may differ by one count where the FP64
value sits within FP32 rounding of an integer boundary.
"""

import numpy as np
import pytest

from conftest import golden
from helpers import err_stats, oracle_block, video_keys

pytestmark = pytest.mark.gpu

RMS_HZ = 1000.0   # demod error target (RMS)
MAX_HZ = 20000.0  # single-sample bound (near-zero analytic magnitude spots)


# every test runs under both FFT decompositions of the demodulator
@pytest.fixture(scope="module", params=[("NTSC", 0), ("NTSC", 1), ("PAL", 0), ("PAL", 1)],
                ids=["NTSC-stockham", "NTSC-inplace", "PAL-stockham", "PAL-inplace"])
def rf(request, cuda_ok):
    from ldgpu import RFDecode
    system, variant = request.param
    r = RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=True, fft_variant=variant)
    yield r
    r.close()


def _check_block(rf, block, mtf, cut=True):
    gpu = rf.demodblock(data=block, mtf_level=mtf, cut=cut)
    ref = oracle_block(rf, block, rf.scaled_mtf(mtf), cut=cut)
    stats = {}
    for k in video_keys(rf.system):
        assert gpu["video"][k].shape == ref["video"][k].shape, k
        rms, mx = err_stats(gpu["video"][k], ref["video"][k])
        stats[k] = (rms, mx)
        assert rms <= RMS_HZ and mx <= MAX_HZ, (k, rms, mx)
    rms, mx = err_stats(gpu["rfhpf"], ref["rfhpf"])
    assert rms <= 0.05 and mx <= 1.0, ("rfhpf", rms, mx)
    d = np.abs(gpu["efm"].astype(int) - ref["efm"].astype(int))
    assert d.max() <= 1 and np.mean(d == 0) > 0.999, ("efm", d.max())
    for ch in ("audio_left", "audio_right"):
        rms, mx = err_stats(gpu["audio"][ch], ref["audio"][ch])
        assert rms <= 50 and mx <= 2000, (ch, rms, mx)
    assert gpu["setupcount"] == rf.setupcount
    return stats


def test_demodblock_golden_blocks(rf):
    g = golden("demod_" + rf.system.lower())
    for mtf in (0, 1):
        stats = _check_block(rf, g["block"], mtf)
        print(rf.system, "mtf", mtf, {k: (round(a, 2), round(b, 1)) for k, (a, b) in stats.items()})
    # and directly against the reference's own outputs (subsampled)
    gpu = rf.demodblock(data=g["block"], mtf_level=1, cut=True)
    for k in video_keys(rf.system):
        rms, mx = err_stats(gpu["video"][k][::9], g["m1_" + k])
        assert rms <= RMS_HZ and mx <= MAX_HZ, (k, rms, mx)


def test_demodblock_uncut_and_float_input(rf):
    g = golden("demod_" + rf.system.lower())
    _check_block(rf, g["block"], 1, cut=False)
    gi = rf.demodblock(data=g["block"], mtf_level=1, cut=True)
    gf = rf.demodblock(data=g["block"].astype(np.float64), mtf_level=1, cut=True)
    for k in video_keys(rf.system):
        np.testing.assert_array_equal(gi["video"][k], gf["video"][k])


def test_demodblock_fftdata_only(rf):
    g = golden("demod_" + rf.system.lower())
    x = g["block"]
    a = rf.demodblock(data=x, mtf_level=0, cut=True)
    b = rf.demodblock(fftdata=np.fft.fft(x), mtf_level=0, cut=True)
    # the float32 block from the spectrum's inverse differs from the int16
    # samples by rounding only: a few Hz at most
    for k in video_keys(rf.system):
        rms, mx = err_stats(a["video"][k], b["video"][k])
        assert rms < 10.0, (k, rms)
    # the spectrum takes precedence over the samples (core.py:758-761)
    c = rf.demodblock(data=np.zeros_like(x), mtf_level=0, fftdata=np.fft.fft(x), cut=True)
    np.testing.assert_array_equal(c["video"]["demod"], b["video"]["demod"])
    # and matches the oracle fed the same spectrum
    ref = oracle_block(rf, x, rf.scaled_mtf(0))
    rms, mx = err_stats(b["video"]["demod"], ref["video"]["demod"])
    assert rms <= RMS_HZ and mx <= MAX_HZ
    with pytest.raises(Exception, match="without raw or FFT data"):
        rf.demodblock(mtf_level=0)


def test_random_blocks_and_edge_values(rf):
    """Random seeded blocks, a constant block and a full-scale block."""
    from ldgpu.synth import synth_capture
    cap = synth_capture(rf.system, 5 * 32768, seed=99, snr_db=30).numpy()
    for off in (0, 40000, 97000):
        _check_block(rf, cap[off:off + 32768], 0.5)
    # degenerate inputs must not fault and must match the oracle's finite outputs
    for blk in (np.zeros(32768, np.int16), np.full(32768, 32767, np.int16)):
        gpu = rf.demodblock(data=blk, mtf_level=0, cut=True)
        for k in video_keys(rf.system):
            assert np.all(np.isfinite(gpu["video"][k]))


def test_batched_equals_plain(rf):
    """All blocks of a capture in one device launch == one call per block."""
    import torch
    from ldgpu.synth import synth_capture
    nb = 7
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    cap = synth_capture(rf.system, (nb - 1) * U + rf.blocklen, seed=5).numpy()
    dcap = torch.from_numpy(cap).cuda()
    keys = list(video_keys(rf.system))
    outs = {k: torch.empty(nb * U, dtype=torch.float32, device="cuda") for k in keys}
    outs["rfhpf"] = torch.empty(nb * U, dtype=torch.float32, device="cuda")
    outs["efm"] = torch.empty(nb * U, dtype=torch.int16, device="cuda")
    outs["audio_left"] = torch.empty(nb * 991, dtype=torch.float32, device="cuda")
    outs["audio_right"] = torch.empty(nb * 991, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rf.demod_blocks_device(dcap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in outs.items()},
                           mtf_level=1, cut=True)
    rf.synchronize()
    rf.demod_status()  # no block skipped
    for b in range(nb):
        plain = rf.demodblock(data=cap[b * U:b * U + rf.blocklen], mtf_level=1, cut=True)
        for k in keys:
            np.testing.assert_array_equal(outs[k][b * U:(b + 1) * U].cpu().numpy(), plain["video"][k])
        np.testing.assert_array_equal(outs["rfhpf"][b * U:(b + 1) * U].cpu().numpy(), plain["rfhpf"])
        np.testing.assert_array_equal(outs["efm"][b * U:(b + 1) * U].cpu().numpy(), plain["efm"])
        np.testing.assert_array_equal(outs["audio_left"][b * 991:(b + 1) * 991].cpu().numpy(),
                                      plain["audio"]["audio_left"])


def test_delays_match_reference(rf):
    """computedelays on the GPU reproduces the reference's calibration."""
    g = golden("filters_" + rf.system.lower())
    sync, white, rot = g["delays"]
    assert rf.delays["video_rot"] == int(rot)
    assert abs(rf.delays["video_sync"] - sync) < 0.01
    assert abs(rf.delays["video_white"] - white) < 0.01


@pytest.mark.parametrize("variant", [0, 1], ids=["stockham", "inplace"])
def test_pal_v4300d_notch(cuda_ok, variant):
    """PAL_V4300D_NotchFilter on a block with spurious 8.5 MHz carriers: the
    GPU demodulator against the oracle with the notch and the reference's
    own outputs; the batched device path gives the plain call's bits."""
    import torch
    from ldgpu import RFDecode
    from oracle import demod as odemod
    g = golden("demod_pal_notch")
    rf = RFDecode(system="PAL", decode_analog_audio=44100, decode_digital_audio=True,
                  extra_options={"PAL_V4300D_NotchFilter": True}, fft_variant=variant)
    block = g["block"]
    gpu = rf.demodblock(data=block, mtf_level=1, cut=True)
    ref = odemod.demodblock(block, rf.Filters, system="PAL", freq_hz=rf.freq_hz, blocklen=rf.blocklen,
                            blockcut=rf.blockcut, blockcut_end=rf.blockcut_end, video_rot=rf.delays["video_rot"],
                            mtf_level=rf.scaled_mtf(1), cut=True, efm=True, audio=rf.audio, pal_notch=True)
    for k in video_keys("PAL"):
        rms, mx = err_stats(gpu["video"][k], ref["video"][k])
        assert rms <= RMS_HZ and mx <= MAX_HZ, (k, rms, mx)
        rms, mx = err_stats(gpu["video"][k][::9], g["m1_" + k])
        assert rms <= RMS_HZ and mx <= MAX_HZ, (k, rms, mx)
    d = np.abs(gpu["efm"].astype(int) - ref["efm"].astype(int))
    assert d.max() <= 1 and np.mean(d == 0) > 0.999
    rms, mx = err_stats(gpu["rfhpf"], ref["rfhpf"])
    assert rms <= 0.05 and mx <= 1.0
    # without the notch the outputs are far from the notched reference
    plain = RFDecode(system="PAL", decode_analog_audio=44100, decode_digital_audio=True, fft_variant=variant)
    p = plain.demodblock(data=block, mtf_level=1, cut=True)
    assert np.abs(p["video"]["demod"][::9].astype(np.float64) - g["m1_demod"]).max() > 1000.0
    # device batch form: same bits as the per-block call
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    d_in = torch.from_numpy(np.ascontiguousarray(block)).cuda()
    out = torch.empty(U, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rf.demod_blocks_device(d_in.data_ptr(), 1, U, {"demod": out.data_ptr()}, mtf_level=1)
    rf.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), gpu["video"]["demod"])
    rf.close()
    plain.close()


LOWBAND = {
    "ntsc_lowband": dict(system="NTSC", decode_analog_audio=44100, decode_digital_audio=True,
                         extra_options={"lowband": True, "deemp_str": 1.5, "NTSC_ColorNotchFilter": True,
                                        "MTF_level": 0.7, "MTF_offset": 0.1}),
    "pal_lowband": dict(system="PAL", decode_analog_audio=44100, decode_digital_audio=True,
                        extra_options={"lowband": True, "deemp_coeff": (2.0, 7.0)}),
}


@pytest.mark.parametrize("variant", [0, 1], ids=["stockham", "inplace"])
@pytest.mark.parametrize("name", list(LOWBAND))
def test_lowband_filter_banks(cuda_ok, name, variant):
    """The reference's lowband configurations (core.py:209, 251 filter
    parameters; NTSC colour notch, MTF level/offset and de-emphasis strength;
    PAL de-emphasis coefficients) through the GPU demodulator: every output
    within the demod tolerances of the FP64 oracle with the same filters, on
    the golden block and on a seeded capture block, at both MTF levels."""
    from ldgpu import RFDecode
    from ldgpu.synth import synth_capture
    kw = LOWBAND[name]
    r = RFDecode(**kw, fft_variant=variant)
    try:
        g = golden("demod_" + kw["system"].lower())
        cap = synth_capture(kw["system"], 3 * r.blocklen, seed=77).numpy()
        for block in (g["block"], cap[r.blocklen:2 * r.blocklen]):
            for mtf in (0, 1):
                stats = _check_block(r, block, mtf)
                print(name, "mtf", mtf, {k: (round(a, 2), round(b, 1)) for k, (a, b) in stats.items()})
    finally:
        r.close()


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_variants_agree(cuda_ok, system):
    """The two FFT decompositions on the same seeded blocks: every output
    within float32 rounding of each other (far inside the oracle tolerances),
    and the in-place one within the same oracle tolerances (checked above)."""
    from ldgpu import RFDecode
    from ldgpu.synth import synth_capture
    a = RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=True, fft_variant=0)
    b = RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=True, fft_variant=1)
    try:
        assert (a.fft_variant, b.fft_variant) == (0, 1)
        cap = synth_capture(system, 3 * 32768, seed=4242).numpy()
        for off in (0, 50000):
            x = cap[off:off + 32768]
            ga = a.demodblock(data=x, mtf_level=1, cut=True)
            gb = b.demodblock(data=x, mtf_level=1, cut=True)
            for k in video_keys(system):
                rms, mx = err_stats(ga["video"][k], gb["video"][k])
                assert rms <= 10.0 and mx <= MAX_HZ, (k, rms, mx)
            d = np.abs(ga["efm"].astype(int) - gb["efm"].astype(int))
            assert d.max() <= 1
    finally:
        a.close()
        b.close()
