"""Analog audio downscale of every located field in one GPU launch
(ldg_audio_downscale) against the host restatement pinned to the reference
(ldgpu.audio.downscale_audio, core.py:1423-1580): int16 samples equal bit
for bit, the same next-field offsets, nothing muted; 44.1 kHz, 48 kHz and
line-locked (4 per line) output, NTSC and PAL."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_audio_downscale_located_equals_host(cuda_ok, system):
    import torch
    from ldgpu import RFDecode
    from ldgpu.audio import av_offset, downscale_audio, downscale_audio_located
    from ldgpu.fieldread import blocks_in_capture
    from ldgpu.lines import LineLocator
    from ldgpu.synth import synth_capture
    rf = RFDecode(system=system, decode_analog_audio=44100, decode_digital_audio=False)
    try:
        n = int(0.6 * rf.freq_hz)
        cap = synth_capture(system, n, seed=12, device="cuda")
        nb = blocks_in_capture(rf, n)
        U = rf.blocklen - rf.blockcut - rf.blockcut_end
        pb = int(round(U / rf.Filters["audio_fdiv"]))
        keys = ["demod", "demod_05", "demod_burst"] + (["demod_pilot"] if system == "PAL" else [])
        outs = {k: torch.empty(nb * U, dtype=torch.float32, device="cuda") for k in keys}
        outs["audio_left"] = torch.empty(nb * pb, dtype=torch.float32, device="cuda")
        outs["audio_right"] = torch.empty(nb * pb, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        rf.demod_blocks_device(cap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in outs.items()}, mtf_level=1)
        rf.synchronize()
        fields = LineLocator(rf).locate({k: outs[k] for k in keys}, nb)
        torch.cuda.synchronize()
        nf = len(fields)
        assert nf >= 20
        al, ar = outs["audio_left"].cpu().numpy(), outs["audio_right"].cpu().numpy()
        a = fields.arrays()
        for freq in (44100, 48000, -4):
            out, offs, muted, nxt = downscale_audio_located(rf, fields, outs["audio_left"], outs["audio_right"],
                                                            freq=freq)
            torch.cuda.synchronize()
            out = out.cpu().numpy()
            assert not muted.cpu().numpy()[:nf].any()
            for i, fl in enumerate(fields):
                w = fl.window
                sl = slice(w.first_block * pb, (w.first_block + w.nblocks) * pb)
                lfw = None if i == 0 else (i, int(a["startloc"][i - 1]))
                off = av_offset(rf, w.startloc, fl.isFirstField, freq, lfw)
                want, wnext = downscale_audio({"audio_left": al[sl], "audio_right": ar[sl]}, fl.host_linelocs(), rf,
                                              fl.linecount, off, freq)
                got = out[offs[i]:offs[i + 1]]
                assert np.array_equal(got, want), (freq, i, np.abs(got.astype(int) - want.astype(int)).max())
                assert nxt[i] == wnext
            print(system, freq, nf, "fields,", offs[-1] // 2, "stereo samples equal")
            # the same fields in two ranges into fixed slots (the batched pipeline's form)
            if freq > 0:
                stride = 2048
                slots = torch.zeros(nf * stride, dtype=torch.int16, device="cuda")
                for lo, hi in ((0, 9), (9, nf)):
                    downscale_audio_located(rf, fields, outs["audio_left"], outs["audio_right"], freq=freq,
                                            first=lo, count=hi - lo, out=slots, stride=stride)
                torch.cuda.synchronize()
                slots = slots.cpu().numpy()
                for i in range(nf):
                    m = offs[i + 1] - offs[i]
                    assert np.array_equal(slots[i * stride:i * stride + m], out[offs[i]:offs[i + 1]])
    finally:
        rf.close()


@pytest.mark.parametrize("dtype", ["float32"])
def test_audio_runs_before_buffer_start(cuda_ok, dtype):
    """A field whose first output samples fall before its audio buffer (a
    negative time offset and a first line near the buffer's start): runs
    with both bounds negative wrap to the buffer's end as the reference's
    slices do, the run across the start is muted (the reference's mean of
    that empty slice raises), and the GPU equals the host restatement."""
    import ctypes

    import torch
    from ldgpu import RFDecode
    from ldgpu import lib as L
    from ldgpu.audio import _AUDIO_DTYPE, downscale_audio, field_clock
    rf = RFDecode(system="NTSC", decode_analog_audio=44100, decode_digital_audio=False)
    try:
        sp = rf.SysParams
        rng = np.random.default_rng(5)
        linecount, alen, freq, toff = 263, 28800, 44100, -1.2e-4
        n = linecount + 12
        wow = 1 + 0.002 * np.sin(np.arange(n) / 37.0)
        lineinfo = 100.5 + np.concatenate([[0], np.cumsum(wow[:-1] * rf.linelen)])
        left = (sp["audio_lfreq"] + rng.integers(-150000, 150000, alen)).astype(dtype)
        right = (sp["audio_rfreq"] + rng.integers(-150000, 150000, alen)).astype(dtype)
        want, _ = downscale_audio({"audio_left": left, "audio_right": right}, lineinfo, rf, linecount, toff, freq)
        off, soundgap, nticks, _ = field_clock(sp["line_period"], linecount, toff, freq)
        dl, dr = torch.from_numpy(left).cuda(), torch.from_numpy(right).cuda()
        dli = torch.from_numpy(lineinfo).cuda()
        out = torch.full((2 * (nticks - 1),), 12345, dtype=torch.int16, device="cuda")
        muted = torch.zeros(1, dtype=torch.int32, device="cuda")
        d = np.zeros(1, _AUDIO_DTYPE)
        d["audio_left"], d["audio_right"], d["audio_len"] = dl.data_ptr(), dr.data_ptr(), alen
        d["linelocs"], d["nlines"], d["nticks"] = dli.data_ptr(), n, nticks
        d["timeoffset"], d["soundgap"], d["out"] = off, soundgap, out.data_ptr()
        p = L.AudioParams(float(sp["line_period"]), float(rf.linelen), float(rf.Filters["audio_fdiv"]),
                          float(sp["audio_lfreq"]), float(sp["audio_rfreq"]))
        descs = (L.AudioField * 1).from_buffer_copy(d.tobytes())
        L.check(rf._ctx._lib.ldg_audio_downscale(rf._ctx.handle, descs, 1, ctypes.byref(p), muted.data_ptr(), 1))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert muted.item() == 1
        assert np.array_equal(got, want)
        assert want[0] != 0  # the first runs (both bounds negative) are not muted
    finally:
        rf.close()
