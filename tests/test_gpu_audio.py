"""Analog audio end to end on the B200: GPU stage-1 audio of a field's blocks
(ldg_demod_blocks), host stage 2 (RFDecode.audio_phase2) and the 44.1 kHz
downscale through Field.downscale(audio=44100), against the same chain fed
by the FP64 oracle's stage-1 audio."""

import numpy as np
import pytest

from conftest import golden
from oracle import demod as odemod

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("system", ["NTSC", "PAL"])
def test_field_analog_audio(system, cuda_ok):
    import torch
    from ldgpu import RFDecode
    from ldgpu.audio import downscale_audio
    from ldgpu.field import FieldNTSC, FieldPAL
    from ldgpu.fieldread import field_window
    from ldgpu.synth import synth_capture

    g = golden("field_" + system.lower())
    rf = RFDecode(system=system, decode_analog_audio=44100)
    cap = synth_capture(system, int(g["capture_len"]), seed=int(g["capture_seed"]),
                        start=int(g["capture_start"])).numpy()
    w = field_window(rf, float(g["f0_start"]))
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    na = rf.blocklen // rf.Filters["audio_fdiv"] - (rf.blockcut + rf.blockcut_end) // rf.Filters["audio_fdiv"]
    mtf = float(g["mtf_level"])

    dcap = torch.from_numpy(cap).cuda()
    al = torch.empty(w.nblocks * na, dtype=torch.float32, device="cuda")
    ar = torch.empty(w.nblocks * na, dtype=torch.float32, device="cuda")
    rf.demod_blocks_device(dcap.data_ptr() + 2 * w.first_block * U, w.nblocks, U,
                           {"audio_left": al.data_ptr(), "audio_right": ar.data_ptr()}, mtf_level=mtf)
    rf.synchronize()
    gpu1 = np.rec.array([al.cpu().numpy(), ar.cpu().numpy()], names=["audio_left", "audio_right"])

    ol, orr = [], []
    for b in range(w.first_block, w.first_block + w.nblocks):
        rv = odemod.demodblock(cap[b * U:b * U + rf.blocklen], rf.Filters, system=system, freq_hz=rf.freq_hz,
                               blocklen=rf.blocklen, blockcut=rf.blockcut, blockcut_end=rf.blockcut_end,
                               video_rot=rf.delays["video_rot"], mtf_level=rf.scaled_mtf(mtf), audio=rf.audio)
        ol.append(rv["audio"]["audio_left"])
        orr.append(rv["audio"]["audio_right"])
    ora1 = np.rec.array([np.concatenate(ol), np.concatenate(orr)], names=["audio_left", "audio_right"])
    for ch in ("audio_left", "audio_right"):
        d = gpu1[ch].astype(np.float64) - ora1[ch]
        print(system, ch, "stage-1 rms Hz", float(np.sqrt(np.mean(d * d))))

    a2 = rf.audio_phase2(gpu1)
    a2o = rf.audio_phase2(ora1)
    cls = FieldPAL if system == "PAL" else FieldNTSC
    isfirst, linecount, lineoffset = (int(v) for v in g["f0_flags"][:3])
    f = cls(rf, {"video": {"demod": np.zeros(1, np.float32)}, "audio": a2, "startloc": int(g["f0_startloc"])})
    f.linelocs = g["f0_linelocs"]
    f.linecount = linecount
    f.lineoffset = lineoffset
    f.isFirstField = bool(isfirst)
    f.data["video"]["demod"] = np.zeros(int(f.linelocs[-1]) + 4096, np.float32)
    _, dsaudio, _ = f.downscale(linesout=f.outlinecount, final=True, audio=44100)
    want, nxt = downscale_audio(a2o, g["f0_linelocs"], rf, linecount, 0, 44100)
    assert dsaudio.dtype == np.int16 and dsaudio.shape == want.shape
    assert f.audio_next_offset == nxt
    d = np.abs(dsaudio.astype(int) - want.astype(int))
    print(system, "44.1 kHz audio vs oracle chain: max LSB", d.max(), "exact", np.mean(d == 0))
    assert np.sqrt(np.mean(d * d)) <= 2.0 and d.max() <= 16
    rf.close()
