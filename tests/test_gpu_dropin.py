"""The drop-in classes (ldgpu.FieldNTSC / FieldPAL, as LDdecode.readfield
uses them) on the GPU: Field.process() runs the GPU line path on each
field's read and Field.downscale() the GPU TBC and analog audio.  Over the
seeded captures of tests/golden/fields_<case>.npz, field after field with
the reference's read offsets, the results equal the batched LineLocator's
(the same kernels over the capture-wide arrays; line locations to 1e-9
samples) and the reference's integers."""

import sys

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)
from field_cases import field_case, field_case_capture  # noqa: E402


@pytest.mark.parametrize("name", ["ntsc_dropouts", "pal_8phase"])
def test_dropin_fields_equal_batched_and_reference(cuda_ok, name):
    import torch
    from ldgpu import RFDecode
    from ldgpu.audio import downscale_audio_located
    from ldgpu.field import FieldNTSC, FieldPAL
    from ldgpu.fieldread import blocks_in_capture, readlen_for
    from ldgpu.lines import LineLocator
    case = field_case(name)
    system = case[1]
    g = golden("fields_" + name)
    rf = RFDecode(system=system, decode_analog_audio=44100)
    try:
        cap, _ = field_case_capture(case, rf.blocklen, readlen_for(rf))
        nb = blocks_in_capture(rf, len(cap))
        U = rf.blocklen - rf.blockcut - rf.blockcut_end
        pb = int(round(U / rf.Filters["audio_fdiv"]))
        keys = ["demod", "demod_05", "demod_burst"] + (["demod_pilot"] if system == "PAL" else [])
        dcap = torch.from_numpy(cap).cuda()
        outs = {k: torch.empty(nb * U, dtype=torch.float32, device="cuda") for k in keys}
        outs["audio_left"] = torch.empty(nb * pb, dtype=torch.float32, device="cuda")
        outs["audio_right"] = torch.empty(nb * pb, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        rf.demod_blocks_device(dcap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in outs.items()}, mtf_level=1)
        rf.synchronize()
        batched = LineLocator(rf).locate({k: outs[k] for k in keys}, nb)
        aud, offs, _, _ = downscale_audio_located(rf, batched, outs["audio_left"], outs["audio_right"], freq=44100)
        torch.cuda.synchronize()
        aud = aud.cpu().numpy()
        host = {k: v.cpu().numpy() for k, v in outs.items()}
        cls = FieldPAL if system == "PAL" else FieldNTSC
        n = int(g["nfields"])
        prev, prev_startloc = None, None
        for i in range(n):
            fl = batched[i]
            w = fl.window
            sl = slice(w.startloc, w.startloc + w.length)
            asl = slice(w.first_block * pb, (w.first_block + w.nblocks) * pb)
            video = np.rec.fromarrays([host[k][sl] for k in keys], names=keys)
            audio = np.rec.fromarrays([host["audio_left"][asl], host["audio_right"][asl]],
                                      names=["audio_left", "audio_right"])
            f = cls(rf, {"video": video, "audio": audio, "startloc": w.startloc}, prevfield=prev,
                    initphase=(i == 0), fields_written=i, readloc=w.startloc)
            f.process()
            assert f.valid
            p = f"f{i}_"
            flags = [int(f.isFirstField), f.linecount, f.lineoffset, f.fieldPhaseID]
            np.testing.assert_array_equal(flags, g[p + "flags"][:4], err_msg=f"{name} field {i}")
            assert flags == [int(fl.isFirstField), fl.linecount, fl.lineoffset, fl.fieldPhaseID]
            # the batched path takes NTSC burst phases from parallel rounds
            # seeded with values equal to the field-by-field ones to the
            # last bits, so its line locations agree to ~1e-11 samples
            np.testing.assert_allclose(np.asarray(f.linelocs), fl.host_linelocs(), rtol=0, atol=1e-9)
            np.testing.assert_array_equal(np.asarray(f.linebad, dtype=bool), fl.linebad)
            assert f.sync_confidence == fl.sync_confidence
            lfw = None if i == 0 else (i, prev_startloc)
            pic, dsaudio, _ = f.downscale(linesout=f.outlinecount, final=True, audio=44100, lastfieldwritten=lfw)
            np.testing.assert_array_equal(dsaudio, aud[offs[i]:offs[i + 1]])
            prev, prev_startloc = f, w.startloc
            print(name, i, "ok", f.fieldPhaseID)
    finally:
        rf.close()
