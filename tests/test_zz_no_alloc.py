"""GPU test of ldg_demod_blocks_noalloc, the allocation-free demod entry point.

That entry point exists for callers that cannot call cudaMalloc while they
decode -- a process whose device memory belongs to another allocator's pool,
or a capture loop that cannot afford cudaMalloc's device-wide
synchronisation -- and keeps the demodulator's scratch in a static device
array instead.  Here it is called through the C ABI twice in a row and must
give the same outputs as the allocating ldg_demod_blocks (same kernel, same
arithmetic: bit-identical), and it must reject sizes beyond its static
scratch and host buffers.  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _args(rf, L, cap_ptr, nb, U, outs, sl):
    a = L.DemodArgs()
    a.in_ = cap_ptr
    a.in_kind = L.LDG_IN_INT16
    a.in_stride = U
    a.nblocks = nb
    a.out_demod = outs["demod"]
    a.out_raw = outs["demod_raw"]
    a.out_05 = outs["demod_05"]
    a.out_burst = outs["demod_burst"]
    a.out_rfhpf = outs["rfhpf"]
    a.out_efm = outs["efm"]
    a.out_audio_left = outs["audio_left"]
    a.out_audio_right = outs["audio_right"]
    a.video = L.Slice(sl["video"][0], sl["video"][1], 0)
    a.roll_05 = int(rf.Filters["F05_offset"])
    a.roll_burst = int(rf.Filters["FVideoBurst_offset"])
    a.rfhpf = L.Slice(sl["rfhpf"][0], sl["rfhpf"][1], 0)
    a.efm = L.Slice(sl["efm"][0], sl["efm"][1], 0)
    a.audio = L.Slice(sl["audio"][0], sl["audio"][1], 0)
    a.stream = None
    return a


def test_noalloc_entry_point_matches_allocating_one(cuda_ok):
    import torch
    from ldgpu import RFDecode
    from ldgpu import lib as L
    from ldgpu.synth import synth_capture

    rf = RFDecode(system="NTSC", decode_analog_audio=44100, decode_digital_audio=True)
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    nb = 40  # more blocks than the 32 static CTA slots: the persistent loop wraps
    cap = torch.from_numpy(synth_capture("NTSC", (nb - 1) * U + rf.blocklen, seed=77).numpy()).cuda()
    sl = rf.output_slices(True)

    def alloc_outs():
        o = {k: torch.full((nb * U,), float("nan"), dtype=torch.float32, device="cuda")
             for k in ("demod", "demod_raw", "demod_05", "demod_burst", "rfhpf")}
        o["efm"] = torch.zeros(nb * U, dtype=torch.int16, device="cuda")
        o["audio_left"] = torch.zeros(nb * 991, dtype=torch.float32, device="cuda")
        o["audio_right"] = torch.zeros(nb * 991, dtype=torch.float32, device="cuda")
        return o

    ref = alloc_outs()
    torch.cuda.synchronize()
    rf.demod_blocks_device(cap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in ref.items()},
                           mtf_level=1, cut=True)
    rf.synchronize()

    lib = L.load()
    for call in range(2):
        out = alloc_outs()
        torch.cuda.synchronize()
        a = _args(rf, L, cap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in out.items()}, sl)
        L.check(lib.ldg_demod_blocks_noalloc(rf._ctx.handle, ctypes.byref(a), 0))
        rf.synchronize()
        for k in ref:
            np.testing.assert_array_equal(out[k].cpu().numpy(), ref[k].cpu().numpy(), err_msg=f"call {call} {k}")

    # sizes beyond the static scratch and host buffers are rejected
    out = alloc_outs()
    a = _args(rf, L, cap.data_ptr(), nb, U, {k: v.data_ptr() for k, v in out.items()}, sl)
    rc = lib.ldg_demod_blocks_noalloc(rf._ctx.handle, ctypes.byref(a), 33)
    assert rc == -1 and b"exceeds the static scratch" in lib.ldg_last_error()
    host = np.zeros(nb * U, dtype=np.float32)
    a.out_demod = host.ctypes.data
    rc = lib.ldg_demod_blocks_noalloc(rf._ctx.handle, ctypes.byref(a), 0)
    assert rc == -1 and b"device memory" in lib.ldg_last_error()
    rf.close()
