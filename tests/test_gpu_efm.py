"""Zero crossings of EFM samples on the GPU (ldg_efm_edges, through
ldgpu.efm.efm_edges) against the same test done sample by sample in numpy
(EFM_PLL.process's detector, efm_pll.py:148-151), on the seeded EFM-like
signals of tests/golden/efm_cases.py and the demodulator's own EFM output;
then the PLL run from the GPU crossings equals the PLL run from the
samples."""

import sys

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import efm_crossings

pytestmark = pytest.mark.gpu

if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)
from efm_cases import EFM_CASES, efm_case  # noqa: E402


@pytest.mark.parametrize("name", [c[0] for c in EFM_CASES])
def test_edges_equal_numpy(cuda_ok, name):
    import torch
    from ldgpu.efm import efm_edges
    x, _ = efm_case(name)
    t = torch.from_numpy(np.ascontiguousarray(x, np.int16)).cuda()
    got = efm_edges(t)
    want = efm_crossings(x)
    assert len(got) == len(want) > 100
    assert got.tobytes() == want.tobytes()
    # a view starting at sample 1000, reading the sample before it, positions kept
    got2 = efm_edges(t[1000:], has_before=True, pos_offset=1000)
    want2 = want[want["pos"] >= 1000]
    assert got2.tobytes() == want2.tobytes()


def test_edges_count_beyond_cap_and_empty(cuda_ok):
    import torch
    from ldgpu import lib as L
    x, _ = efm_case(EFM_CASES[0][0])
    t = torch.from_numpy(np.ascontiguousarray(x, np.int16)).cuda()
    lib = L.load()
    n = t.numel()
    scratch = torch.empty(int(lib.ldg_efm_edges_scratch_bytes(n)), dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    cap = 10
    out = torch.zeros(cap * 8, dtype=torch.uint8, device="cuda")
    L.check(lib.ldg_efm_edges(t.data_ptr(), n, 0, 0, out.data_ptr(), cap, count.data_ptr(), scratch.data_ptr(),
                              torch.cuda.current_stream().cuda_stream))
    want = efm_crossings(x)
    assert int(count.item()) == len(want)
    assert out.cpu().numpy().view(L.EFM_EDGE_DTYPE).tobytes() == want[:cap].tobytes()
    L.check(lib.ldg_efm_edges(t.data_ptr(), 0, 0, 0, out.data_ptr(), cap, count.data_ptr(), scratch.data_ptr(),
                              torch.cuda.current_stream().cuda_stream))
    assert int(count.item()) == 0
    with pytest.raises(L.LdgError):
        L.check(lib.ldg_efm_edges(t.data_ptr(), n, 0, 2**31 - 10, out.data_ptr(), cap, count.data_ptr(),
                                  scratch.data_ptr(), 0))


def test_pll_from_gpu_edges_of_demodulated_efm(cuda_ok):
    """The demodulator's EFM output of a seeded capture and its located
    fields: each field's EFM slice (Field.downscale's efmout) found on the
    GPU equals the one from the field's line locations, and the PLL fed the
    fields' slices of the samples and the PLL fed the GPU's crossings give
    the same T-values and state."""
    import torch
    from ldgpu import RFDecode
    from ldgpu.efm import EFM_PLL, efm_edges, field_efm_slices
    from ldgpu.fieldread import blocks_in_capture
    from ldgpu.lines import LineLocator
    from ldgpu.synth import synth_capture
    rf = RFDecode(system="NTSC", decode_digital_audio=True)
    cap = synth_capture("NTSC", 4_000_000, seed=11).numpy()
    nb = blocks_in_capture(rf, len(cap))
    U = rf.blocklen - rf.blockcut - rf.blockcut_end
    outs = {k: torch.empty(nb * U, dtype=torch.float32, device="cuda") for k in ("demod", "demod_05", "demod_burst")}
    efm = torch.empty(nb * U, dtype=torch.int16, device="cuda")
    d = torch.from_numpy(cap).cuda()
    torch.cuda.synchronize()
    rf.demod_blocks_device(d.data_ptr(), nb, U, dict({k: v.data_ptr() for k, v in outs.items()}, efm=efm.data_ptr()),
                           mtf_level=1)
    rf.synchronize()
    fields = LineLocator(rf).locate(outs, nb)
    torch.cuda.synchronize()
    assert len(fields) >= 4
    x = efm.cpu().numpy()
    edges = efm_edges(efm)
    assert edges.tobytes() == efm_crossings(x).tobytes()
    bounds, samples = field_efm_slices(fields, efm)
    bounds, samples = bounds.cpu().numpy(), samples.cpu().numpy()
    # into pinned host memory directly, for a range of the fields
    hb = torch.zeros((3, 2), dtype=torch.int64).pin_memory()
    hs = torch.zeros((3, 2), dtype=torch.int16).pin_memory()
    field_efm_slices(fields, efm, 1, 3, bounds=hb, samples=hs)
    torch.cuda.synchronize()
    assert (hb.numpy() == bounds[1:4]).all() and (hs.numpy() == samples[1:4]).all()
    a, b = EFM_PLL(), EFM_PLL()
    total = 0
    for i, fl in enumerate(fields):
        ll = fl.host_linelocs()
        lo = fl.window.startloc + int(ll[1])
        hi = fl.window.startloc + int(ll[fl.linecount + 1])
        assert (bounds[i] == [lo, hi]).all() and (samples[i] == [x[lo], x[hi - 1]]).all()
        ta = a.process(x[lo:hi])
        tb = b.process_edges(edges, lo, hi, samples[i, 0], samples[i, 1])
        np.testing.assert_array_equal(tb, ta)
        total += len(ta)
    assert total > 1000 and a.state() == b.state()
    rf.close()
