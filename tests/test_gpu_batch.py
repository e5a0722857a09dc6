"""Mixed batches on the B200: captures of uneven length, NTSC and PAL
together, demodulated in one persistent launch from the device work queue
(ldg_queue_*, replayed from a CUDA graph) and resampled in one TBC launch.

Every output of the queue is bit-identical to demodulating each capture
alone with ldg_demod_blocks (same per-block arithmetic), under every
schedule the autotuner tries, with and without the graph; the fields and
pictures of the whole mixed path equal those of each capture run alone."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (system, seconds, seed, SNR dB): uneven lengths, both systems, one capture
# shorter than two blocks and one with a single block
CAPTURES = [("NTSC", 0.40, 101, 35.0), ("PAL", 0.31, 102, 42.0), ("NTSC", 0.93, 103, 31.0),
            ("PAL", 1.07, 104, 44.0), ("NTSC", 0.0009, 105, 38.0), ("PAL", 0.0015, 106, 30.0),
            ("PAL", 0.55, 107, 36.0), ("NTSC", 0.21, 108, 40.0)]


@pytest.fixture(scope="module")
def batch(cuda_ok):
    import torch
    from ldgpu.batch import MixedBatch
    from ldgpu.synth import synth_capture
    caps = []
    for system, secs, seed, snr in CAPTURES:
        n = max(int(secs * 40e6), 32768 + 2000) if secs < 0.001 else int(secs * 40e6)
        caps.append((system, synth_capture(system, n, seed=seed, snr_db=snr, start=seed * 1000, device="cuda")))
    mb = MixedBatch(caps, locate_threads=3)
    yield mb
    mb.close()


def _alone(mb, i):
    """Capture i demodulated alone with ldg_demod_blocks (fresh outputs)."""
    import torch
    rf, in_ptr, nb, U, outs, level = mb.items[i]
    ref = {k: torch.empty_like(v) for k, v in mb.outs[i].items()}
    rf.demod_blocks_device(in_ptr, nb, U, {k: v.data_ptr() for k, v in ref.items()}, mtf_level=level)
    torch.cuda.synchronize()
    return ref


def _same(mb, refs):
    import torch
    torch.cuda.synchronize()
    for i, ref in enumerate(refs):
        for k, v in ref.items():
            assert torch.equal(mb.outs[i][k].view(torch.int32 if v.dtype == torch.float32 else torch.int16),
                               v.view(torch.int32 if v.dtype == torch.float32 else torch.int16)), (i, k)


def test_queue_equals_captures_alone(batch):
    import torch
    mb = batch
    total, grid = mb.queue.info()
    assert total == sum(mb.nblocks) and 0 < grid <= torch.cuda.get_device_properties(0).multi_processor_count
    assert mb.nblocks[4] == 1 and mb.nblocks[5] == 1
    refs = [_alone(mb, i) for i in range(len(CAPTURES))]
    for o in mb.outs:
        for v in o.values():
            v.fill_(7)
    torch.cuda.synchronize()
    mb.demod(graph=True)
    _same(mb, refs)
    # other schedules, graph replays and plain launches give the same bits
    for grab, ctas, graph in [(4, 37, True), (1, 0, False), (8, 0, True), (2, 300, False)]:
        for o in mb.outs:
            for v in o.values():
                v.fill_(3)
        torch.cuda.synchronize()
        mb.queue.set_schedule(grab, ctas)
        mb.demod(graph=graph)
        mb.demod(graph=graph)  # second replay of the same graph
        _same(mb, refs)
    mb.queue.set_schedule(1, 0)


def test_autotune_keeps_results(batch):
    import torch
    from ldgpu.batch import autotune
    mb = batch
    refs = [_alone(mb, i) for i in range(len(CAPTURES))]
    for o in mb.outs:
        for v in o.values():
            v.fill_(5)
    torch.cuda.synchronize()
    res = autotune(mb.queue, mb.stream, grabs=(1, 2, 4), ctas=(0, 74), reps=1)
    assert res["best"] in res["ms"] and len(res["ms"]) == 6
    assert all(v > 0 for v in res["ms"].values())
    assert mb.queue.schedule == res["best"][:2]
    mb.demod()
    _same(mb, refs)
    torch.cuda.synchronize()


def test_mixed_path_equals_captures_alone(batch):
    import torch
    from ldgpu.field import tbc_fields, tbc_status
    from ldgpu.lines import LineLocator, field_levels, tbc_batch
    mb = batch
    torch.cuda.synchronize()
    n = mb.run()
    torch.cuda.synchronize()
    tbc_status(mb.rfs["NTSC"])
    counts = [len(f) for f in mb.fields]
    assert n == sum(counts)
    # whole captures of 0.2 s or more hold fields; one-block captures none
    for (system, secs, _, _), c in zip(CAPTURES, counts):
        rate = 59.94 if system == "NTSC" else 50.0
        if secs >= 0.2:
            assert c >= int(secs * rate) - 4, (system, secs, c)
        else:
            assert c == 0
    # each capture alone: its own locator and its own TBC launch
    for i, (system, _) in enumerate(mb.captures):
        if counts[i] == 0:
            continue
        rf = mb.rfs[system]
        o = mb.outs[i]
        loc = LineLocator(rf)
        fl = loc.locate({k: o[k] for k in ("demod", "demod_05", "demod_burst", "demod_pilot") if k in o},
                        mb.nblocks[i])
        assert len(fl) == counts[i]
        w, h = mb.field_geometry(system)
        pics = torch.empty(len(fl) * w * h, dtype=torch.uint16, device="cuda")
        tbc_fields(rf, tbc_batch(rf, fl, o["demod"].data_ptr(), pics.data_ptr(), field_levels(rf)))
        torch.cuda.synchronize()
        a = fl.arrays()
        b = mb.fields[i].arrays()
        for k in ("startloc", "length", "nlines", "lineoffset"):
            np.testing.assert_array_equal(a[k], b[k])
        off = int(mb.picture_offsets[i])
        got = mb.pictures[off:off + len(fl) * w * h]
        assert torch.equal(got.view(torch.int16), pics.view(torch.int16)), i
        assert mb.picture(i, 0).shape == (h, w)


def test_pipelined_groups_equal_one_pass(batch):
    """The same captures in 3 groups (3 queues, each group's line
    locations and TBC overlapping the next group's demodulation) give the
    same fields and pictures as the one-queue pass."""
    import torch
    from ldgpu.batch import MixedBatch
    mb = batch
    torch.cuda.synchronize()
    mb.run()
    torch.cuda.synchronize()
    want = {i: [mb.picture(i, f).clone() for f in range(len(mb.fields[i]))] for i in range(len(mb.captures))}
    mp = MixedBatch(mb.captures, pipeline=3, reserve_sms=40, locate_threads=2, rfs=mb.rfs)
    assert len(mp._groups) == 3 and sum(len(g) for g in mp._groups) == len(mb.captures)
    for _ in range(2):
        n = mp.run()
        torch.cuda.synchronize()
        assert n == sum(len(f) for f in mb.fields)
        for i in range(len(mb.captures)):
            assert len(mp.fields[i]) == len(mb.fields[i])
            for f in range(len(mb.fields[i])):
                assert torch.equal(mp.picture(i, f).view(torch.int16), want[i][f].view(torch.int16)), (i, f)
    mp.close()
