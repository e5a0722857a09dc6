"""Host side of mixed batches (ldgpu.batch): grouping captures into waves
that fit a device memory budget, and the queue failing loudly without a
GPU."""

import pytest

from ldgpu import lib as L
from ldgpu.batch import output_bytes_per_sample, waves


def test_waves_respect_budget():
    lengths = [20_000_000, 320_000_000, 100_000_000, 5_000_000, 250_000_000, 40_000_000]
    systems = ["NTSC", "PAL", "PAL", "NTSC", "NTSC", "PAL"]
    per = {s: 2 + output_bytes_per_sample(s) for s in ("NTSC", "PAL")}
    budget = 12e9
    groups = waves(lengths, systems, budget)
    assert [i for g in groups for i in g] == list(range(len(lengths)))
    for g in groups:
        used = sum(lengths[i] * per[systems[i]] for i in g)
        assert used <= budget or len(g) == 1
    # a capture larger than the budget gets a wave of its own
    assert waves([10, 10**12, 10], ["NTSC"] * 3, 1e9) == [[0], [1], [2]]
    assert output_bytes_per_sample("PAL") == output_bytes_per_sample("NTSC") + 4


def test_queue_needs_a_gpu():
    import torch
    from ldgpu.batch import DemodQueue
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(L.LdgError):
        DemodQueue(0)
