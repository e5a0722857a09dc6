""".lds ingest (load_packed_data_4_40 / unpack_data_4_40, lddecode/utils.py:
371-410): the oracle pinned to the reference's loader on seeded packed
bytes; on the B200 the unpack kernel (ldg_unpack_lds) and the file loader
equal the oracle at every offset and length, across CTA boundaries."""

import io

import numpy as np
import pytest

from conftest import golden
from oracle import ingest as oing


def _ref_cases():
    g = golden("lds_unpack")
    for k in range(int(g["ncases"])):
        sample, readlen = (int(x) for x in g[f"case{k}"])
        yield g["packed"], sample, readlen, g[f"out{k}"]


def test_oracle_equals_reference_loader():
    for data, sample, readlen, want in _ref_cases():
        start = (sample // 4) * 5
        got = oing.unpack_4_40(data[start:start + readlen * 5 // 4 + 5], readlen, sample % 4)
        np.testing.assert_array_equal(got, want)


def test_pack_roundtrip():
    rng = np.random.default_rng(3)
    v = rng.integers(0, 1024, 4 * 777)
    np.testing.assert_array_equal(oing.unpack_4_40(oing.pack_4_40(v), len(v), 0),
                                  ((v.astype(np.int32) - 512) * 64).astype(np.int16))


@pytest.mark.gpu
def test_gpu_unpack_equals_oracle(cuda_ok):
    import torch
    from ldgpu import lib as L
    from ldgpu.ingest import load_packed_data_4_40, unpack_lds
    rng = np.random.default_rng(5)
    packed = rng.integers(0, 256, 5 * 300_001, dtype=np.uint8)
    d = torch.from_numpy(packed).cuda()
    ref = oing.unpack_4_40(packed, 4 * 300_001, 0)
    for first, n in [(0, 4 * 300_001), (1, 1_000_000), (3, 7), (4097, 65_536 + 3), (2, 1), (1_199_999, 5),
                     (17, 4096 * 3 - 1)]:
        got = unpack_lds(d, first, n).cpu().numpy()
        np.testing.assert_array_equal(got, ref[first:first + n])
    # past the end of the packed bytes
    with pytest.raises(L.LdgError):
        unpack_lds(d, 4 * 300_001 - 2, 8)
    # the reference's loader signature, on an in-memory file
    for data, sample, readlen, want in _ref_cases():
        np.testing.assert_array_equal(load_packed_data_4_40(io.BytesIO(data.tobytes()), sample, readlen), want)
    assert load_packed_data_4_40(io.BytesIO(packed[:100].tobytes()), 0, 4096) is None
