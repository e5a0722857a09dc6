"""The output files of the batched path (ldgpu.writers) hold exactly the
bytes LDdecode.writeout writes (lddecode/core.py:3918-4015): each field's
uint16 picture, interleaved int16 audio, pre-PLL int16 EFM samples and
int16 RF TBC lines appended in order.  Host only."""

import os

import numpy as np
import pytest

from ldgpu.writers import FieldWriter


def _fields(n, seed=0):
    rng = np.random.default_rng(seed)
    pics = rng.integers(0, 65536, size=(n, 263 * 910), dtype=np.uint16)
    audio = [rng.integers(-32768, 32767, size=2 * int(rng.integers(700, 760)), dtype=np.int16) for _ in range(n)]
    efm = [rng.integers(-2048, 2047, size=int(rng.integers(660000, 670000)), dtype=np.int16) for _ in range(n)]
    rftbc = [rng.integers(-2048, 2047, size=int(rng.integers(1000, 2000)), dtype=np.int16) for _ in range(n)]
    return pics, audio, efm, rftbc


@pytest.mark.parametrize("background", [False, True])
def test_files_hold_the_reference_bytes(tmp_path, background):
    pics, audio, efm, rftbc = _fields(6)
    name = str(tmp_path / "cap")
    with FieldWriter(name, audio=True, prefm=True, rftbc=True, background=background) as w:
        w.write_batch(pics[:4], audio[:4], efm[:4], rftbc[:4])
        w.write(pics[4], audio[4], efm[4], rftbc[4])
        w.write_batch(pics[5:], audio[5:], efm[5:], rftbc[5:])
        w.flush()
        assert w.fields_written == 6
    # what writeout appends, field by field: file.write(array) of the native arrays
    want = {".tbc": b"".join(p.tobytes() for p in pics), ".pcm": b"".join(a.tobytes() for a in audio),
            ".prefm": b"".join(e.tobytes() for e in efm), ".rftbc": b"".join(r.tobytes() for r in rftbc)}
    for ext, b in want.items():
        with open(name + ext, "rb") as f:
            assert f.read() == b, ext


def test_optional_files_and_types(tmp_path):
    pics, audio, efm, _ = _fields(2, seed=1)
    name = str(tmp_path / "v")
    with FieldWriter(name) as w:
        w.write_batch(pics, audio, efm)
        with pytest.raises(TypeError):
            w.write(pics[0].astype(np.int32))
    assert os.path.getsize(name + ".tbc") == pics.nbytes
    for ext in (".pcm", ".prefm", ".rftbc"):
        assert not os.path.exists(name + ext)


def test_background_errors_reach_the_caller(tmp_path):
    pics, _, _, _ = _fields(2, seed=2)
    w = FieldWriter(str(tmp_path / "e"), background=True)
    w.write_batch([pics[0], pics[1].astype(np.float32)])
    with pytest.raises(TypeError):
        w.flush()
    w.close()


def test_efm_file_holds_the_reference_pll_output(tmp_path):
    """<name>.efm: the reference's EFM_PLL output of the fields' EFM samples
    in order (tests/golden/efm_pll.npz, one seeded signal cut into
    field-like pieces), written from a background thread."""
    import sys
    from conftest import GOLDEN, golden
    sys.path.insert(0, GOLDEN)
    from efm_cases import efm_case, split
    g = golden("efm_pll")
    x, bufs = efm_case("drift_up")
    parts = split(x, bufs)
    name = str(tmp_path / "d")
    pics = np.zeros((len(parts), 16), dtype=np.uint16)
    with FieldWriter(name, efm=True, prefm=True, background=True) as w:
        w.write_batch(pics[:5], None, parts[:5])
        w.write_batch(pics[5:], None, parts[5:])
    with open(name + ".efm", "rb") as f:
        assert f.read() == g["drift_up_t"].tobytes()
    with open(name + ".prefm", "rb") as f:
        assert f.read() == x.tobytes()
