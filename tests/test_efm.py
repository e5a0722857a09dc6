"""EFM PLL (native host code, csrc/ldg_efm.cpp, through ldgpu.efm.EFM_PLL)
against the reference's EFM_PLL (efm_pll.py:80-244) on seeded EFM-like
signals fed in buffers of uneven length (tests/golden/efm_pll.npz): every
call's T-values and the loop state at the end identical.  The PLL is host
code, so these run without a GPU."""

import hashlib
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, golden

sys.path.insert(0, GOLDEN)
from efm_cases import EFM_CASES, efm_case, split  # noqa: E402


@pytest.mark.parametrize("name", [c[0] for c in EFM_CASES])
def test_efm_pll_matches_reference(name):
    from ldgpu.efm import EFM_PLL
    g = golden("efm_pll")
    x, bufs = efm_case(name)
    assert hashlib.sha256(x.tobytes()).hexdigest() == str(g[name + "_in_sha256"])
    pll = EFM_PLL()
    res = [pll.process(b) for b in split(x, bufs)]
    np.testing.assert_array_equal([len(r) for r in res], g[name + "_counts"])
    np.testing.assert_array_equal(np.concatenate(res), g[name + "_t"])
    st = pll.state()
    np.testing.assert_array_equal([st["delta"], st["currentPeriod"], st["phaseAdjust"], st["refClockTime"]],
                                  g[name + "_state_f"])
    np.testing.assert_array_equal([st["zcPreviousInput"], st["frequencyHysteresis"], st["tCounter"]],
                                  g[name + "_state_i"])
    pll.close()


def _plain_delta(d, k):
    for _ in range(k):
        d += 1.0
    return d


def test_efm_pll_one_call_equals_many():
    """The loop state carries across calls: one call over the whole signal
    gives the concatenation of the per-buffer T-values."""
    from ldgpu.efm import EFM_PLL
    x, bufs = efm_case("dropout")
    a = EFM_PLL()
    whole = a.process(x)
    b = EFM_PLL()
    parts = np.concatenate([b.process(p) for p in split(x, [3, 70001, 1])])
    np.testing.assert_array_equal(whole, parts)
    assert a.state() == b.state()


def test_efm_pll_long_gap_delta_rounding():
    """Long runs without a crossing: the running delta after k samples must
    round as k separate additions of 1.0 do (checked against a plain loop
    through the state after a gap of each length)."""
    from ldgpu.efm import EFM_PLL
    for k in (0, 1, 2, 3, 7, 8, 9, 1000, 4097, 65537, 300001):
        # one crossing (5 -> -7, at 5/12 of a sample), then k samples without one
        x = np.concatenate([np.array([5, -7], np.int16), np.full(k, -9, np.int16)])
        pll = EFM_PLL()
        pll.process(x)
        want = _plain_delta(1.0 - 5.0 / 12.0, k)
        assert pll.state()["delta"] == want, k


def test_efm_pll_rejects_small_output_and_wrong_dtype():
    from ldgpu import lib as L
    from ldgpu.efm import EFM_PLL
    import ctypes
    pll = EFM_PLL()
    with pytest.raises(TypeError):
        pll.process(np.zeros(10, np.float32))
    x = np.zeros(100, np.int16)
    out = np.zeros(10, np.int8)
    n = ctypes.c_int64()
    rc = L.load().ldg_efm_pll_process(pll._h, x.ctypes.data, 100, out.ctypes.data, 10, ctypes.byref(n))
    assert rc == L.LDG_ERR_ARG


@pytest.mark.parametrize("name", [c[0] for c in EFM_CASES])
def test_efm_pll_from_edges_equals_samples(name):
    """The PLL run from the signal's zero crossings over field-like slices
    that overlap or leave gaps (as consecutive fields' EFM slices do) gives
    the T-values and state of the PLL fed those slices' samples."""
    from ldgpu.efm import EFM_PLL
    from helpers import efm_crossings
    x, _ = efm_case(name)
    edges = efm_crossings(x)
    rng = np.random.default_rng(7)
    slices, lo = [], 0
    while lo < len(x) - 10:
        hi = min(len(x), lo + int(rng.integers(1, 40000)))
        slices.append((lo, hi))
        lo = max(0, hi + int(rng.integers(-3, 4)))  # overlap, touch or gap
    a, b = EFM_PLL(), EFM_PLL()
    for lo, hi in slices:
        want = a.process(x[lo:hi])
        got = b.process_edges(edges, lo, hi, x[lo], x[hi - 1])
        np.testing.assert_array_equal(got, want)
    assert a.state() == b.state()
    a.close()
    b.close()
