"""AC3-RF (2.88 MHz DQPSK) demodulator: oracle pinned to the reference's
golden vectors, the native DPLL against the oracle on the CPU, and the GPU
front end (ldg_ac3_frontend) against the oracle and the reference symbols.

The reference's own tests (tests/test_ac3rf.py) are loopback tests: a random
symbol stream modulated as DQPSK on 2.88 MHz at 40 MSPS, fed in uneven
blocks, must come back with a > 99.9 % (clean) / > 99 % (noisy) match after
aligning on a probe subsequence.  The same criterion is used here, on a
signal whose samples are exact on every CPU (integer carrier phase index).
"""

import hashlib

import numpy as np
import pytest

from conftest import golden
from oracle import ac3 as oac3


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def g():
    return golden("ac3_loopback")


@pytest.fixture(scope="module")
def signals(g):
    clean = oac3.dqpsk_signal(g["tx"], cos_table=g["cos_table"])
    noisy = oac3.dqpsk_signal(g["tx"], noise_int=64, noise_scale=0.25 / 74.5, seed=99, cos_table=g["cos_table"])
    assert _sha(clean) == str(g["clean_sha256"]) and _sha(noisy) == str(g["noisy_sha256"])
    return clean, noisy


@pytest.fixture(scope="module")
def oracle_iq(signals):
    i, q = oac3.frontend(signals[0])
    return i, q


def _windows(g, a):
    return np.concatenate([a[lo:hi] for lo, hi in g["windows"]])


# ---- CPU: design, oracle pins, native DPLL

def test_host_taps_equal_reference(g):
    from ldgpu.ac3 import Ac3Design, halfband_kaiser, rrc_filter
    np.testing.assert_allclose(halfband_kaiser(19), g["hb19"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(halfband_kaiser(23), g["hb23"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(rrc_filter(55, 2.5e6 / 288e3, 0.7), g["rrc"], rtol=0, atol=1e-15)
    d = Ac3Design(40e6)
    assert (d.mix_frequency, d.final_frequency, d.phase_step, len(d.rrc)) == (10e6, 2.5e6, 4718, 55)
    np.testing.assert_array_equal(d.rrc, g["rrc"].astype(np.float32))
    with pytest.raises(NotImplementedError):
        Ac3Design(20e6)


def test_oracle_iq_matches_reference(g, oracle_iq):
    i, q = oracle_iq
    assert len(i) == int(g["n_iq"])
    scale = max(np.abs(g["iq_i"]).max(), np.abs(g["iq_q"]).max())
    ei = np.abs(_windows(g, i) - g["iq_i"]).max() / scale
    eq = np.abs(_windows(g, q) - g["iq_q"]).max() / scale
    # the reference runs float32 stages (numba fastmath); the oracle float64
    assert ei < 2e-5 and eq < 2e-5, (ei, eq)


def test_oracle_symbols_match_reference(g, oracle_iq):
    i, q = oracle_iq
    rx = oac3.Dpll(2.5e6).reclock(i.astype(np.float32), q.astype(np.float32))
    ref = g["rx_clean"]
    n = min(len(rx), len(ref))
    assert abs(len(rx) - len(ref)) <= 1
    assert np.mean(rx[:n] == ref[:n]) > 0.9999
    assert oac3.match_rate(g["tx"], rx) > 0.999


def test_native_dpll_equals_oracle(oracle_iq):
    from ldgpu.ac3 import Ac3Dpll
    i = oracle_iq[0].astype(np.float32)
    q = oracle_iq[1].astype(np.float32)
    want = oac3.Dpll(2.5e6).reclock(i, q)
    whole = Ac3Dpll(2.5e6).reclock_symbols(i, q)
    np.testing.assert_array_equal(whole, want)
    # streamed in uneven chunks, some shorter than one symbol distance (9)
    d = Ac3Dpll(2.5e6)
    parts, pos, k = [], 0, 0
    sizes = [5000, 3, 7, 9, 12345, 1, 20000]
    while pos < len(i):
        n = sizes[k % len(sizes)]
        parts.append(d.reclock_symbols(i[pos:pos + n], q[pos:pos + n]))
        pos += n
        k += 1
    np.testing.assert_array_equal(np.concatenate(parts), want)


def test_native_dpll_rejects_bad_args():
    from ldgpu import lib as L
    from ldgpu.ac3 import Ac3Dpll
    with pytest.raises(L.LdgError):
        Ac3Dpll(100e3)
    d = Ac3Dpll(2.5e6)
    assert len(d.reclock_symbols(np.zeros(0, np.float32), np.zeros(0, np.float32))) == 0


def test_oracle_noisy_loopback(signals, g):
    i, q = oac3.frontend(signals[1])
    rx = oac3.Dpll(2.5e6).reclock(i.astype(np.float32), q.astype(np.float32))
    assert oac3.match_rate(g["tx"], rx) > 0.99
    assert oac3.match_rate(g["tx"], g["rx_noisy"]) > 0.99


# ---- GPU

@pytest.mark.gpu
def test_gpu_frontend_matches_oracle_and_reference(cuda_ok, g, signals, oracle_iq):
    from ldgpu.ac3 import Ac3Frontend
    fe = Ac3Frontend(40e6)
    clean = signals[0]
    n_out = (len(clean) + 15) // 16
    i, q = fe.run(clean, 0, 0, n_out)
    oi, oq = oracle_iq
    assert len(oi) == n_out
    scale = np.abs(oi).max()
    assert np.abs(i - oi).max() / scale < 2e-5
    assert np.abs(q - oq).max() / scale < 2e-5
    assert np.abs(_windows(g, i) - g["iq_i"]).max() / scale < 2e-5
    assert np.abs(_windows(g, q) - g["iq_q"]).max() / scale < 2e-5
    # an interior window from a partial input reproduces the same floats
    a = 10000
    lo = 16 * a - 2048
    i2, q2 = fe.run(clean[lo:16 * (a + 777)], lo, a, 777)
    np.testing.assert_array_equal(i2, i[a:a + 777])
    np.testing.assert_array_equal(q2, q[a:a + 777])
    fe.close()


@pytest.mark.gpu
def test_gpu_frontend_int16_and_device_buffers(cuda_ok, signals):
    import torch
    from ldgpu import lib as L
    from ldgpu.ac3 import Ac3Frontend
    fe = Ac3Frontend(40e6)
    x16 = np.round(signals[1] * 8000).astype(np.int16)
    n_out = (len(x16) + 15) // 16
    oi, oq = oac3.frontend(x16.astype(np.float64))
    d_in = torch.from_numpy(x16).cuda()
    d_i = torch.empty(n_out, dtype=torch.float32, device="cuda")
    d_q = torch.empty(n_out, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    fe.run((d_in.data_ptr(), L.LDG_IN_INT16, len(x16)), 0, 0, n_out, d_i.data_ptr(), d_q.data_ptr())
    torch.cuda.synchronize()
    scale = np.abs(oi).max()
    assert np.abs(d_i.cpu().numpy() - oi).max() / scale < 2e-5
    assert np.abs(d_q.cpu().numpy() - oq).max() / scale < 2e-5
    # outputs past ceil(n/16) and windows without the filters' history are rejected
    with pytest.raises(L.LdgError):
        fe.run(x16, 0, 0, n_out + 1)
    with pytest.raises(L.LdgError):
        fe.run(x16[1000:], 1000, 100, 10)
    fe.close()


@pytest.mark.gpu
def test_gpu_streaming_demodulator_loopback(cuda_ok, g, signals):
    from ldgpu.ac3 import Ac3RfDemodulator
    clean, noisy = signals
    d = Ac3RfDemodulator(40e6)
    assert d.input_sample_alignment() == 1
    rx, pos, k = b"", 0, 0
    blocks = [int(b) for b in g["blocks"]]
    while pos < len(clean):
        n = blocks[k % 3]
        rx += d.demodulate_to_symbols(clean[pos:pos + n])
        pos += n
        k += 1
    rx = np.frombuffer(rx, np.uint8)
    ref = g["rx_clean"]
    n = min(len(rx), len(ref))
    assert abs(len(rx) - len(ref)) <= 1 and np.mean(rx[:n] == ref[:n]) > 0.9999
    assert oac3.match_rate(g["tx"], rx) > 0.999
    rxn = np.frombuffer(Ac3RfDemodulator(40e6).demodulate_to_symbols(noisy), np.uint8)
    assert oac3.match_rate(g["tx"], rxn) > 0.99
    # tiny and uneven blocks give the same symbols as one call
    d2 = Ac3RfDemodulator(40e6)
    parts, pos = [], 0
    for n in [17, 1, 4000, 33333, 2, 160000] * 100:
        if pos >= len(clean):
            break
        parts.append(d2.demodulate_to_symbols(clean[pos:pos + n]))
        pos += n
    whole = Ac3RfDemodulator(40e6).demodulate_to_symbols(clean)
    assert b"".join(parts) == whole


@pytest.mark.gpu
def test_gpu_capture_qpsk_carrier(cuda_ok):
    """A synthetic NTSC capture with the QPSK carrier in place of the right
    audio carrier (video FM, left audio, EFM and noise alongside): the
    transmitted symbols come back."""
    from ldgpu.ac3 import Ac3RfDemodulator
    from ldgpu.synth import synth_capture
    cap, tx = synth_capture("NTSC", 2_000_000, seed=5, qpsk=True, return_symbols=True)
    rx = np.frombuffer(Ac3RfDemodulator(40e6).demodulate_to_symbols(cap.numpy().astype(np.float32)), np.uint8)
    assert oac3.match_rate(tx[:len(rx)], rx) > 0.99
