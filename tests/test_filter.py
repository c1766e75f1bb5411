"""The frequency filter's restatement in the oracle (freq_filter,
src/auxiliar.f90:498-531, Butterworth of src/filters.f90:50-232): the
response's shape at its corners, Hermitian symmetry, linearity, all-zero
traces left as they are.  The engine's filter is checked against it in
tests/test_gpu_filter.py."""
import numpy as np
import pytest


def test_response_corners(oracle):
    ts, fe = 24000, 1000.0  # 1/24 Hz per bin
    b = lambda hz: int(round(hz * ts / fe))
    lo = np.abs(oracle.butterworth_response(ts, fe, 1, 0.0, 30.0))
    hi = np.abs(oracle.butterworth_response(ts, fe, 2, 0.0, 30.0))
    bp = np.abs(oracle.butterworth_response(ts, fe, 3, 5.0, 30.0))
    # -3 dB at the corners: fc for the low-pass, the fixed 40 Hz for the
    # high-pass, f1 and f2 for the band-pass
    for H, hz in ((lo, 30.0), (hi, 40.0), (bp, 5.0), (bp, 30.0)):
        assert abs(H[b(hz)] - 2 ** -0.5) < 1e-4, hz
    assert lo[0] == 1.0 and hi[0] == 0.0 and bp[0] == 0.0
    assert lo[b(5)] > 0.9999 and lo[b(200)] < 1e-4
    assert hi[b(5)] < 1e-5 and hi[b(200)] > 0.9999
    assert bp[b(np.sqrt(150.0))] > 0.9999 and bp[b(200)] < 1e-4


@pytest.mark.parametrize("typef", [1, 2, 3])
def test_response_is_hermitian(oracle, typef):
    ts = 24 * 37
    H = oracle.butterworth_response(ts, 250.0, typef, 4.0, 20.0)
    # the reference mirrors bins 1 .. ts/2-1; the Nyquist bin keeps the response's value
    half = ts // 2
    assert np.array_equal(H[half + 1:], np.conj(H[1:half][::-1]))


def test_filter_linear_and_real(oracle):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((3, 200))
    b = rng.standard_normal((3, 200))
    fa = oracle.freq_filter(a, 2e-3, 3, 5.0, 40.0)
    fb = oracle.freq_filter(b, 2e-3, 3, 5.0, 40.0)
    fab = oracle.freq_filter(2 * a + b, 2e-3, 3, 5.0, 40.0)
    assert np.allclose(fab, 2 * fa + fb, rtol=0, atol=1e-9 * np.abs(fab).max())


def test_low_pass_keeps_low_and_removes_high(oracle):
    dt, nt = 1e-3, 2000
    t = np.arange(nt) * dt
    low = np.sin(2 * np.pi * 4.0 * t) * np.hanning(nt)
    high = np.sin(2 * np.pi * 150.0 * t) * np.hanning(nt)
    out = oracle.freq_filter(np.stack([low + high]), dt, 1, 0.0, 30.0)[0]
    # a causal filter delays the 4 Hz wave a little: compare energies
    assert abs(np.linalg.norm(out) / np.linalg.norm(low) - 1) < 0.02
    spec = np.abs(np.fft.rfft(out))
    assert spec[int(150 * nt * dt)] < 1e-3 * spec.max()


def test_zero_traces_untouched(oracle):
    x = np.zeros((3, 50), np.float32)
    x[1, 10] = 1.0
    out = oracle.freq_filter(x, 1e-3, 1, 0.0, 25.0)
    assert np.all(out[0] == 0) and np.all(out[2] == 0) and np.any(out[1] != 0)
    assert np.array_equal(oracle.freq_filter(np.zeros((2, 9)), 1e-3, 3, 5.0, 30.0), np.zeros((2, 9)))


@pytest.mark.parametrize("typef,f1,f2", [(1, 0.0, 25.0), (2, 0.0, 30.0), (3, 5.0, 40.0)])
@pytest.mark.parametrize("ts,fe", [(24 * 750, 250.0), (24 * 1001, 500.0)])
def test_engine_response_matches_oracle(engine_lib, oracle, typef, f1, f2, ts, fe):
    """The engine computes the response on the host in single precision in
    the reference's order.  Its complex arithmetic (C++ std::complex) and
    cosine differ from numpy's in the last bits of each operation, so against
    the oracle's restatement the bar is 1e-5 of the response's largest value
    (about 10 ulp accumulated over the three section products and the
    division), ten times inside the filter's own 1e-4."""
    from psdm_b200 import rtm
    got = rtm.butterworth_response(ts, fe, typef, f1, f2)
    want = oracle.butterworth_response(ts, fe, typef, f1, f2)
    assert got.shape == want.shape
    assert got[0] == want[0]
    half = ts // 2 + 1
    err = np.abs(got[:half] - want[:half]).max()
    assert err <= 1e-5 * np.abs(want).max(), err
    assert np.array_equal(got[half:], np.conj(got[1:ts - half + 1][::-1]))
