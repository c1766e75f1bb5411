"""Host-side set-up arithmetic of the engine library vs the oracle (CPU only).

These routines run on the host in the product (coefficients, wavelet,
window, taper); they must agree with the oracle bit for bit.
"""
import numpy as np
import pytest

from psdm_b200 import rtm as R


@pytest.fixture(scope="module", autouse=True)
def _lib(engine_lib):
    return engine_lib


@pytest.mark.parametrize("num", [1, 2])
def test_fd_coef_matches_oracle(oracle, num):
    assert np.array_equal(R.fd_coef(num), oracle.fd_coef(num))


@pytest.mark.parametrize("dPML,dt,d", [(10, 1e-3, 10.0), (40, 1e-3, 10.0), (50, 5e-4, 6.25), (2, 4e-4, 5.0)])
def test_pml_coeffs_match_oracle(oracle, dPML, dt, d):
    fA, fB, cg = R.pml_coeffs(dPML, dt, d, corners=True)
    oA, oB, co = oracle.pml_coeffs(dPML, dt, d)
    assert np.array_equal(fA, oA) and np.array_equal(fB, oB)
    for k in co:
        assert np.array_equal(cg[k], co[k]), k


def test_ricker_matches_oracle(oracle):
    for f0, dt, t0 in [(15.0, 1e-3, 0.0), (20.0, 5e-4, 0.05), (25.0, 4e-4, 0.0)]:
        assert np.array_equal(R.ricker_mcs(3000, dt, f0, t0), oracle.ricker_mcs(3000, dt, f0, t0))


@pytest.mark.parametrize("nxSou,lo,hi,nx,space", [(50, 10, 49, 600, 500.0), (3, 1, 200, 600, 500.0),
                                                  (590, 400, 600, 600, 500.0), (100, 20, 99, 120, 0.0)])
def test_dynamic_window_matches_oracle(oracle, nxSou, lo, hi, nx, space):
    rec = np.linspace(lo, hi, 37).astype(np.int32)
    assert R.dynamic_window(nxSou, rec, 10.0, nx, space) == oracle.dynamic_window(nxSou, rec, 10.0, nx, space)


@pytest.mark.parametrize("nt,N_taper,N_zeros", [(300, 40, 50), (300, 400, 0), (10, 1, 5)])
def test_taper_matches_oracle(oracle, nt, N_taper, N_zeros):
    tr = np.random.default_rng(1).standard_normal(nt + N_zeros).astype(np.float32)
    assert np.array_equal(R.taper_pad_trace(tr, nt, N_taper, N_zeros), oracle.taper_pad_trace(tr, nt, N_taper, N_zeros))


def test_optimization_dt():
    dt, ntp, nts = R.optimization_dt(10.0, 3500.0, 3.0, 1)
    assert dt == np.float32(np.float32(10.0) / np.float32(3500.0)) / np.float32(2.0)
    assert ntp == nts == 1 + int(np.ceil(np.float32(3.0) / np.float32(dt)))
    dt4, ntp4, nts4 = R.optimization_dt(10.0, 3500.0, 3.0, 4)
    assert ntp4 == nts4 * 4 and ntp4 >= ntp


def test_normalize_matches_oracle(oracle):
    rng = np.random.default_rng(2)
    s = rng.standard_normal((30, 20)).astype(np.float32)
    c = rng.integers(0, 3, size=(30, 20)).astype(np.float32)
    assert np.array_equal(R.normalize_psdm(s, c), oracle.normalize_psdm(s, c))
