"""The engine's frequency filter (psdm_freq_filter) against the oracle's
float64 restatement of freq_filter (src/auxiliar.f90:498-531).  The engine
transforms with cuFFT in FP32, so the bar is a tolerance, not bit equality:
rel-L2 of the filtered traces <= 1e-4, all-zero traces bit-identical
(untouched)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _traces(num, nt, dt, seed, zero_rows=()):
    rng = np.random.default_rng(seed)
    t = np.arange(nt) * dt
    x = rng.standard_normal((num, nt)).astype(np.float32)
    x += (5 * np.sin(2 * np.pi * 12.0 * t)).astype(np.float32)
    for r in zero_rows:
        x[r] = 0.0
    return x


@pytest.mark.parametrize("typef,f1,f2", [(1, 0.0, 25.0), (2, 0.0, 30.0), (3, 5.0, 40.0), (3, 2.0, 12.0)])
@pytest.mark.parametrize("num,nt,dt", [(1, 3000, 1e-3), (24, 1001, 2e-3), (120, 750, 4e-3)])
def test_filter_matches_oracle(engine, oracle, typef, f1, f2, num, nt, dt):
    x = _traces(num, nt, dt, seed=num + nt, zero_rows=(0, num - 1) if num > 2 else ())
    got = engine.freq_filter(x, dt, typef, f1, f2)
    want = oracle.freq_filter(x, dt, typef, f1, f2)
    assert got.shape == x.shape and got.dtype == np.float32
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert rel <= 1e-4, rel
    zero = ~np.any(x != 0, axis=1)
    assert np.array_equal(got[zero], x[zero])


def test_filter_rejects_bad_type(engine):
    from psdm_b200._lib import PsdmError
    with pytest.raises(PsdmError):
        engine.freq_filter(np.ones((2, 10), np.float32), 1e-3, 4, 5.0, 30.0)


def test_filter_then_condition_matches_oracle(engine, oracle):
    """The data preparation of calculate_PSDM_RTM.f90:300-355 in order:
    filter the field data, then cut, resample and taper it; the conditioning
    of the engine's filtered traces is bit-exact."""
    from psdm_b200 import rtm, synth
    from psdm_b200._lib import Conditioning
    from tests.test_conditioning import _bathymetry
    sv = synth.config1_survey()
    bat = _bathymetry(synth.config1_model(seed=1), 10.0)
    dt_prop, nt_prop, dt_data, s = 1e-3, 3000, 4e-3, 1
    nt_data = int(np.ceil(nt_prop * dt_prop / dt_data)) + 3
    c = Conditioning(1, 1, 1, 0.06, 0.25)
    cut, sf, lens = rtm.trace_windows(c, sv.nxSou[s], sv.nySou[s], sv.nxRec[s], sv.nyRec[s], bat, 10.0, dt_prop,
                                      nt_prop)
    x = _traces(len(sv.nxRec[s]), nt_data, dt_data, seed=9)
    fx = engine.freq_filter(x, dt_data, 3, 3.0, 30.0)
    want_f = oracle.freq_filter(x, dt_data, 3, 3.0, 30.0)
    assert np.linalg.norm(fx - want_f) / np.linalg.norm(want_f) <= 1e-4
    got = engine.condition_traces(c, fx, dt_data, dt_prop, cut, sf, lens)
    want = oracle.condition_traces(cut_multiple=1, cut_sf=1, taper_option=1, Field_Data=fx, dt_data=dt_data,
                                   dt_prop=dt_prop, nt_prop2=int(lens[0]), nt_taper=int(lens[1]),
                                   N_taper=int(lens[2]), N_zeros=int(lens[3]), nt_cut=cut, nt_sf=sf)
    assert np.abs(want).max() > 0
    assert np.array_equal(got, want)
