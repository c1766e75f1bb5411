"""Trace conditioning on the GPU (psdm_condition_traces) against the oracle,
bit for bit: resampling (up and down), the sea-floor cut, the multiple cut
with its taper, and the plain taper with zero padding."""
import numpy as np
import pytest

from tests.test_conditioning import _bathymetry

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cm,csf,taper,dt_data", [(0, 0, 0, 1e-3), (0, 0, 1, 2e-3), (1, 1, 1, 4e-3), (1, 0, 0, 1e-3),
                                                  (0, 1, 1, 7e-4)])
def test_condition_matches_oracle(engine, oracle, cm, csf, taper, dt_data):
    from psdm_b200 import rtm, synth
    from psdm_b200._lib import Conditioning
    sv = synth.config1_survey()
    bat = _bathymetry(synth.config1_model(seed=1), 10.0)
    dt_prop, nt_prop = 1e-3, 3000
    nt_data = int(np.ceil(nt_prop * dt_prop / dt_data)) + 3
    s = 2
    c = Conditioning(cm, csf, taper, 0.06, 0.25)
    cut, sf, lens = rtm.trace_windows(c, sv.nxSou[s], sv.nySou[s], sv.nxRec[s], sv.nyRec[s], bat, 10.0, dt_prop,
                                      nt_prop)
    rng = np.random.default_rng(7)
    F = np.cumsum(rng.standard_normal((len(sv.nxRec[s]), nt_data)), axis=1).astype(np.float32)
    got = engine.condition_traces(c, F, dt_data, dt_prop, cut, sf, lens)
    want = oracle.condition_traces(cut_multiple=cm, cut_sf=csf, taper_option=taper, Field_Data=F, dt_data=dt_data,
                                   dt_prop=dt_prop, nt_prop2=int(lens[0]), nt_taper=int(lens[1]),
                                   N_taper=int(lens[2]), N_zeros=int(lens[3]), nt_cut=cut, nt_sf=sf)
    assert got.shape == want.shape
    assert np.abs(want).max() > 0
    bad = np.flatnonzero(~(got == want))
    assert bad.size == 0, f"{bad.size} of {got.size} samples differ"
