"""Trace conditioning before the backward pass (calculate_PSDM_RTM.f90:231-355):
the engine's host window arithmetic against the oracle, and the oracle's
Akima resampling and taper against known answers."""
import numpy as np
import pytest


def _bathymetry(vel, dd, v_water=1500.0):
    """Sea-floor depth per column: (j-1-1)*dd at the first row j (1-based)
    faster than water (00-main.f90:146-157)."""
    nx, ny = vel.shape
    bat = np.zeros(nx, np.float32)
    for i in range(nx):
        j = np.flatnonzero(vel[i] > v_water)
        if j.size:
            bat[i] = np.float32(j[0] + 1 - 1 - 1) * np.float32(dd)
    return bat


@pytest.fixture(scope="module")
def geometry():
    from psdm_b200 import synth
    sv = synth.config1_survey()
    vel = synth.config1_model(seed=1)
    return sv, _bathymetry(vel, 10.0)


@pytest.mark.parametrize("cm,csf,taper,Tt,Tz", [(0, 0, 0, 0.0, 0.5), (1, 0, 0, 0.05, 0.2), (0, 1, 1, 0.1, 0.4),
                                               (1, 1, 1, 0.125, 0.5)])
def test_trace_windows_match_oracle(engine_lib, oracle, geometry, cm, csf, taper, Tt, Tz):
    from psdm_b200 import rtm
    from psdm_b200._lib import Conditioning
    sv, bat = geometry
    for s in range(sv.nshots):
        c = Conditioning(cm, csf, taper, Tt, Tz)
        cut, sf, lens = rtm.trace_windows(c, sv.nxSou[s], sv.nySou[s], sv.nxRec[s], sv.nyRec[s], bat, 10.0, 1e-3, 3000)
        o_cut, o_sf, *o_lens = oracle.trace_windows(cut_multiple=cm, cut_sf=csf, taper_option=taper, T_taper=Tt,
                                                    T_zeros=Tz, nxSou=sv.nxSou[s], nySou=sv.nySou[s],
                                                    nxRec=sv.nxRec[s], nyRec=sv.nyRec[s], Batmodel=bat,
                                                    dmodel_prop=10.0, dt_prop=1e-3, nt_prop=3000)
        assert np.array_equal(cut, o_cut) and np.array_equal(sf, o_sf) and list(lens) == o_lens
        if cm:
            assert cut.min() >= 1 and lens[0] == min(3000, cut.max())


def test_akima_known_answers(oracle):
    x = np.arange(40) * 0.004
    lin = (1.5 - 20.0 * x).astype(np.float32)
    t = np.arange(150) * 0.001
    assert np.abs(oracle.akima(lin, 0.004, 150, 0.001) - (1.5 - 20.0 * t)).max() < 1e-5
    # the nodes themselves are reproduced exactly
    y = np.random.default_rng(0).standard_normal(64).astype(np.float32)
    assert np.array_equal(oracle.akima(y, 0.002, 64, 0.002), y)
    # no overshoot at a step (Akima's locality)
    step = np.r_[np.zeros(30), np.ones(30)].astype(np.float32)
    r = oracle.akima(step, 1.0, 117, 0.5)
    assert r.min() >= 0.0 and r.max() <= 1.0


def test_condition_identity_and_taper(oracle):
    rng = np.random.default_rng(1)
    F = rng.standard_normal((5, 400)).astype(np.float32)
    cut = np.full(5, 400, np.int32)
    sf = np.ones(5, np.int32)
    out = oracle.condition_traces(cut_multiple=0, cut_sf=0, taper_option=0, Field_Data=F, dt_data=1e-3,
                                  dt_prop=1e-3, nt_prop2=400, nt_taper=400, N_taper=1, N_zeros=0, nt_cut=cut,
                                  nt_sf=sf)
    assert np.array_equal(out, F)
    # taper over the last 50 samples of 300, then 40 zeros (filters.f90:20-48)
    out = oracle.condition_traces(cut_multiple=0, cut_sf=0, taper_option=1, Field_Data=F, dt_data=1e-3,
                                  dt_prop=1e-3, nt_prop2=300, nt_taper=340, N_taper=50, N_zeros=40, nt_cut=cut,
                                  nt_sf=sf)
    w = (0.5 * (1.0 + np.cos(np.pi * np.arange(50) / 50))).astype(np.float32)
    np.testing.assert_allclose(out[:, 250:300], F[:, 250:300] * w, rtol=0, atol=1e-6 * np.abs(F).max())
    assert np.array_equal(out[:, :250], F[:, :250]) and not out[:, 300:].any()
