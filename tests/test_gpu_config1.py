"""Config 1 at full size (200 x 600 cells at 10 m, CPML 40, nt 3000, 120
channels, the configuration the reference can run on a CPU): the engine's
forward modelling and per-shot RTM against the oracle, bit for bit.

The observed data are the engine's forward modelling on the true model with
the direct arrival muted; the migration uses the true model smoothed over
100 m.  The source sits at 8 m depth (row 1), so the top is absorbing
(free_surface 0), as the configuration requires.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NY, NX, DD, DT, NT, DPML, F0, ADDED = 200, 600, 10.0, 1e-3, 3000, 40, 15.0, 500.0


@pytest.fixture(scope="module")
def setup():
    from psdm_b200 import synth
    sv = synth.config1_survey()
    vt = synth.config1_model(seed=1)
    vm = synth.smooth_model(vt, 100.0, DD)
    return sv, vt, vm


def _assert_same(got, want, what):
    assert got.shape == want.shape, (what, got.shape, want.shape)
    assert np.abs(want).max() > 0, what
    bad = np.flatnonzero(~(got == want))
    assert bad.size == 0, f"{what}: {bad.size} of {got.size} values differ"


@pytest.mark.parametrize("shot", [0, 3])
def test_config1_shot_exact(engine, oracle, setup, shot):
    from psdm_b200 import rtm, synth
    sv, vt, vm = setup
    nxS, nyS = int(sv.nxSou[shot]), int(sv.nySou[shot])
    nxR, nyR = sv.nxRec[shot], sv.nyRec[shot]
    nx_w, x_i, x_f = oracle.dynamic_window(nxS, nxR, DD, NX, ADDED)
    vt_w = np.ascontiguousarray(vt[x_i - 1:x_f])
    vm_w = np.ascontiguousarray(vm[x_i - 1:x_f])
    src = oracle.ricker_mcs(NT, DT, F0, 0.0)
    prm = rtm.Params(dPML=DPML, fs=0, strategy=1)
    obs = engine.model_shot(prm, nxS, nyS, nxR, nyR, src, DD, DT, NY, NX, nx_w, vt_w, ADDED, NT)
    if shot == 0:  # the forward modelling itself, once
        _, synth_o = oracle.rtm_shot(dPML=DPML, fs=0, nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, Data_source=src,
                                     Data_target=np.zeros_like(obs), dd=DD, dt=DT, nx=NX, vp_w=vt_w,
                                     added_space=ADDED, store_snap=1, nt_snap=NT, nt_prop2=NT, nt_taper=NT,
                                     want_synth=True)
        _assert_same(obs, synth_o, "Data_synth")
    tgt = synth.mute_direct(obs, sv.pos_rec[shot] - sv.pos_shot[shot], DT)
    img = engine.rtm_shot(prm, nxS, nyS, nxR, nyR, src, tgt, DD, DT, NY, NX, nx_w, vm_w, ADDED, 1, NT, NT, NT)
    want = oracle.rtm_shot(dPML=DPML, fs=0, nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, Data_source=src,
                           Data_target=tgt, dd=DD, dt=DT, nx=NX, vp_w=vm_w, added_space=ADDED, store_snap=1,
                           nt_snap=NT, nt_prop2=NT, nt_taper=NT)
    _assert_same(img, want, "PSDM_w")
