"""Config 2 at full size (1200 x 4000 at 6.25 m, window 1200 x 1136, CPML 50,
free surface, 480 channels, nt 8000): one shot's RTM image (on data modelled
by the engine on the true model) against the oracle, bit for bit.  The oracle takes a few minutes on
one core.  Opt-in: set PSDM_SLOW_TESTS=1."""
import os

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.environ.get("PSDM_SLOW_TESTS"), reason="slow: set PSDM_SLOW_TESTS=1")]

NY, NX, DD, DT, DPML, F0, ADDED = 1200, 4000, 6.25, 5e-4, 50, 20.0, 500.0


@pytest.mark.parametrize("nt", [8000])
def test_config2_grid_exact(engine, oracle, nt):
    from psdm_b200 import rtm, synth
    sv = synth.config2_survey(4)
    vt = synth.config2_model(seed=2)
    vm = synth.smooth_model(vt, 100.0, DD)
    s = 1
    nxS, nyS = int(sv.nxSou[s]), int(sv.nySou[s])
    nxR, nyR = sv.nxRec[s], sv.nyRec[s]
    nx_w, x_i, x_f = oracle.dynamic_window(nxS, nxR, DD, NX, ADDED)
    src = oracle.ricker_mcs(nt, DT, F0, 0.0)
    prm = rtm.Params(dPML=DPML, fs=1, strategy=1)
    obs = engine.model_shot(prm, nxS, nyS, nxR, nyR, src, DD, DT, NY, NX, nx_w,
                            np.ascontiguousarray(vt[x_i - 1:x_f]), ADDED, nt)
    tgt = synth.mute_direct(obs, sv.pos_rec[s] - sv.pos_shot[s], DT)
    vm_w = np.ascontiguousarray(vm[x_i - 1:x_f])
    img = engine.rtm_shot(prm, nxS, nyS, nxR, nyR, src, tgt, DD, DT, NY, NX, nx_w, vm_w, ADDED, 1, nt, nt, nt)
    want = oracle.rtm_shot(dPML=DPML, fs=1, nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, Data_source=src,
                           Data_target=tgt, dd=DD, dt=DT, nx=NX, vp_w=vm_w, added_space=ADDED, store_snap=1,
                           nt_snap=nt, nt_prop2=nt, nt_taper=nt)
    assert np.abs(want).max() > 0
    bad = np.flatnonzero(~(img == want))
    assert bad.size == 0, f"{bad.size} of {img.size} values differ"
