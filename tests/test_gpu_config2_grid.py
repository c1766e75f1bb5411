"""The benchmarked configuration's grid in the default GPU suite: the full
config-2 window (1200 x 1136 cells at 6.25 m, CPML 50, free surface, 480
channels at 12.5 m) on a short record, bit for bit against the oracle.

The record is cut to a few hundred steps so that the oracle finishes in
seconds; the grid, window, tile plan, kernels and launch form are those of
the 8000-step bench shot.  Checked: every snapshot and receiver trace of the
forward pass (solver_ac_forward_ram.f90:344-577), and the image of the full
per-shot block (calculate_PSDM_RTM.f90:395-466, imaging at
solver_ac_backward_ram.f90:455-470).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NY, NX, DD, DT, DPML, F0, ADDED = 1200, 4000, 6.25, 5e-4, 50, 20.0, 500.0


@pytest.fixture(scope="module")
def shot():
    from oracle import oracle as O
    from psdm_b200 import synth
    sv = synth.config2_survey(4)
    vt = synth.config2_model(seed=2)
    vm = synth.smooth_model(vt, 100.0, DD)
    s = 1
    nxS, nyS = int(sv.nxSou[s]), int(sv.nySou[s])
    nxR, nyR = sv.nxRec[s], sv.nyRec[s]
    nx_w, x_i, x_f = O.dynamic_window(nxS, nxR, DD, NX, ADDED)
    assert nx_w == 1136
    return dict(nxS=nxS, nyS=nyS, nxR=nxR, nyR=nyR, nx_w=nx_w, x_i=x_i,
                vt_w=np.ascontiguousarray(vt[x_i - 1:x_f]), vm_w=np.ascontiguousarray(vm[x_i - 1:x_f]))


def _assert_same(got, want, what):
    assert got.shape == want.shape, (what, got.shape, want.shape)
    assert np.abs(want).max() > 0, what
    bad = np.flatnonzero(~(got == want))
    assert bad.size == 0, f"{what}: {bad.size} of {got.size} values differ (first at flat {bad[:1]})"


def test_config2_grid_forward_exact(engine, oracle, shot):
    from psdm_b200 import rtm
    nt = 120
    src = oracle.ricker_mcs(nt, DT, F0, 0.0)
    xi = shot["x_i"]
    F_o, rec_o = oracle.solver(1, dPML=DPML, fs=1, nxSou=[shot["nxS"] - xi + 1], nySou=[shot["nyS"]],
                               nxRec=shot["nxR"] - xi + 1, nyRec=shot["nyR"], S=src, dmodel=DD, dt=DT,
                               vp=shot["vt_w"], store_snap=1, nt_snap=nt, nt=nt)
    F_g = np.zeros_like(F_o)
    rec_g = np.zeros_like(rec_o)
    engine.dynamic_window_solver_forward_ram(rtm.Params(dPML=DPML, fs=1, strategy=1), [shot["nxS"]], [shot["nyS"]],
                                             shot["nxR"], shot["nyR"], src, DD, DT, NY, NX, shot["nx_w"],
                                             shot["vt_w"], ADDED, 1, nt, nt, F_g, rec_g)
    _assert_same(F_g, F_o, "Fields")
    _assert_same(rec_g, rec_o, "Data_synth")


def test_config2_grid_image_exact(engine, oracle, shot):
    from psdm_b200 import rtm
    nt = 400
    src = oracle.ricker_mcs(nt, DT, F0, 0.0)
    prm = rtm.Params(dPML=DPML, fs=1, strategy=1)
    # Observed data: the engine's modelling on the true model (the record is
    # too short for the direct-arrival mute to leave anything).
    tgt = engine.model_shot(prm, shot["nxS"], shot["nyS"], shot["nxR"], shot["nyR"], src, DD, DT, NY, NX,
                            shot["nx_w"], shot["vt_w"], ADDED, nt)
    img = engine.rtm_shot(prm, shot["nxS"], shot["nyS"], shot["nxR"], shot["nyR"], src, tgt, DD, DT, NY, NX,
                          shot["nx_w"], shot["vm_w"], ADDED, 1, nt, nt, nt)
    want = oracle.rtm_shot(dPML=DPML, fs=1, nxSou=shot["nxS"], nySou=shot["nyS"], nxRec=shot["nxR"],
                           nyRec=shot["nyR"], Data_source=src, Data_target=tgt, dd=DD, dt=DT, nx=NX,
                           vp_w=shot["vm_w"], added_space=ADDED, store_snap=1, nt_snap=nt, nt_prop2=nt,
                           nt_taper=nt)
    _assert_same(img, want, "PSDM_w")
