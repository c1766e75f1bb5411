"""Boundary-saved reconstruction of the source wavefield
(psdm_engine_set_reconstruction): the image against the plain FP32 shot's
(every snapshot kept) and against the oracle.  The reverse recursion repeats
the forward step's rounding in the opposite direction, so the bar is a
tolerance: image rel-L2 <= 2e-5 against the exact image (measured 1e-6 to
3e-6), with the measured value printed; both statement orders, with and
without a free surface, a taper, and config 1 at full size."""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu


def _shot(engine, c, recon):
    from psdm_b200.rtm import Params
    try:
        engine.set_reconstruction(recon)
        return engine.rtm_shot(Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"]), c["nxSou"], c["nySou"],
                               c["nxRec"], c["nyRec"], c["src"], c["tgt"], c["dd"], c["dt"], c["ny"], c["nx"],
                               c["nx_w"], c["vp_w"], c["added_space"], 1, c["nt_taper"], c["nt_prop2"],
                               c["nt_taper"], c["taper_option"], c["N_taper"], c["N_zeros"])
    finally:
        engine.set_reconstruction(False)


CASES = [
    dict(fs=1, strategy=1, nt=300, seed=1),
    dict(fs=0, strategy=2, nt=271, seed=2, taper_option=1, N_taper=40, N_zeros=9),
    dict(ny=150, nx_model=420, nt=401, dPML=9, fs=1, strategy=1, nrec=60, rec_step=3, sou_x=300, sou_z=5,
         rec_z=3, added_space=150.0, seed=13),
]


@pytest.mark.parametrize("ci", range(len(CASES)))
def test_reconstruction_vs_plain(engine, ci):
    c = make_case(**CASES[ci])
    want = _shot(engine, c, False)
    got = _shot(engine, c, True)
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    peak = np.abs(got - want).max() / np.abs(want).max()
    print(f"\nreconstruction case {ci}: image rel-L2 {rel:.2e}, peak {peak:.2e}")
    assert np.abs(want).max() > 0
    assert rel <= 2e-5, rel


def test_reconstruction_config1(engine, oracle):
    from psdm_b200 import rtm, synth
    NY, NX, DD, DT, NT, DPML, F0, ADDED = 200, 600, 10.0, 1e-3, 3000, 40, 15.0, 500.0
    sv = synth.config1_survey()
    vt = synth.config1_model(seed=1)
    vm = synth.smooth_model(vt, 100.0, DD)
    s = 1
    nxS, nyS, nxR, nyR = int(sv.nxSou[s]), int(sv.nySou[s]), sv.nxRec[s], sv.nyRec[s]
    nx_w, x_i, x_f = oracle.dynamic_window(nxS, nxR, DD, NX, ADDED)
    src = oracle.ricker_mcs(NT, DT, F0, 0.0)
    prm = rtm.Params(dPML=DPML, fs=0, strategy=1)
    obs = engine.model_shot(prm, nxS, nyS, nxR, nyR, src, DD, DT, NY, NX, nx_w,
                            np.ascontiguousarray(vt[x_i - 1:x_f]), ADDED, NT)
    tgt = synth.mute_direct(obs, sv.pos_rec[s] - sv.pos_shot[s], DT)
    vm_w = np.ascontiguousarray(vm[x_i - 1:x_f])
    c = dict(dPML=DPML, fs=0, strategy=1, nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, src=src, tgt=tgt, dd=DD,
             dt=DT, ny=NY, nx=NX, nx_w=nx_w, vp_w=vm_w, added_space=ADDED, nt_taper=NT, nt_prop2=NT, taper_option=0,
             N_taper=1, N_zeros=0)
    got = _shot(engine, c, True)
    want = oracle.rtm_shot(dPML=DPML, fs=0, nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, Data_source=src,
                           Data_target=tgt, dd=DD, dt=DT, nx=NX, vp_w=vm_w, added_space=ADDED, store_snap=1,
                           nt_snap=NT, nt_prop2=NT, nt_taper=NT)
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    print(f"\nreconstruction config 1 (nt 3000): image rel-L2 {rel:.2e} against the oracle")
    assert rel <= 2e-5, rel
