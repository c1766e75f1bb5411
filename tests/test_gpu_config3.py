"""Config 3: the mixed-precision form on the config-1 model and geometry
(200 x 600 cells at 10 m, CPML 40, no free surface, Ricker 15 Hz, dt 1 ms,
nt 3000, 120 channels), binary16 and bfloat16 snapshots with a power-of-two
scale every 4 steps, FP32 image with Kahan compensation.

For each 16-bit format the GPU image must equal the oracle's float emulation
of the form bit for bit, and stay within image rel-L2 1e-3 of the FP64 build
of the same form (snapshots every 4 steps, imaging at the paired backward
steps).  The errors against the FP64 image at the full snapshot rate
(store_snap 1, the reference's imaging, solver_ac_backward_ram.f90:455-470)
and of the stored snapshots (solver_ac_forward_ram.f90:476-488) are printed
for the record: decimating the imaging to every 4th step is a property of
the form, not of the precision.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NY, NX, DD, DT, NT, DPML, F0, ADDED = 200, 600, 10.0, 1e-3, 3000, 40, 15.0, 500.0
KS = 4
FP16, BF16 = 1, 2


def _stats(a, ref):
    d = np.asarray(a, np.float64) - np.asarray(ref, np.float64)
    return float(np.linalg.norm(d) / np.linalg.norm(ref)), float(np.abs(d).max() / np.abs(ref).max())


@pytest.fixture(scope="module")
def c3(engine, oracle):
    from psdm_b200 import rtm, synth
    sv = synth.config1_survey()
    vt = synth.config1_model(seed=1)
    vm = synth.smooth_model(vt, 100.0, DD)
    s = 0
    nxS, nyS = int(sv.nxSou[s]), int(sv.nySou[s])
    nxR, nyR = sv.nxRec[s], sv.nyRec[s]
    nx_w, x_i, x_f = oracle.dynamic_window(nxS, nxR, DD, NX, ADDED)
    src = oracle.ricker_mcs(NT, DT, F0, 0.0)
    prm = rtm.Params(dPML=DPML, fs=0, strategy=1)
    obs = engine.model_shot(prm, nxS, nyS, nxR, nyR, src, DD, DT, NY, NX, nx_w,
                            np.ascontiguousarray(vt[x_i - 1:x_f]), ADDED, NT)
    tgt = synth.mute_direct(obs, sv.pos_rec[s] - sv.pos_shot[s], DT)
    kw = dict(dPML=DPML, fs=0, nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, Data_source=src, Data_target=tgt,
              dd=DD, dt=DT, nx=NX, vp_w=np.ascontiguousarray(vm[x_i - 1:x_f]), added_space=ADDED, nt_prop2=NT,
              nt_taper=NT)
    form64, snaps64 = oracle.rtm_shot_mixed(store_snap=KS, dtype=np.float64, want_fields=True, **kw)
    full64 = oracle.rtm_shot(store_snap=1, nt_snap=NT, dtype=np.float64, **kw)
    return dict(kw=kw, nx_w=nx_w, form64=form64, snaps64=snaps64, full64=full64)


@pytest.mark.parametrize("precision", [FP16, BF16])
def test_config3_mixed_image(engine, oracle, c3, precision):
    from psdm_b200 import rtm
    kw = c3["kw"]
    prm = rtm.Params(dPML=DPML, fs=0, strategy=1, precision=precision)
    img = engine.rtm_shot(prm, kw["nxSou"], kw["nySou"], kw["nxRec"], kw["nyRec"], kw["Data_source"],
                          kw["Data_target"], DD, DT, NY, NX, c3["nx_w"], kw["vp_w"], ADDED, KS, NT, NT, NT)
    emu, snaps = oracle.rtm_shot_mixed(store_snap=KS, q16=precision, kahan=1, want_fields=True, **kw)
    bad = np.flatnonzero(~(img == emu))
    assert bad.size == 0, f"{bad.size} of {img.size} image values differ from the float emulation"
    rel, peak = _stats(img, c3["form64"])
    rel_full, peak_full = _stats(img, c3["full64"])
    picks = [0, len(snaps) // 4, len(snaps) // 2, 3 * len(snaps) // 4, len(snaps) - 1]
    snap = [(m + 1, *_stats(snaps[m], c3["snaps64"][m])) for m in picks]
    name = "binary16" if precision == FP16 else "bfloat16"
    print(f"\nconfig3 {name}: image vs FP64 same form rel-L2 {rel:.3e} peak {peak:.3e}; vs FP64 full rate "
          f"rel-L2 {rel_full:.3e} peak {peak_full:.3e}; snapshots (slot, rel-L2, peak) "
          + ", ".join(f"({m}, {r:.2e}, {p:.2e})" for m, r, p in snap))
    assert rel <= 1e-3, rel
