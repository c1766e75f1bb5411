"""The FP64 build of the step on the GPU (psdm_rtm_shot_fp64) against the
oracle's double build of the same schedule: the same per-cell arithmetic in
double precision in the same order, so the images and snapshots agree to
rounding level (asserted within 1e-12 relative; printed whether bit for bit),
for both statement orders, with and without a free surface, a taper and
store_snap 1 and 4.  It is the GPU-side error reference of the FP32 and
mixed-precision forms (tests/test_gpu_config3.py)."""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu

CASES = [
    dict(fs=1, strategy=1, nt=240, seed=1),
    dict(fs=0, strategy=2, nt=230, seed=2, taper_option=1, N_taper=40, N_zeros=9),
    dict(ny=150, nx_model=420, nt=161, dPML=9, fs=1, strategy=1, nrec=60, rec_step=3, sou_x=300, sou_z=5,
         rec_z=3, added_space=150.0, seed=13),
]


@pytest.mark.parametrize("ks", [1, 4])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_fp64_build_vs_oracle(engine_lib, oracle, ci, ks):
    import torch
    from psdm_b200 import rtm
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = make_case(**CASES[ci])
    prm = rtm.Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"])
    img, F = rtm.rtm_shot_fp64(0, prm, c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["tgt"], c["dd"],
                               c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], ks, c["nt_prop2"],
                               c["nt_taper"], c["taper_option"], c["N_taper"], c["N_zeros"], want_fields=True)
    want, Fw = oracle.rtm_shot_mixed(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"],
                                      nxRec=c["nxRec"], nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"],
                                      dd=c["dd"], dt=c["dt"], nx=c["nx"], vp_w=c["vp_w"],
                                      added_space=c["added_space"], store_snap=ks, nt_prop2=c["nt_prop2"],
                                      nt_taper=c["nt_taper"], taper_option=c["taper_option"], N_taper=c["N_taper"],
                                      N_zeros=c["N_zeros"], disk_mode=int(c["strategy"] == 2), dtype=np.float64,
                                      want_fields=True)
    assert np.abs(want).max() > 0
    rel = np.abs(img - want).max() / np.abs(want).max()
    relF = np.abs(F - Fw).max() / np.abs(Fw).max()
    print(f"\nfp64 case {ci} ks {ks}: image max rel diff {rel:.2e} (bit for bit: {np.array_equal(img, want)}), "
          f"snapshots {relF:.2e} (bit for bit: {np.array_equal(F, Fw)})")
    assert rel <= 1e-12 and relF <= 1e-12
