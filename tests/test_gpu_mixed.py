"""The engine's mixed-precision form (prm.precision = FP16 / BF16) against
its float emulation in the oracle, bit for bit, and, for binary16 snapshots,
against the FP64 oracle of the same form within image rel-L2 1e-3 on a small
case.  bfloat16 snapshots (8 significant bits) measure 1.4e-3 on that small
case; their accuracy bar is checked on config 3 (tests/test_gpu_config3.py),
where they measure 7.6e-4."""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu

FP16, BF16 = 1, 2


def _prm(c, precision):
    from psdm_b200.rtm import Params
    return Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"], precision=precision)


def _gpu(engine, c, precision, ks):
    return engine.rtm_shot(_prm(c, precision), c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["tgt"],
                           c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], ks,
                           c["nt_taper"], c["nt_prop2"], c["nt_taper"], c["taper_option"], c["N_taper"],
                           c["N_zeros"])


def _oracle(oracle, c, q16, ks, dtype=np.float32):
    return oracle.rtm_shot_mixed(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                                 nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"],
                                 dt=c["dt"], nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"],
                                 store_snap=ks, nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"],
                                 taper_option=c["taper_option"], N_taper=c["N_taper"], N_zeros=c["N_zeros"],
                                 disk_mode=int(c["strategy"] == 2), q16=q16, kahan=1, dtype=dtype)


def _assert_same(got, want, what):
    assert got.shape == want.shape, (what, got.shape, want.shape)
    assert np.abs(want).max() > 0, what
    bad = np.flatnonzero(~(got == want))
    assert bad.size == 0, f"{what}: {bad.size} of {got.size} values differ"


CASES = [
    dict(ny=40, nx_model=120, nt=260, dPML=8, fs=1, strategy=1, seed=11),
    dict(ny=52, nx_model=140, nt=230, dPML=11, fs=0, strategy=2, seed=12, taper_option=1, N_taper=30, N_zeros=12),
    dict(ny=150, nx_model=420, nt=120, dPML=9, fs=1, strategy=1, nrec=60, rec_step=3, sou_x=300, sou_z=5,
         rec_z=3, added_space=150.0, seed=13),
]


@pytest.mark.parametrize("precision", [FP16, BF16])
@pytest.mark.parametrize("ks", [4, 1, 3])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_mixed_matches_emulation(engine, oracle, precision, ks, ci):
    c = make_case(**CASES[ci])
    _assert_same(_gpu(engine, c, precision, ks), _oracle(oracle, c, precision, ks), "PSDM_w")


@pytest.mark.parametrize("precision,tol", [(FP16, 1e-3)])
def test_mixed_accuracy_vs_fp64(engine, oracle, precision, tol):
    c = make_case(ny=64, nx_model=200, nt=600, dPML=10, fs=1, nrec=40, rec_step=2, sou_x=100, seed=5, f0=20.0)
    img = _gpu(engine, c, precision, 4)
    ref = _oracle(oracle, c, 0, 4, dtype=np.float64)
    rel = np.linalg.norm(img - ref) / np.linalg.norm(ref)
    assert rel <= tol, rel


@pytest.mark.parametrize("precision", [FP16, BF16])
def test_mixed_batch_matches_single(engine, precision):
    from psdm_b200.rtm import Params
    geo = [dict(nt=150, sou_x=52, nrec=24, rec_step=2, seed=1),
           dict(nt=210, sou_x=110, nrec=16, rec_step=3, seed=2, dir_boat=1),
           dict(nt=120, sou_x=80, nrec=30, rec_step=1, seed=3)]
    cases = [make_case(ny=40, nx_model=160, dPML=8, fs=1, strategy=1, **g) for g in geo]
    src = max(cases, key=lambda c: c["nt"])["src"]
    prm = Params(dPML=8, fs=1, strategy=1, precision=precision)
    c0 = cases[0]
    shots = [dict(nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"], nyRec=c["nyRec"], nx_w=c["nx_w"],
                  nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"], Vp_w=c["vp_w"], Data_target=c["tgt"])
             for c in cases]
    imgs = engine.rtm_batch(prm, shots, src, c0["dd"], c0["dt"], c0["ny"], c0["nx"], c0["added_space"],
                            store_snap=4, max_slots=2)
    for i, (c, img) in enumerate(zip(cases, imgs)):
        _assert_same(img, _gpu(engine, c, precision, 4), f"shot {i}")
