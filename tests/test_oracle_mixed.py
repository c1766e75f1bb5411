"""The mixed-precision form in the oracle (no reference counterpart): its FP32
emulation against its FP64 build, and its pairing against the reference's.

The form keeps a snapshot every store_snap forward steps as 16-bit values
(binary16 or bfloat16, scaled per snapshot by a power of two) and images at
the backward steps paired with them in time, summing with Kahan
compensation.  The engine's form is checked bit for bit against the float
emulation in tests/test_gpu_mixed.py; here the emulation itself is pinned.
"""
import numpy as np
import pytest

from tests.cases import make_case


def _kw(c):
    return dict(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"], nx=c["nx"],
                vp_w=c["vp_w"], added_space=c["added_space"], nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"],
                taper_option=c["taper_option"], N_taper=c["N_taper"], N_zeros=c["N_zeros"],
                disk_mode=int(c["strategy"] == 2))


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case():
    return make_case(ny=48, nx_model=160, nt=400, dPML=8, fs=1, nrec=30, rec_step=2, sou_x=80, seed=5, f0=20.0)


def test_unit_interval_pairing_is_the_reference(oracle, case):
    """store_snap = 1 without rounding or compensation is the reference's RTM."""
    kw = _kw(case)
    a = oracle.rtm_shot_mixed(**kw, store_snap=1, q16=0, kahan=0)
    b = oracle.rtm_shot(**kw, store_snap=1, nt_snap=case["nt"])
    assert np.array_equal(a, b)


def test_emulation_against_fp64(oracle, case):
    """Image and snapshot errors of the FP32 emulation against the FP64 build.
    Tolerances: image rel-L2 <= 1e-3 with binary16 snapshots (the form's
    target); bfloat16 keeps 8 significant bits and is held to 3e-3."""
    kw = _kw(case)
    ref, F64 = oracle.rtm_shot_mixed(**kw, store_snap=4, dtype=np.float64, want_fields=True)
    assert np.abs(ref).max() > 0
    for q16, tol_img, tol_snap in ((1, 1e-3, 1e-3), (2, 3e-3, 5e-3)):
        img, F = oracle.rtm_shot_mixed(**kw, store_snap=4, q16=q16, kahan=1, want_fields=True)
        assert _rel(img, ref) <= tol_img, (q16, _rel(img, ref))
        errs = [_rel(F[m], F64[m]) for m in range(F.shape[0]) if np.abs(F64[m]).max() > 0]
        assert max(errs) <= tol_snap, (q16, max(errs))
    # unrounded FP32 snapshots: the propagation's own FP32 error only
    img = oracle.rtm_shot_mixed(**kw, store_snap=4, q16=0, kahan=1)
    assert _rel(img, ref) <= 1e-4


def test_binary16_rounding_is_nearest_even(oracle, case):
    """Snapshot values read back are multiples of the binary16 spacing of
    their scaled magnitude: scaled by the snapshot's power of two they are
    exact binary16 numbers."""
    kw = _kw(case)
    _, F = oracle.rtm_shot_mixed(**kw, store_snap=8, q16=1, kahan=1, want_fields=True)
    m = F.shape[0] // 2
    v = F[m].ravel().astype(np.float64)
    amax = np.abs(v).max()
    assert amax > 0
    k = 14 - int(np.floor(np.log2(amax)))
    scaled = v * 2.0 ** k
    assert np.abs(scaled).max() < 2 ** 15
    assert np.array_equal(scaled.astype(np.float16).astype(np.float64), scaled)
