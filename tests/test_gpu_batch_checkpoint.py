"""Checkpointed shots in the batched and mixed-precision forms
(psdm_engine_set_checkpointing with psdm_rtm_batch, and with a 16-bit
precision through psdm_rtm_shot) against the same forms keeping every
snapshot, bit for bit: a checkpointed slot runs its forward pass without
snapshots, saving its state every K steps, and recomputes each segment's
snapshots (FP32, or staged and converted to 16 bits exactly as in the
uncheckpointed pass) just before the backward steps that image them.

Shots of different window widths and record lengths share fewer slots than
shots, so checkpointed slots run beside slots in other phases and are reused.
"""
import numpy as np
import pytest

from tests.test_gpu_batch import _desc, _shots

pytestmark = pytest.mark.gpu


def _prm(dPML, fs, strategy, precision):
    from psdm_b200.rtm import Params
    return Params(dPML=dPML, fs=fs, strategy=strategy, precision=precision)


def _batch(engine, prm, cases, src, ks, slots, K):
    c0 = cases[0]
    engine.set_checkpointing(K)
    try:
        return engine.rtm_batch(prm, [_desc(c) for c in cases], src, c0["dd"], c0["dt"], c0["ny"], c0["nx"],
                                c0["added_space"], ks, c0["taper_option"], c0["N_taper"], c0["N_zeros"],
                                max_slots=slots)
    finally:
        engine.set_checkpointing(0)


@pytest.mark.parametrize("precision,ks", [(0, 1), (1, 4), (2, 3), (1, 1)])
@pytest.mark.parametrize("dPML,fs,strategy,taper,slots,K", [(8, 1, 1, 0, 2, 16), (11, 0, 2, 1, 3, 7),
                                                           (10, 1, 1, 0, 4, 1000)])
def test_batch_checkpointed_equals_all_snapshots(engine, precision, ks, dPML, fs, strategy, taper, slots, K):
    cases, src = _shots(dPML, fs, strategy, taper)
    prm = _prm(dPML, fs, strategy, precision)
    want = _batch(engine, prm, cases, src, ks, slots, 0)
    got = _batch(engine, prm, cases, src, ks, slots, K)
    for i, (g, w) in enumerate(zip(got, want)):
        if precision or ks == 1:
            assert np.abs(w).max() > 0, f"shot {i}"
        bad = np.flatnonzero(~(g == w))
        assert bad.size == 0, f"shot {i}: {bad.size} of {g.size} values differ"


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("K", [5, 64])
def test_mixed_shot_checkpointed_equals_mixed(engine, oracle, precision, K):
    from tests.cases import make_case
    c = make_case(fs=1, strategy=1, nt=230, seed=44)
    prm = _prm(c["dPML"], c["fs"], c["strategy"], precision)

    def shot():
        return engine.rtm_shot(prm, c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["tgt"], c["dd"],
                               c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], 4, c["nt_taper"],
                               c["nt_prop2"], c["nt_taper"], c["taper_option"], c["N_taper"], c["N_zeros"])

    engine.set_checkpointing(0)
    want = shot()
    engine.set_checkpointing(K)
    try:
        got = shot()
    finally:
        engine.set_checkpointing(0)
    emu = oracle.rtm_shot_mixed(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                                nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"],
                                nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"], store_snap=4,
                                nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"], q16=precision, kahan=1)
    assert np.abs(want).max() > 0
    assert np.array_equal(want, emu)
    assert np.array_equal(got, want)
