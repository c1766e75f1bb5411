"""Checkpointed FP32 shots (psdm_engine_set_checkpointing) against the plain
shot, bit for bit: the forward pass keeps states every K steps and the
backward pass recomputes each segment's snapshots from its checkpoint."""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu


def _shot(engine, c, ks=1):
    from psdm_b200.rtm import Params
    return engine.rtm_shot(Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"]), c["nxSou"], c["nySou"],
                           c["nxRec"], c["nyRec"], c["src"], c["tgt"], c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"],
                           c["vp_w"], c["added_space"], ks, c["nt_taper"], c["nt_prop2"], c["nt_taper"],
                           c["taper_option"], c["N_taper"], c["N_zeros"])


@pytest.mark.parametrize("K", [1, 7, 64, 1000])
@pytest.mark.parametrize("ci", [0, 1])
def test_checkpointed_shot_equals_plain(engine, K, ci):
    cases = [dict(fs=1, strategy=1, nt=230, seed=41),
             dict(ny=52, nx_model=140, nt=190, dPML=11, fs=0, strategy=2, seed=42, taper_option=1, N_taper=25,
                  N_zeros=10)]
    c = make_case(**cases[ci])
    engine.set_checkpointing(0)
    want = _shot(engine, c)
    engine.set_checkpointing(K)
    try:
        got = _shot(engine, c)
    finally:
        engine.set_checkpointing(0)
    assert np.abs(want).max() > 0
    assert np.array_equal(got, want)


def test_checkpointed_shot_with_snapshot_interval(engine, oracle):
    c = make_case(fs=1, strategy=1, nt=150, seed=43)
    engine.set_checkpointing(16)
    try:
        got = _shot(engine, c, ks=3)
    finally:
        engine.set_checkpointing(0)
    want = oracle.rtm_shot(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                           nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"],
                           nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"], store_snap=3,
                           nt_snap=c["nt_taper"], nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"])
    assert np.array_equal(got, want)
