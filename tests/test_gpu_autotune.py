"""psdm_engine_autotune on the GPU: the plan against the device's free
memory, the timed probe of one and two steps per launch, and the plan
applied to the engine (its images stay equal to the oracle's)."""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu


def test_autotune_probe_and_apply(engine, oracle):
    from psdm_b200.rtm import Params
    prm = Params(dPML=50, fs=1, strategy=1)
    try:
        plan = engine.autotune(prm, 1200, 1136, 8000, 8000, 1, 480, probe=True)
        print(f"\nautotune config-2 window: {plan}")
        assert plan["fits"] and plan["slots"] >= 1
        assert plan["probe_us"][0] > 0 and plan["probe_us"][1] > 0
        assert plan["steps_per_launch"] in (1, 2)
        c = make_case(fs=1, strategy=1, nt=181, seed=31)
        img = engine.rtm_shot(Params(dPML=c["dPML"], fs=1, strategy=1), c["nxSou"], c["nySou"], c["nxRec"],
                              c["nyRec"], c["src"], c["tgt"], c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"],
                              c["added_space"], 1, c["nt"], c["nt"], c["nt"])
        want = oracle.rtm_shot(dPML=c["dPML"], fs=1, nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                               nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"],
                               nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"], store_snap=1,
                               nt_snap=c["nt"], nt_prop2=c["nt"], nt_taper=c["nt"])
        assert np.array_equal(img, want)
    finally:
        engine.set_steps_per_launch(1)
        engine.set_checkpointing(0)
