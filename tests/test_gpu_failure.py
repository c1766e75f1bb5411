"""The step kernels' failure path, exercised without a GPU fault: a kernel
waits with the step kernels' time limit for copies that are never issued,
gives up, reports through the engine's error word, and the engine returns
PSDM_ERR_CUDA; the next call works normally."""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu


def test_copy_wait_times_out_and_engine_recovers(engine, oracle):
    from psdm_b200._lib import PsdmError, PSDM_ERR_CUDA
    from psdm_b200.rtm import Params
    with pytest.raises(PsdmError, match="timed out") as ei:
        engine.check_wait_timeout()
    assert ei.value.code == PSDM_ERR_CUDA
    c = make_case(fs=1, nt=120, seed=21)
    prm = Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"])
    rec = engine.model_shot(prm, c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["dd"], c["dt"],
                            c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], c["nt"])
    _, want = oracle.rtm_shot(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                              nyRec=c["nyRec"], Data_source=c["src"], Data_target=np.zeros_like(c["tgt"]),
                              dd=c["dd"], dt=c["dt"], nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"],
                              store_snap=1, nt_snap=c["nt"], nt_prop2=c["nt"], nt_taper=c["nt"], want_synth=True)
    assert np.array_equal(rec, want)
