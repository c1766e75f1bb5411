"""Stored golden vectors (tests/golden/, made by make_golden.py).

CPU: the oracle reproduces them bit for bit.  GPU: the engine, through the
C ABI, reproduces them bit for bit.
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(HERE, "*.npz")))


def load(path):
    d = dict(np.load(path))
    return {k: (v.item() if v.ndim == 0 else v) for k, v in d.items()}


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_oracle_reproduces_golden(oracle, path):
    g = load(path)
    disk = int(g["strategy"] == 2)
    xi = g["x_i"]
    F, rec = oracle.solver(1, dPML=g["dPML"], fs=g["fs"], nxSou=[g["nxSou"] - xi + 1], nySou=[g["nySou"]],
                           nxRec=g["nxRec"] - xi + 1, nyRec=g["nyRec"], S=g["src"], dmodel=g["dd"], dt=g["dt"],
                           vp=g["vp_w"], store_snap=1, nt_snap=g["nt"], nt=g["nt"], disk_mode=disk)
    assert np.array_equal(rec, g["rec"])
    assert np.array_equal(F[g["nt"] - 2], g["snap_last"])
    img = oracle.rtm_shot(dPML=g["dPML"], fs=g["fs"], nxSou=g["nxSou"], nySou=g["nySou"], nxRec=g["nxRec"],
                          nyRec=g["nyRec"], Data_source=g["src"], Data_target=g["tgt"], dd=g["dd"], dt=g["dt"],
                          nx=g["nx"], vp_w=g["vp_w"], added_space=g["added_space"], store_snap=1, nt_snap=g["nt"],
                          nt_prop2=g["nt_prop2"], nt_taper=g["nt_taper"], taper_option=g["taper_option"],
                          N_taper=g["N_taper"], N_zeros=g["N_zeros"], disk_mode=disk)
    assert np.array_equal(img, g["image"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_engine_reproduces_golden(engine, path):
    from psdm_b200.rtm import Params
    g = load(path)
    prm = Params(dPML=g["dPML"], fs=g["fs"], strategy=g["strategy"])
    F = np.zeros((g["nt"], g["nx_w"], g["ny"]), dtype=np.float32)
    rec = np.zeros((len(g["nxRec"]), g["nt"]), dtype=np.float32)
    engine.dynamic_window_solver_forward_ram(prm, [g["nxSou"]], [g["nySou"]], g["nxRec"], g["nyRec"], g["src"],
                                             g["dd"], g["dt"], g["ny"], g["nx"], g["nx_w"], g["vp_w"],
                                             g["added_space"], 1, g["nt"], g["nt"], F, rec)
    assert np.array_equal(rec, g["rec"])
    assert np.array_equal(F[g["nt"] - 2], g["snap_last"])
    img = engine.rtm_shot(prm, g["nxSou"], g["nySou"], g["nxRec"], g["nyRec"], g["src"], g["tgt"], g["dd"], g["dt"],
                          g["ny"], g["nx"], g["nx_w"], g["vp_w"], g["added_space"], 1, g["nt"], g["nt_prop2"],
                          g["nt_taper"], g["taper_option"], g["N_taper"], g["N_zeros"])
    assert np.array_equal(img, g["image"])
