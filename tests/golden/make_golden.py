"""Generate tests/golden/*.npz: small RTM cases run through the CPU oracle.

    python tests/golden/make_golden.py

The reference (Fortran) cannot be compiled or run in this environment and
ships no fixtures, so these vectors are the oracle's own outputs on seeded
inputs.  They pin the oracle against regressions (test_golden.py) and give
the GPU tests a stored expectation that does not depend on re-running the
oracle.  Inputs are stored next to the outputs.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from tests.cases import make_case  # noqa: E402

CASES = {
    "ram_fs1": dict(fs=1, strategy=1, nt=240, seed=101),
    "disk_fs0_taper": dict(fs=0, strategy=2, nt=220, seed=102, taper_option=1, N_taper=30, N_zeros=20),
    "ram_fs0_collide": dict(fs=0, strategy=1, nt=200, seed=103, collide=True, sou_x=20, dir_boat=1),
}


def run(name, kw):
    c = make_case(**kw)
    disk = int(c["strategy"] == 2)
    xi = c["x_i"]
    F, rec = O.solver(1, dPML=c["dPML"], fs=c["fs"], nxSou=[c["nxSou"] - xi + 1], nySou=[c["nySou"]],
                      nxRec=c["nxRec"] - xi + 1, nyRec=c["nyRec"], S=c["src"], dmodel=c["dd"], dt=c["dt"],
                      vp=c["vp_w"], store_snap=1, nt_snap=c["nt"], nt=c["nt"], disk_mode=disk)
    img = O.rtm_shot(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                     nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"],
                     nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"], store_snap=1, nt_snap=c["nt"],
                     nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"], taper_option=c["taper_option"],
                     N_taper=c["N_taper"], N_zeros=c["N_zeros"], disk_mode=disk)
    scal = {k: c[k] for k in ("ny", "nx", "dd", "dt", "nt", "dPML", "fs", "strategy", "nxSou", "nySou", "nx_w",
                              "x_i", "added_space", "nt_prop2", "nt_taper", "taper_option", "N_taper", "N_zeros")}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), vp_w=c["vp_w"], src=c["src"], tgt=c["tgt"],
                        nxRec=c["nxRec"], nyRec=c["nyRec"], rec=rec, snap_last=F[c["nt"] - 2], image=img,
                        **{k: np.asarray(v) for k, v in scal.items()})


if __name__ == "__main__":
    for name, kw in CASES.items():
        run(name, kw)
        print("wrote", name)
