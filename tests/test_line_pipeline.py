"""A whole marine line through the host side of the library, on the CPU:
navigation and SU files -> survey.load_line / shot_inputs -> the shot's
window (psdm_dynamic_window) -> time windows from the sea floor of the
velocity model (psdm_batmodel_from_velocity, psdm_trace_windows) -> the
driver's shot loop and image stack -> normalisation -> the SU image file.
The GPU steps (conditioning and migration) are stood in for by the oracle's
CPU restatements, which the GPU tests hold the engine to bit for bit."""
import numpy as np
import pytest

from tests.cases import layered_model
from tests.test_survey import NS_MAX, _write_su

DD, DT, NT, DPML = 10.0, 1e-3, 220, 8
NY, NX, NREC = 30, 150, 16


@pytest.fixture
def line(tmp_path, oracle):
    vel = layered_model(NY, NX, DD, seed=3, water_m=60.0)
    src = oracle.ricker_mcs(NT, DT, 25.0, 0.0)
    nshots = 4
    xs = 600.0 + 60.0 * np.arange(nshots)                 # metres along the line, dir_boat = 1
    (tmp_path / "nav.txt").write_text("".join(f"{10 + k} {float(xs[k])!r}\n" for k in range(nshots)))
    paths = []
    for k in range(nshots):
        # observed gather: the oracle's forward modelling at this shot's geometry
        nxs = 1 + int(np.floor(np.float32(xs[k]) / np.float32(DD)))
        pos_rec = np.float32(xs[k]) - (np.float32(40.0) + np.arange(NREC, dtype=np.float32) * np.float32(20.0))
        nxr = (1 + np.floor(pos_rec / np.float32(DD))).astype(np.int32)
        nyr = np.full(NREC, 2, np.int32)
        nx_w, x_i, x_f = oracle.dynamic_window(nxs, nxr, DD, NX, 100.0)
        # rtm_shot takes model coordinates and the window's slice of the model
        _, obs = oracle.rtm_shot(dPML=DPML, fs=0, nxSou=nxs, nySou=2, nxRec=nxr, nyRec=nyr,
                                 Data_source=src, Data_target=np.zeros((NREC, NT), np.float32), dd=DD, dt=DT,
                                 nx=NX, vp_w=np.ascontiguousarray(vel[x_i - 1:x_f]), added_space=100.0,
                                 store_snap=1, nt_snap=NT, nt_prop2=NT, nt_taper=NT, want_synth=True)
        p = str(tmp_path / f"shot{k}.su")
        _write_su(p, obs, np.full(NREC, 0, np.int32), 10 + k)
        paths.append(p)
    return tmp_path, vel, src, paths


def test_marine_line_on_the_host(engine_lib, oracle, line, tmp_path):
    import torch
    from psdm_b200 import driver, rtm, survey
    from psdm_b200._lib import Conditioning
    tmp, vel, src, paths = line
    # positions along the line start at d_shot_model for the first shot: 600 m,
    # where the gathers above were modelled
    cfg = survey.McsLine(nav_path=str(tmp / "nav.txt"), su_paths=paths, num_rec=NREC, ns_max=NS_MAX, nt=NT, dt=DT,
                         dd=DD, cols=11, dir_boat=1, d_shot_model=600.0, shot_depth=10.0, streamer_depth=10.0,
                         offset_header=0, near_offset=40.0, drec=20.0)
    geom = survey.load_line(cfg)
    assert (geom.line_i, geom.line_f) == (1, 4)
    assert all(r.min() >= 1 for r in geom.nxRec) and max(geom.nxSou) <= NX
    bat = rtm.batmodel_from_velocity(vel, DD, 1500.0)
    cond = Conditioning(0, 0, 0, 0.0, 0.0)
    windows = {}

    def migrate_shot(icount):
        s = survey.shot_inputs(cfg, geom, icount - geom.line_i, icount)
        nx_w, x_i, x_f = rtm.dynamic_window(s["nxSou"], s["nxRec"], DD, NX, 100.0)
        cut, sf, lens = rtm.trace_windows(cond, s["nxSou"], s["nySou"], s["nxRec"], s["nyRec"], bat, DD, DT, NT)
        tgt = oracle.condition_traces(cut_multiple=0, cut_sf=0, taper_option=0, Field_Data=s["Field_Data"],
                                      dt_data=DT, dt_prop=DT, nt_prop2=int(lens[0]), nt_taper=int(lens[1]),
                                      N_taper=int(lens[2]), N_zeros=int(lens[3]), nt_cut=cut, nt_sf=sf)
        img = oracle.rtm_shot(dPML=DPML, fs=0, nxSou=s["nxSou"], nySou=s["nySou"],
                              nxRec=s["nxRec"], nyRec=s["nyRec"], Data_source=src, Data_target=tgt, dd=DD,
                              dt=DT, nx=NX, vp_w=np.ascontiguousarray(vel[x_i - 1:x_f]), added_space=100.0,
                              store_snap=1, nt_snap=int(lens[1]), nt_prop2=int(lens[0]), nt_taper=int(lens[1]))
        windows[icount] = (img, x_i, x_f)
        return torch.from_numpy(img), x_i, x_f

    stack = driver.migrate_lines(migrate_shot, geom.line_i, geom.line_f, driver.ImageStack(NY, NX))
    final = stack.normalized()
    # the same stack by hand
    s_img = np.zeros((NX, NY), np.float32)
    s_cov = np.zeros((NX, NY), np.float32)
    for img, x_i, x_f in windows.values():
        s_img[x_i - 1:x_f] += img
        s_cov[x_i - 1:x_f] += 1.0
    assert np.array_equal(final, oracle.normalize_psdm(s_img, s_cov))
    assert np.abs(final).max() > 0 and len(windows) == 4
    # the SU image file round trip
    out = tmp_path / "PSDM_RTM.su"
    rtm.su_write_image(out, final, DD, DD)
    back, _ = rtm.su_read_shot(out, NX, NY, NY)
    assert np.array_equal(back, final)
