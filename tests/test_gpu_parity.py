"""GPU engine vs the FP32 oracle, through the C ABI.

The plain FP32 engine evaluates the reference's arithmetic in the same order
with no FMA contraction, so the bar is exact equality (value-wise: -0 == +0)
on every snapshot, receiver trace and image.
"""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu


def _prm(c, precision=0):
    from psdm_b200.rtm import Params
    return Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"], precision=precision)


def _assert_same(got, want, what):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (what, got.shape, want.shape)
    bad = np.flatnonzero(~(got == want))
    if bad.size:
        i = bad[0]
        rel = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30)
        pytest.fail(f"{what}: {bad.size} of {got.size} values differ; first at flat {i}: "
                    f"{got.flat[i]!r} vs {want.flat[i]!r}; rel-L2 {rel:.3e}")


def _forward_both(engine, oracle, c, nt_snap=None):
    nt, s = c["nt"], c["store_snap"]
    nt_snap = nt_snap or nt
    xi = c["x_i"]
    F_o, rec_o = oracle.solver(1, dPML=c["dPML"], fs=c["fs"], nxSou=[c["nxSou"] - xi + 1], nySou=[c["nySou"]],
                               nxRec=c["nxRec"] - xi + 1, nyRec=c["nyRec"], S=c["src"], dmodel=c["dd"],
                               dt=c["dt"], vp=c["vp_w"], store_snap=s, nt_snap=nt_snap, nt=nt,
                               disk_mode=int(c["strategy"] == 2))
    F_g = np.zeros_like(F_o)
    rec_g = np.zeros_like(rec_o)
    engine.dynamic_window_solver_forward_ram(_prm(c), [c["nxSou"]], [c["nySou"]], c["nxRec"], c["nyRec"], c["src"],
                                             c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"],
                                             c["added_space"], s, nt_snap, nt, F_g, rec_g)
    return F_o, rec_o, F_g, rec_g


@pytest.mark.parametrize("fs,strategy", [(0, 1), (1, 1), (1, 2)])
def test_forward_ram_exact(engine, oracle, fs, strategy):
    c = make_case(fs=fs, strategy=strategy, nt=240, seed=fs * 7 + strategy)
    F_o, rec_o, F_g, rec_g = _forward_both(engine, oracle, c)
    assert np.abs(F_o).max() > 0
    _assert_same(F_g, F_o, "Fields")
    _assert_same(rec_g, rec_o, "Data_synth")


def test_forward_store_snap(engine, oracle):
    c = make_case(store_snap=3, nt=200, fs=1, seed=3)
    F_o, rec_o, F_g, rec_g = _forward_both(engine, oracle, c, nt_snap=(200 + 2) // 3)
    _assert_same(F_g, F_o, "Fields")
    _assert_same(rec_g, rec_o, "Data_synth")


@pytest.mark.parametrize("fs,strategy,collide", [(0, 1, False), (1, 1, True), (1, 2, False)])
def test_backward_ram_exact(engine, oracle, fs, strategy, collide):
    c = make_case(fs=fs, strategy=strategy, collide=collide, nt=220, seed=11 + fs)
    nt = c["nt"]
    xi = c["x_i"]
    rng = np.random.default_rng(5)
    F = rng.standard_normal((nt, c["nx_w"], c["ny"])).astype(np.float32)
    adj = c["tgt"][:, :nt].copy()
    img_o = oracle.solver(2, dPML=c["dPML"], fs=fs, nxSou=[c["nxSou"] - xi + 1], nySou=[c["nySou"]],
                          nxRec=c["nxRec"] - xi + 1, nyRec=c["nyRec"], S=adj, dmodel=c["dd"], dt=c["dt"],
                          vp=c["vp_w"], store_snap=1, nt_snap=nt, nt=nt, Fields=F, disk_mode=int(strategy == 2))
    img_g = np.zeros((c["nx_w"], c["ny"]), dtype=np.float32)
    engine.dynamic_window_solver_backward_ram(_prm(c), [c["nxSou"]], [c["nySou"]], c["nxRec"], c["nyRec"], adj,
                                              c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"],
                                              c["added_space"], 1, nt, nt, F, img_g)
    assert np.abs(img_o).max() > 0
    _assert_same(img_g, img_o, "PSDM_thread")


@pytest.mark.parametrize("kw", [
    dict(fs=0, strategy=1),
    dict(fs=1, strategy=1),
    dict(fs=1, strategy=2),
    dict(fs=1, strategy=1, taper_option=1, N_taper=20, N_zeros=15),
    dict(fs=1, strategy=1, store_snap=2),
    dict(fs=0, strategy=1, collide=True, sou_x=20, dir_boat=1),
    dict(fs=1, strategy=1, sou_z=1),          # source on the free-surface row: wiped every step
    dict(fs=1, strategy=1, sou_x=8, nx_model=70, added_space=200.0, dir_boat=1),  # window clipped at both model edges
])
def test_rtm_shot_exact(engine, oracle, kw):
    c = make_case(nt=230, seed=21, **kw)
    img_o = oracle.rtm_shot(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                            nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"],
                            nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"], store_snap=c["store_snap"],
                            nt_snap=c["nt"], nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"],
                            taper_option=c["taper_option"], N_taper=c["N_taper"], N_zeros=c["N_zeros"],
                            disk_mode=int(c["strategy"] == 2))
    img_g = engine.rtm_shot(_prm(c), c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["tgt"], c["dd"],
                            c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], c["store_snap"],
                            c["nt"], c["nt_prop2"], c["nt_taper"], c["taper_option"], c["N_taper"], c["N_zeros"])
    if c["store_snap"] == 1 and c["nySou"] > 1:
        assert np.abs(img_o).max() > 0
    _assert_same(img_g, img_o, "PSDM_w")


def test_model_shot_matches_forward(engine, oracle):
    c = make_case(fs=1, nt=200, seed=4)
    F_o, rec_o, _, _ = _forward_both(engine, oracle, c)
    rec = engine.model_shot(_prm(c), c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["dd"], c["dt"],
                            c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], c["nt"])
    _assert_same(rec, rec_o, "Data_synth")


def test_rejects_geometry_outside_grid(engine):
    from psdm_b200._lib import PsdmError
    c = make_case(nt=50)
    bad = c["nyRec"].copy()
    bad[0] = c["ny"] + 100
    with pytest.raises(PsdmError):
        engine.model_shot(_prm(c), c["nxSou"], c["nySou"], c["nxRec"], bad, c["src"], c["dd"], c["dt"], c["ny"],
                          c["nx"], c["nx_w"], c["vp_w"], c["added_space"], c["nt"])


@pytest.mark.parametrize("dPML,fs,strategy", [(8, 1, 1), (11, 0, 2), (20, 1, 2)])
def test_rtm_shot_multi_tile_exact(engine, oracle, dPML, fs, strategy):
    """Windows spanning several 128x32 tiles, including dn not a multiple of 4."""
    c = make_case(ny=150, nx_model=420, nt=90, dPML=dPML, fs=fs, strategy=strategy, nrec=60, rec_step=3,
                  sou_x=300, sou_z=5, rec_z=3, added_space=150.0, seed=31 + dPML)
    img_o = oracle.rtm_shot(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                            nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"],
                            nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"], store_snap=1,
                            nt_snap=c["nt"], nt_prop2=c["nt"], nt_taper=c["nt"], disk_mode=int(strategy == 2))
    img_g = engine.rtm_shot(_prm(c), c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["tgt"], c["dd"],
                            c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], 1, c["nt"], c["nt"],
                            c["nt"])
    assert np.abs(img_o).max() > 0
    _assert_same(img_g, img_o, "PSDM_w")
    F_o, rec_o, F_g, rec_g = _forward_both(engine, oracle, c)
    _assert_same(F_g, F_o, "Fields")
    _assert_same(rec_g, rec_o, "Data_synth")
