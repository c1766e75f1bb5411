"""One cooperative launch per pass against one launch per time step, for
both pass forms: tiles that re-read their inputs every step
(psdm_engine_set_pass_launch(1)) and regions resident in shared memory
(psdm_engine_set_pass_launch(2)).  The same images, receiver traces and
mixed-precision images bit for bit, the images against the oracle, and the
launch count showing which form ran.  The large case has more tiles than
co-resident blocks, so tile blocks own several tiles, and a config-2 window
with its 480 receivers runs as resident regions."""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu

FP16 = 1
_DEFAULT = False  # the engine's default launch form


def _prm(c, precision=0):
    from psdm_b200.rtm import Params
    return Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"], precision=precision)


def _rtm(engine, c, precision=0, ks=1):
    return engine.rtm_shot(_prm(c, precision), c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["tgt"],
                           c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], ks,
                           c["nt_taper"], c["nt_prop2"], c["nt_taper"], c["taper_option"], c["N_taper"],
                           c["N_zeros"])


def _model(engine, c):
    return engine.model_shot(_prm(c), c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["dd"], c["dt"],
                             c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], c["nt"])


def _both(engine, fn, form=1):
    """fn() with one launch per pass (form 1 or 2), then with one launch per
    time step, and the engine's launch counts of each; the engine is left in
    its default form (one step per launch)."""
    out = []
    try:
        for on in (form, 0):
            engine.set_pass_launch(on)
            engine.set_steps_per_launch(1)
            engine.reset_stats()
            r = fn()
            out.append((r, engine.stats()["launches"]))
    finally:
        engine.set_pass_launch(_DEFAULT)
        engine.set_steps_per_launch(1)
    return out


def _same(a, b, what):
    assert a.shape == b.shape, what
    assert np.abs(b).max() > 0, what
    bad = np.flatnonzero(~(a == b))
    assert bad.size == 0, f"{what}: {bad.size} of {a.size} values differ"


CASES = [
    dict(ny=36, nx_model=90, nt=200, dPML=8, fs=0, strategy=1, seed=1),
    dict(ny=40, nx_model=120, nt=180, dPML=8, fs=1, strategy=1, seed=2),
    dict(ny=52, nx_model=140, nt=150, dPML=11, fs=1, strategy=2, seed=3, taper_option=1, N_taper=30, N_zeros=12),
    dict(ny=150, nx_model=420, nt=90, dPML=9, fs=0, strategy=1, nrec=60, rec_step=3, sou_x=300, sou_z=5, rec_z=3,
         added_space=150.0, seed=4, collide=True),
]


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("ci", range(len(CASES)))
def test_pass_launch_image_exact(engine, oracle, ci, form):
    c = make_case(**CASES[ci])
    (img_p, n_p), (img_s, n_s) = _both(engine, lambda: _rtm(engine, c), form)
    _same(img_p, img_s, "PSDM_w pass vs step launches")
    assert n_p < 20 and n_s >= 2 * (c["nt"] - 1), (n_p, n_s)
    want = oracle.rtm_shot(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                           nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"],
                           nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"], store_snap=1,
                           nt_snap=c["nt_taper"], nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"],
                           taper_option=c["taper_option"], N_taper=c["N_taper"], N_zeros=c["N_zeros"],
                           disk_mode=int(c["strategy"] == 2))
    _same(img_p, want, "PSDM_w pass launch vs oracle")


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("ci", [0, 1, 3])
def test_pass_launch_receivers_exact(engine, ci, form):
    c = make_case(**CASES[ci])
    (rec_p, n_p), (rec_s, _) = _both(engine, lambda: _model(engine, c), form)
    _same(rec_p, rec_s, "Rec_point pass vs step launches")
    assert n_p < 10


def test_pass_launch_mixed_backward_exact(engine):
    c = make_case(**CASES[1])
    (img_p, n_p), (img_s, n_s) = _both(engine, lambda: _rtm(engine, c, FP16, 4))
    _same(img_p, img_s, "mixed PSDM_w pass vs step launches")
    assert n_p < n_s


def test_resident_mixed_falls_back_to_steps(engine):
    """The resident form leaves the mixed-precision passes to one launch per
    step: same image, more launches than a resident shot."""
    c = make_case(**CASES[1])
    (img_p, n_p), (img_s, n_s) = _both(engine, lambda: _rtm(engine, c, FP16, 4), 2)
    _same(img_p, img_s, "mixed PSDM_w resident vs step launches")


def test_resident_config2_window(engine):
    """The config-2 window (1200 x 1136 cells, CPML 50, free surface, 480
    receivers on a 12.5 m spread) as resident regions: image and receiver
    traces equal one launch per step."""
    c = make_case(ny=1200, nx_model=1600, dd=6.25, dt=5e-4, nt=80, dPML=50, fs=1, nrec=480, rec_step=2, sou_x=1100,
                  sou_z=2, rec_z=2, added_space=540.0, seed=7)
    assert c["nx_w"] == 1136
    (img_p, n_p), (img_s, _) = _both(engine, lambda: _rtm(engine, c), 2)
    _same(img_p, img_s, "PSDM_w resident vs step launches (config-2 window)")
    assert n_p < 10
    (rec_p, n_p), (rec_s, _) = _both(engine, lambda: _model(engine, c), 2)
    _same(rec_p, rec_s, "Rec_point resident vs step launches (config-2 window)")
    assert n_p < 10


def test_pass_launch_many_tiles_per_block(engine):
    """1800 x 1361 cells: 15 x 49 interior tiles alone exceed the 5 x 148
    co-resident blocks."""
    c = make_case(ny=1800, nx_model=1600, dd=6.25, dt=5e-4, nt=60, dPML=50, fs=1, nrec=120, rec_step=2, sou_x=800,
                  sou_z=2, rec_z=2, added_space=3500.0, seed=6)
    assert c["nx_w"] == 1361
    (img_p, _), (img_s, _) = _both(engine, lambda: _rtm(engine, c))
    _same(img_p, img_s, "PSDM_w pass vs step launches (many tiles)")
    (rec_p, _), (rec_s, _) = _both(engine, lambda: _model(engine, c))
    _same(rec_p, rec_s, "Rec_point pass vs step launches (many tiles)")
