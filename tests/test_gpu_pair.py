"""Two time steps per launch against one launch per step (the default), bit
for bit, through the C ABI: snapshots and receiver traces of forward passes
with an even and an odd number of steps, images of both statement orders
with and without a free surface, tapers, store_snap > 1, colliding
receivers, sources and receivers on the free-surface row or inside the
interior, the mixed-precision form with one or two snapshots per launch,
and batched shots.  The rest of the GPU suite checks the default form
against the oracle; the two-step form is checked against it here too."""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu


def _prm(c, precision=0):
    from psdm_b200.rtm import Params
    return Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"], precision=precision)


def _same(got, want, what, allow_zero=False):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (what, got.shape, want.shape)
    assert allow_zero or np.abs(want).max() > 0, what
    bad = np.flatnonzero(~(got == want))
    assert bad.size == 0, f"{what}: {bad.size} of {got.size} values differ (first at flat {bad[:1]})"


def _both(engine, fn):
    """fn() with one step per launch, then with two; the engine is left in its
    default form (one step per launch)."""
    one = fn()
    try:
        engine.set_steps_per_launch(2)
        two = fn()
    finally:
        engine.set_steps_per_launch(1)
    return one, two


def _shot(engine, c, precision=0, ks=None):
    ks = c["store_snap"] if ks is None else ks
    return engine.rtm_shot(_prm(c, precision), c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["tgt"],
                           c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], ks,
                           c["nt_taper"], c["nt_prop2"], c["nt_taper"], c["taper_option"], c["N_taper"],
                           c["N_zeros"])


@pytest.mark.parametrize("nt", [240, 241])
@pytest.mark.parametrize("fs,strategy", [(0, 1), (1, 1), (1, 2)])
def test_forward_pair_vs_single(engine, fs, strategy, nt):
    c = make_case(fs=fs, strategy=strategy, nt=nt, seed=fs * 3 + strategy)

    def run():
        F = np.zeros((nt, c["nx_w"], c["ny"]), np.float32)
        rec = np.zeros((c["nxRec"].size, nt), np.float32)
        engine.dynamic_window_solver_forward_ram(_prm(c), [c["nxSou"]], [c["nySou"]], c["nxRec"], c["nyRec"],
                                                 c["src"], c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"],
                                                 c["added_space"], 1, nt, nt, F, rec)
        return F, rec

    (F1, r1), (F2, r2) = _both(engine, run)
    _same(F2, F1, "Fields")
    _same(r2, r1, "Data_synth")


CASES = [
    dict(fs=0, strategy=1, nt=220, seed=1),
    dict(fs=1, strategy=1, nt=221, seed=2),
    dict(fs=1, strategy=2, nt=230, seed=3, taper_option=1, N_taper=40, N_zeros=9),
    dict(fs=1, strategy=1, nt=200, seed=4, collide=True),
    dict(fs=1, strategy=1, nt=211, seed=5, sou_z=2, rec_z=2),  # injection on the row below the free surface
    dict(ny=150, nx_model=420, nt=121, dPML=9, fs=1, strategy=1, nrec=60, rec_step=3, sou_x=300, sou_z=5,
         rec_z=3, added_space=150.0, seed=13),  # clean interior tiles
    dict(ny=143, nx_model=400, nt=90, dPML=11, fs=0, strategy=2, nrec=40, rec_step=4, sou_x=260, sou_z=70,
         rec_z=90, added_space=120.0, seed=14),  # injection rows inside the interior
]


@pytest.mark.parametrize("ci", range(len(CASES)))
def test_image_pair_vs_single(engine, ci):
    c = make_case(**CASES[ci])
    one, two = _both(engine, lambda: _shot(engine, c))
    _same(two, one, "PSDM_w")


@pytest.mark.parametrize("strategy,sou_z,rec_z", [(1, 1, 2), (2, 2, 1)])
def test_injection_on_free_surface_pair_vs_single(engine, strategy, sou_z, rec_z):
    # A source or adjoint source on the free-surface row is wiped every step
    # (the reference zeroes that row after the update), so both forms give a
    # zero image.
    c = make_case(fs=1, strategy=strategy, nt=151, seed=5, sou_z=sou_z, rec_z=rec_z)
    one, two = _both(engine, lambda: _shot(engine, c))
    _same(two, one, "PSDM_w", allow_zero=True)


def test_store_snap_pair_vs_single(engine):
    # store_snap > 1 through the solver entry points (the per-shot driver's
    # pairing gives a zero image then, as the reference's RAM driver does).
    nt, ss = 200, 3
    nt_snap = (nt + ss - 1) // ss
    c = make_case(fs=1, nt=nt, seed=6)

    def fwd():
        F = np.zeros((nt_snap, c["nx_w"], c["ny"]), np.float32)
        rec = np.zeros((c["nxRec"].size, nt), np.float32)
        engine.dynamic_window_solver_forward_ram(_prm(c), [c["nxSou"]], [c["nySou"]], c["nxRec"], c["nyRec"],
                                                 c["src"], c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"],
                                                 c["added_space"], ss, nt_snap, nt, F, rec)
        return F, rec

    (F1, r1), (F2, r2) = _both(engine, fwd)
    _same(F2, F1, "Fields")
    _same(r2, r1, "Data_synth")
    Fr = np.random.default_rng(7).standard_normal((nt_snap, c["nx_w"], c["ny"])).astype(np.float32)

    def bwd():
        img = np.zeros((c["nx_w"], c["ny"]), np.float32)
        engine.dynamic_window_solver_backward_ram(_prm(c), [c["nxSou"]], [c["nySou"]], c["nxRec"], c["nyRec"],
                                                  c["tgt"][:, :nt].copy(), c["dd"], c["dt"], c["ny"], c["nx"],
                                                  c["nx_w"], c["vp_w"], c["added_space"], ss, nt_snap, nt, Fr, img)
        return img

    one, two = _both(engine, bwd)
    _same(two, one, "PSDM_thread")


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("ks", [1, 2, 3, 4])
def test_mixed_pair_vs_single(engine, precision, ks):
    c = make_case(ny=150, nx_model=420, nt=161, dPML=9, fs=1, strategy=1, nrec=60, rec_step=3, sou_x=300,
                  sou_z=5, rec_z=3, added_space=150.0, seed=20 + ks)
    one, two = _both(engine, lambda: _shot(engine, c, precision, ks))
    _same(two, one, "PSDM_w")


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_pair_vs_single(engine, precision):
    from psdm_b200.rtm import Params
    geo = [dict(nt=150, sou_x=52, nrec=24, rec_step=2, seed=1),
           dict(nt=211, sou_x=110, nrec=16, rec_step=3, seed=2, dir_boat=1),
           dict(nt=121, sou_x=80, nrec=30, rec_step=1, seed=3)]
    cases = [make_case(ny=40, nx_model=160, dPML=8, fs=1, strategy=1, **g) for g in geo]
    src = max(cases, key=lambda c: c["nt"])["src"]
    prm = Params(dPML=8, fs=1, strategy=1, precision=precision)
    c0 = cases[0]
    shots = [dict(nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"], nyRec=c["nyRec"], nx_w=c["nx_w"],
                  nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"], Vp_w=c["vp_w"], Data_target=c["tgt"])
             for c in cases]
    run = lambda: engine.rtm_batch(prm, shots, src, c0["dd"], c0["dt"], c0["ny"], c0["nx"], c0["added_space"],
                                   store_snap=4 if precision else 1, max_slots=2)
    one, two = _both(engine, run)
    for i, (a, b) in enumerate(zip(one, two)):
        _same(b, a, f"shot {i}")


def test_single_step_form_vs_oracle(engine, oracle):
    c = make_case(fs=1, strategy=1, nt=201, seed=8)
    want = oracle.rtm_shot(dPML=c["dPML"], fs=c["fs"], nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"],
                           nyRec=c["nyRec"], Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"],
                           nx=c["nx"], vp_w=c["vp_w"], added_space=c["added_space"], store_snap=1,
                           nt_snap=c["nt"], nt_prop2=c["nt"], nt_taper=c["nt"])
    one, two = _both(engine, lambda: _shot(engine, c))
    _same(one, want, "one step per launch")
    _same(two, want, "two steps per launch")
