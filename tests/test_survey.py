"""The MCS line preparation of psdm_b200.survey on files written here: a
navigation file and one SU gather per shot with offsets in the trace headers.
Geometry must equal the oracle's single-precision restatements and the
gathers the samples written, with and without a delay shift.  CPU only."""
import numpy as np
import pytest

NREC, NS_MAX, NT = 24, 300, 250


def _write_su(path, data, offsets, shot_id):
    """Fixed-length SU traces: 240-byte header (fldr @8, offset @36, ns @114)
    then NS_MAX float samples."""
    with open(path, "wb") as f:
        for j in range(data.shape[0]):
            h = np.zeros(240, np.uint8)
            h[8:12] = np.frombuffer(np.int32(shot_id).tobytes(), np.uint8)
            h[36:40] = np.frombuffer(np.int32(offsets[j]).tobytes(), np.uint8)
            h[114:116] = np.frombuffer(np.uint16(NS_MAX).tobytes(), np.uint8)
            f.write(h.tobytes())
            tr = np.zeros(NS_MAX, np.float32)
            tr[:data.shape[1]] = data[j]
            f.write(tr.tobytes())


@pytest.fixture
def line(tmp_path):
    rng = np.random.default_rng(11)
    nshots = 6
    xs = 500000.0 + 25.0 * np.arange(nshots)
    nav = "".join(f"{2000 + k} {float(xs[k])!r} 4100000.0 {-1500.0 - 3 * k!r}\n" for k in range(nshots))
    (tmp_path / "nav.txt").write_text(nav)
    paths, gathers, offs = [], [], []
    for k in range(nshots):
        g = rng.standard_normal((NREC, NS_MAX)).astype(np.float32)
        o = (-(150 + 25 * np.arange(NREC))).astype(np.int32)  # signed offsets, as many headers hold them
        p = str(tmp_path / f"shot{k}.su")
        _write_su(p, g, o, 2000 + k)
        paths.append(p)
        gathers.append(g)
        offs.append(o)
    return tmp_path, nav, paths, gathers, offs


def _cfg(tmp_path, paths, **kw):
    from psdm_b200.survey import McsLine
    base = dict(nav_path=str(tmp_path / "nav.txt"), su_paths=paths, num_rec=NREC, ns_max=NS_MAX, nt=NT, dt=4e-3,
                dd=6.25, cols=1111, dir_boat=1, d_shot_model=4000.0, shot_i=2001, shot_f=2004, shot_depth=7.5,
                streamer_depth=9.0, offset_header=1, offset_unit=1.0, byte_offset=37)
    base.update(kw)
    return McsLine(**base)


def test_line_geometry_matches_oracle(engine_lib, oracle, line):
    from psdm_b200 import survey
    tmp_path, nav, paths, gathers, offs = line
    cfg = _cfg(tmp_path, paths)
    g = survey.load_line(cfg)
    assert (g.line_i, g.line_f) == (2, 5)
    ids, pos, bat, li, lf = oracle.nav_read(nav, 1111, 1, 4000.0, 2001, 2004)
    assert np.array_equal(g.pos_shot, pos) and np.array_equal(g.pos_bat, bat)
    for k, icount in enumerate(range(2, 6)):
        pr = oracle.channel_positions(pos[icount - 1], NREC, 1, 1, 1.0, offs[icount - 1])
        assert np.array_equal(g.pos_rec[k], pr)
        nxs, nys, nxr, nyr = oracle.geometry_mcs(pos[icount - 1], pr, 7.5, 9.0, 6.25)
        assert (g.nxSou[k], g.nySou[k]) == (nxs, nys)
        assert np.array_equal(g.nxRec[k], nxr) and np.array_equal(g.nyRec[k], nyr)
        # channels trail the source (dir_boat = 1: smaller x)
        assert g.nxRec[k].max() < g.nxSou[k]


@pytest.mark.parametrize("delay", [0.0, 0.02, -0.012])
def test_shot_inputs_read_the_gather(engine_lib, line, delay):
    from psdm_b200 import survey
    tmp_path, nav, paths, gathers, offs = line
    cfg = _cfg(tmp_path, paths, delay_time=delay)
    g = survey.load_line(cfg, shots=[3])
    s = survey.shot_inputs(cfg, g, 0, 3)
    assert s["shot_id"] == 2002
    want = gathers[2][:, :NT]
    d = survey.delay_samples(cfg)
    assert d == int(np.float32(delay) / np.float32(4e-3))
    if d > 0:
        want = np.concatenate([np.zeros((NREC, d), np.float32), want[:, :NT - d]], 1)
    elif d < 0:
        want = np.concatenate([want[:, -d:], np.zeros((NREC, -d), np.float32)], 1)
    assert np.array_equal(s["Field_Data"], want)


def test_spread_geometry_without_headers(engine_lib, oracle, line):
    from psdm_b200 import survey
    tmp_path, nav, paths, gathers, offs = line
    cfg = _cfg(tmp_path, paths, offset_header=0, near_offset=150.0, drec=25.0, dir_boat=-1)
    g = survey.load_line(cfg, shots=[1, 6])
    ids, pos, *_ = oracle.nav_read(nav, 1111, -1, 4000.0)
    for k, icount in enumerate([1, 6]):
        pr = oracle.channel_positions(pos[icount - 1], NREC, -1, 0, near_offset=150.0, drec=25.0)
        assert np.array_equal(g.pos_rec[k], pr)
        assert g.nxRec[k].min() > g.nxSou[k]   # dir_boat = -1: channels at larger x


@pytest.fixture
def was_line(tmp_path):
    rng = np.random.default_rng(5)
    nshots, nobs = 40, 3
    xs = 300000.0 + 50.0 * np.arange(nshots)
    nav = "".join(f"{100 + k} {float(xs[k])!r} 4000000.0 {-1200.0 - 10.0 * np.sin(k / 5):.4f}\n"
                  for k in range(nshots))
    (tmp_path / "nav_was.txt").write_text(nav)
    obs = "".join(f"{k + 1} {500.0 + 700.0 * k!r} {-1150.0 - 20.0 * k!r}\n" for k in range(nobs))
    (tmp_path / "nav_obs.txt").write_text(obs)
    paths, gathers = [], []
    for k in range(nobs):
        g = rng.standard_normal((nshots, NS_MAX)).astype(np.float32)
        p = str(tmp_path / f"obs{k}.su")
        _write_su(p, g, np.zeros(nshots, np.int32), k + 1)
        paths.append(p)
        gathers.append(g)
    return tmp_path, nav, obs, paths, gathers


def test_was_geometry_matches_oracle(engine_lib, oracle, was_line):
    from psdm_b200 import survey
    tmp_path, nav, obs, paths, gathers = was_line
    cfg = survey.WasLine(nav_shot_path=str(tmp_path / "nav_was.txt"), nav_obs_path=str(tmp_path / "nav_obs.txt"),
                         su_paths=paths, num_shots=40, num_obs=3, ns_max=NS_MAX, nt=NT, dd=12.5, dmodel=12.5,
                         length_model=2600.0, nxmodel=209, cols=1111, d_shot_model=200.0, added_space=500.0,
                         shot_depth=6.0)
    g = survey.load_was(cfg)
    ids, pos, bat, lines, spacing = oracle.nav_read_was(nav, 1111, 40, 200.0, 500.0, 12.5)
    assert np.array_equal(g.pos_shot, pos) and g.lines == lines and g.spacing == spacing
    bm = oracle.bathymetry_nav(pos, bat, 2600.0, 209, 12.5)
    assert np.array_equal(g.bat_model, bm)
    oid, px, pz, gx, gz = oracle.nav_read_obs(obs, 3, 12.5)
    pz_r, gz_r = oracle.relocate_obs(gx, bm, 12.5)
    for i in range(3):
        zrow = gz[i] if i == 0 else gz_r[i]   # the first OBS keeps its navigation depth
        want = oracle.geometry_was(int(gx[i]), int(zrow), pos, 6.0, 12.5)
        assert (g.nxSou[i], g.nySou[i]) == want[:2]
        assert np.array_equal(g.nxRec[i], want[2]) and np.array_equal(g.nyRec[i], want[3])
    assert np.array_equal(g.pos_zobs, pz_r) and np.array_equal(g.zgrid, gz_r)
    s = survey.was_inputs(cfg, g, 2)
    assert s["obs_id"] == 2 and np.array_equal(s["Field_Data"], gathers[1][:, :NT])
