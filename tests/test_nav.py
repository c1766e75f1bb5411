"""Survey geometry on the host against the oracle's single-precision
restatements, bit for bit: the shot navigation file (read_nav_shot_mcs,
get_mcs_data.f90:30-126), channel positions (get_pos_channels, :418-510),
grid indices (get_geometry_mcs, :128-148), the velocity model on the
propagation grid (linear_2D, linear_interpolation.f90:1-117) and the
sea-floor depth from it (00-main.f90:146-158).  All on the CPU."""
import numpy as np
import pytest


def _nav_text(n, cols, seed, sep=" ", dexp=False):
    rng = np.random.default_rng(seed)
    ids = 1000 + np.arange(n)
    xs = 512345.25 + np.cumsum(rng.uniform(24.0, 26.0, n))
    ys = 4123456.5 + np.cumsum(rng.uniform(-1.0, 1.0, n))
    bat = -rng.uniform(800.0, 2500.0, n)
    lines = []
    for k in range(n):
        v = [str(ids[k]), repr(float(xs[k]))]
        if cols >= 111:
            v.append(repr(float(ys[k])))
        if cols == 1111:
            b = float(bat[k])
            v.append(("%.6Ed" % b).replace("E", "D")[:-1] if dexp else repr(b))
        lines.append(sep.join(v))
    return "\n".join(lines) + "\n"


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape and a.dtype == b.dtype
    assert np.array_equal(a, b), np.flatnonzero(a != b)[:5]


@pytest.mark.parametrize("cols", [11, 111, 1111])
@pytest.mark.parametrize("dir_boat", [1, -1])
@pytest.mark.parametrize("sep,dexp", [(" ", False), (", ", False), ("\t", True)])
def test_nav_matches_oracle(engine_lib, oracle, tmp_path, cols, dir_boat, sep, dexp):
    from psdm_b200 import rtm
    text = _nav_text(57, cols, seed=cols + dir_boat, sep=sep, dexp=dexp)
    p = tmp_path / "nav.txt"
    p.write_text(text)
    got = rtm.nav_read(p, cols, dir_boat, 250.0)
    want = oracle.nav_read(text, cols, dir_boat, 250.0)
    for g, w in zip(got[:3], want[:3]):
        _same(g, w)
    assert got[3:] == want[3:] == (1, 57)
    assert got[1][0 if dir_boat == 1 else -1] == np.float32(250.0)


def test_nav_selects_shots_and_last_duplicate_wins(engine_lib, oracle, tmp_path):
    from psdm_b200 import rtm
    text = _nav_text(20, 111, seed=3)
    text += text.splitlines()[4] + "\n"  # shot 1004 again as record 21
    p = tmp_path / "nav.txt"
    p.write_text(text)
    ids, pos, bat, li, lf = rtm.nav_read(p, 111, 1, 0.0, shot_i=1004, shot_f=1010)
    assert (li, lf) == (21, 11)
    assert oracle.nav_read(text, 111, 1, 0.0, 1004, 1010)[3:] == (21, 11)


def test_nav_errors(engine_lib, tmp_path):
    from psdm_b200 import rtm
    from psdm_b200._lib import PsdmError
    p = tmp_path / "nav.txt"
    p.write_text(_nav_text(10, 11, seed=1))
    with pytest.raises(PsdmError, match="not found"):
        rtm.nav_read(p, 11, 1, 0.0, shot_i=77)
    with pytest.raises(PsdmError, match="values"):
        rtm.nav_read(p, 1111, 1, 0.0)       # records hold 2 values, 4 asked for
    with pytest.raises(PsdmError, match="cols"):
        rtm.nav_read(p, 12, 1, 0.0)
    with pytest.raises(PsdmError, match="cannot open"):
        rtm.nav_read(tmp_path / "missing.txt", 11, 1, 0.0)


@pytest.mark.parametrize("dir_boat", [1, -1])
@pytest.mark.parametrize("header,unit", [(0, 1.0), (1, 0.1), (1, 1.0), (1, -3.0)])
def test_channel_positions_match_oracle(engine_lib, oracle, dir_boat, header, unit):
    from psdm_b200 import rtm
    rng = np.random.default_rng(9)
    offsets = (rng.integers(50, 6000, 480) * np.where(rng.random(480) < 0.5, -1, 1)).astype(np.int32)
    kw = dict(offset_unit=unit, offsets=offsets, near_offset=100.0, drec=12.5)
    got = rtm.channel_positions(7312.75, 480, dir_boat, header, **kw)
    _same(got, oracle.channel_positions(7312.75, 480, dir_boat, header, **kw))


def test_geometry_matches_oracle(engine_lib, oracle):
    from psdm_b200 import rtm
    pos_rec = rtm.channel_positions(7312.75, 480, 1, 0, near_offset=100.0, drec=12.5)
    got = rtm.geometry_mcs(7312.75, pos_rec, 8.0, 10.0, 6.25)
    want = oracle.geometry_mcs(7312.75, pos_rec, 8.0, 10.0, 6.25)
    assert got[:2] == want[:2] == (1 + int(7312.75 // 6.25), 2)
    _same(got[2], want[2])
    _same(got[3], want[3])


@pytest.mark.parametrize("d0,d1", [(10.0, 6.25), (6.25, 10.0), (12.5, 12.5)])
def test_linear_2d_matches_oracle(engine_lib, oracle, d0, d1):
    from psdm_b200 import rtm
    rng = np.random.default_rng(4)
    vel = rng.uniform(1500.0, 4000.0, (23, 17)).astype(np.float32)
    vel[5, 3:6] = 0.0      # zero nodes: the reference skips their intervals
    vel[:, 0] = 1500.0
    nxp = int((vel.shape[0] - 1) * d0 / d1) + 3   # one point past the end: held constant
    nyp = int((vel.shape[1] - 1) * d0 / d1) + 2
    got = rtm.linear_2d(vel, d0, nxp, nyp, d1)
    _same(got, oracle.linear_2d(vel, d0, nxp, nyp, d1))


def test_batmodel_matches_oracle_and_model_rule(engine_lib, oracle):
    from psdm_b200 import rtm, synth
    vel = synth.config1_model(seed=1)
    got = rtm.batmodel_from_velocity(vel, 10.0, 1500.0)
    _same(got, oracle.batmodel_from_velocity(vel, 10.0, 1500.0))
    j = np.argmax(vel > 1500.0, axis=1)
    assert np.array_equal(got, ((j - 1) * 10.0).astype(np.float32))


def test_geometry_chain_feeds_the_windows(engine_lib, oracle, tmp_path):
    """Navigation -> channel positions -> grid indices -> window, as the
    driver strings them together for one shot."""
    from psdm_b200 import rtm
    text = _nav_text(30, 1111, seed=7)
    p = tmp_path / "nav.txt"
    p.write_text(text)
    ids, pos, bat, li, lf = rtm.nav_read(p, 1111, 1, 500.0)
    k = 12
    pos_rec = rtm.channel_positions(pos[k], 60, 1, 0, near_offset=100.0, drec=6.25)
    nxs, nys, nxr, nyr = rtm.geometry_mcs(pos[k], pos_rec, 8.0, 10.0, 10.0)
    assert nxr.max() < nxs and nxr.min() >= 1
    nx_w, x_i, x_f = oracle.dynamic_window(nxs, nxr, 10.0, 1400, 500.0)
    assert 1 <= x_i <= nxr.min() and x_f >= nxs and nx_w == x_f - x_i + 1


def _obs_text(n, seed):
    rng = np.random.default_rng(seed)
    xs = np.sort(rng.uniform(1000.0, 30000.0, n))
    zs = -rng.uniform(800.0, 3000.0, n)
    return "".join(f"{k + 1} {float(xs[k])!r} {float(zs[k])!r}\n" for k in range(n))


@pytest.mark.parametrize("cols", [11, 111, 1111])
def test_nav_was_matches_oracle(engine_lib, oracle, tmp_path, cols):
    from psdm_b200 import rtm
    text = _nav_text(40, cols, seed=20 + cols)
    p = tmp_path / "nav_was.txt"
    p.write_text(text + "999 1.0 2.0 3.0\n")  # records beyond NumShots are not read
    got = rtm.nav_read_was(p, cols, 40, 250.0, 2500.0, 12.5, shot_i=1003, shot_f=1030)
    want = oracle.nav_read_was(text, cols, 40, 250.0, 2500.0, 12.5, 1003, 1030)
    for g, w in zip(got[:3], want[:3]):
        _same(g, w)
    assert got[3] == want[3] and got[3][:2] == (4, 31)
    assert got[4] == want[4]
    from psdm_b200._lib import PsdmError
    with pytest.raises(PsdmError, match="expected"):
        rtm.nav_read_was(p, cols, 60, 250.0, 2500.0, 12.5)


def test_nav_obs_and_geometry_was_match_oracle(engine_lib, oracle, tmp_path):
    from psdm_b200 import rtm
    text = _obs_text(12, seed=5)
    p = tmp_path / "nav_obs.txt"
    p.write_text(text)
    got = rtm.nav_read_obs(p, 12, 12.5)
    want = oracle.nav_read_obs(text, 12, 12.5)
    for g, w in zip(got, want):
        _same(g, w)
    shots = rtm.nav_read_was(_write(tmp_path, _nav_text(40, 11, seed=2)), 11, 40, 0.0, 0.0, 12.5)[1]
    g2 = rtm.geometry_was(int(got[3][4]), int(got[4][4]), shots, 7.5, 6.25)
    w2 = oracle.geometry_was(int(got[3][4]), int(got[4][4]), shots, 7.5, 6.25)
    assert g2[:2] == w2[:2]
    _same(g2[2], w2[2])
    _same(g2[3], w2[3])


def _write(tmp_path, text, name="n.txt"):
    p = tmp_path / name
    p.write_text(text)
    return p


@pytest.mark.parametrize("nshots", [1, 2, 5, 40])
def test_bathymetry_nav_matches_oracle(engine_lib, oracle, nshots):
    from psdm_b200 import rtm
    rng = np.random.default_rng(nshots)
    pos = np.sort(rng.uniform(100.0, 9800.0, nshots)).astype(np.float32)
    bat = rng.uniform(800.0, 2500.0, nshots).astype(np.float32)
    nxm = 801
    got = rtm.bathymetry_nav(pos, bat, 10000.0, nxm, 12.5)
    _same(got, oracle.bathymetry_nav(pos, bat, 10000.0, nxm, 12.5))
    # the interpolant passes through the shots and holds the end depths
    assert got[0] == bat[0] and got[-1] == bat[-1]


def test_akima_reproduces_cubic_free_cases(oracle):
    """Akima's method is exact for straight lines and returns its nodes."""
    from psdm_b200 import rtm
    x = np.array([0.0, 3.0, 4.5, 9.0, 10.0, 14.0], np.float32)
    y = (2.0 + 0.5 * x).astype(np.float32)
    u = np.linspace(0, 14, 57).astype(np.float32)
    v = oracle.akima_nonuniform(x, y, u)
    assert np.allclose(v, 2.0 + 0.5 * u, atol=1e-5)
    assert np.array_equal(oracle.akima_nonuniform(x, y, x), y)
    got = rtm.bathymetry_nav(x[1:-1], y[1:-1], 14.0, 15, 1.0)
    assert np.isfinite(got).all()


def test_bathymetry_rejects_unordered_shots(engine_lib):
    from psdm_b200 import rtm
    from psdm_b200._lib import PsdmError
    with pytest.raises(PsdmError, match="increase"):
        rtm.bathymetry_nav(np.array([5.0, 3.0], np.float32), np.ones(2, np.float32), 10.0, 11, 1.0)


def test_relocate_obs_matches_oracle(engine_lib, oracle):
    from psdm_b200 import rtm
    bm = np.linspace(900.0, 2100.0, 500).astype(np.float32)
    xg = np.array([1, 17, 250, 500], np.int32)
    got = rtm.relocate_obs(xg, bm, 12.5)
    want = oracle.relocate_obs(xg, bm, 12.5)
    _same(got[0], want[0])
    _same(got[1], want[1])
    from psdm_b200._lib import PsdmError
    with pytest.raises(PsdmError, match="outside"):
        rtm.relocate_obs(np.array([501], np.int32), bm, 12.5)
