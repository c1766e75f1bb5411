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
