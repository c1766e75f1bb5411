"""The forward kernels' snapshot quotient x / dt against the IEEE FP32
quotient (numpy's float32 division, rounded to nearest), bit for bit: the
branch-free form of the interior tiles, its fallback for float4s holding a
rare input, and the general form alone.  The reference stores
(p3 - p1) * 0.5 / dt in FP32 (src/solver_ac_forward_ram.f90:485).

Inputs cover every binary exponent from the subnormals (the values of a
wavelet's onset and of the numerical precursor ahead of a wavefront) to the
top of the range, both signs, signed zeros, the boundary where the quotient
becomes subnormal, infinities and NaN."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DTS = [5e-4, 6.25e-4, 7.5e-4, 1e-3, 1.3e-3, 3.7e-4]


def _inputs(dt, seed):
    rng = np.random.default_rng(seed)
    n = 1 << 16
    # random mantissas at every exponent, both signs
    e = rng.integers(-149, 128, size=n)
    m = rng.random(n) + 1.0
    x = (np.ldexp(m, e) * rng.choice([-1.0, 1.0], size=n)).astype(np.float32)
    # raw bit patterns of subnormal and small normal floats
    bits = rng.integers(1, 0x0D000000, size=n, dtype=np.uint32) | (rng.integers(0, 2, size=n, dtype=np.uint32) << 31)
    xs = bits.view(np.float32)
    # around the input whose quotient is the smallest normal, 2^-126 dt
    b = np.float32(np.ldexp(np.float64(dt), -126)).view(np.int32)
    edge = (b + np.arange(-2048, 2048, dtype=np.int32)).view(np.float32)
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, np.finfo(np.float32).max,
                        np.finfo(np.float32).tiny, np.float32(2.0 ** -149), -np.float32(2.0 ** -149),
                        np.float32(2.0 ** 36), np.float32(2.0 ** -90), np.float32(2.0 ** -91)], dtype=np.float32)
    x = np.concatenate([x, xs, edge, -edge, special])
    pad = (-x.size) % 4
    return np.concatenate([x, np.zeros(pad, np.float32)])


def _same(got, want):
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(got), nan)
    g, w = got[~nan].view(np.uint32), want[~nan].view(np.uint32)
    bad = np.nonzero(g != w)[0]
    assert bad.size == 0, (bad.size, got[~nan][bad[:5]], want[~nan][bad[:5]])


@pytest.mark.parametrize("dt", DTS)
def test_snapshot_quotient_is_the_ieee_quotient(engine, dt):
    x = _inputs(dt, seed=int(dt * 1e7))
    with np.errstate(all="ignore"):
        want = (x / np.float32(dt)).astype(np.float32)
    tiles, general = engine.dt_quotients(dt, x)
    _same(tiles, want)
    _same(general, want)


def test_snapshot_quotient_rejects_ragged_input(engine):
    from psdm_b200._lib import PsdmError
    with pytest.raises(PsdmError):
        engine.dt_quotients(1e-3, np.ones(6, np.float32))
