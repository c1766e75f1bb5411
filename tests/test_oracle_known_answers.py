"""Known-answer tests that pin the CPU oracle (no GPU).

The reference ships no tests, fixtures or data and cannot be compiled here
(Fortran, no compiler), so the oracle's restatement of the RTM propagators is
pinned against closed forms and physics instead:
  * exact finite-difference coefficients (moment conditions),
  * closed-form C-PML profiles and Ricker wavelet,
  * the analytic 2-D Green's function of the acoustic wave equation,
  * exact mirror symmetry of the scheme,
  * FP32 vs FP64 consistency,
  * C-PML absorption (and the reflecting top/bottom strips of the RAM
    solvers' partial model padding, src/solver_ac_forward_ram.f90:288-302).
"""
import numpy as np
import pytest

def test_fd_coefficients_moments(oracle):
    c2 = oracle.fd_coef(2, dtype=np.float64)
    c1 = oracle.fd_coef(1, dtype=np.float64)
    k = np.arange(4, dtype=np.float64)
    # second derivative: sum_k c_k (f(x+k)+f(x-k)) = f'' exactly for degree <= 7
    assert abs(2 * c2.sum()) < 1e-15
    assert abs((c2 * k ** 2).sum() - 1.0) < 1e-14
    assert abs((c2 * k ** 4).sum()) < 1e-13
    assert abs((c2 * k ** 6).sum()) < 1e-12
    # first derivative: sum_k c_k (f(x+k)-f(x-k)) = f' exactly for degree <= 6
    assert abs(2 * (c1 * k).sum() - 1.0) < 1e-15
    assert abs((c1 * k ** 3).sum()) < 1e-14
    assert abs((c1 * k ** 5).sum()) < 1e-13


def test_fd_coefficients_are_rounded_rationals(oracle):
    from fractions import Fraction as Fr
    want2 = [Fr(-49, 18) / 2, Fr(3, 2), Fr(-3, 20), Fr(1, 90)]
    want1 = [Fr(0), Fr(3, 4), Fr(-3, 20), Fr(1, 60)]
    got2, got1 = oracle.fd_coef(2), oracle.fd_coef(1)
    for g, w in zip(got2, want2):
        assert abs(float(g) - float(w)) <= abs(float(w)) * 2 ** -23
    for g, w in zip(got1, want1):
        assert abs(float(g) - float(w)) <= abs(float(w)) * 2 ** -23


@pytest.mark.parametrize("dPML,dt,d", [(40, 1e-3, 10.0), (50, 5e-4, 6.25)])
def test_pml_profile_closed_form(oracle, dPML, dt, d):
    acc = 3
    fA, fB, corners = oracle.pml_coeffs(dPML, dt, d, dtype=np.float64)
    dn = dPML + 2 * acc
    i = np.arange(1, dn + 1)
    y = np.clip(i - (acc + 1), 0, dPML - 1) * d
    w = (dPML - 1) * d
    alpha = 30 * 3.14159265 * (1 - y / w)
    sigma = -(3 * 2000 * np.log(1e-5) / (2 * w)) * (y / w) ** 2
    A = np.exp(-(sigma + alpha) * dt)
    B = (A - 1) * sigma / (sigma + alpha)
    A[:acc] = 0
    B[:acc] = 0
    np.testing.assert_allclose(fA, A, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(fB, B, rtol=1e-13, atol=1e-15)
    # corners: factor at max(kx, kz), k = 1 next to the interior
    k = np.arange(1, dn + 1)
    kz, kx = np.meshgrid(k, k, indexing="ij")  # [row j, col i]
    rd = fA[np.maximum(kz, kx) - 1]
    assert np.array_equal(corners["rdA"].T, rd)              # stored [col, row]
    assert np.array_equal(corners["ldA"].T, fA[np.maximum(kz, dn - kx + 1) - 1])
    assert np.array_equal(corners["luA"].T, fA[np.maximum(dn - kz + 1, dn - kx + 1) - 1])
    assert np.array_equal(corners["ruA"].T, fA[np.maximum(dn - kz + 1, kx) - 1])


def test_ricker_closed_form(oracle):
    nt, dt, f0, t0 = 4000, 5e-4, 20.0, 0.05
    got = oracle.ricker_mcs(nt, dt, f0, t0)
    t = np.arange(nt) * dt
    a = (np.pi * f0 * (t - t0)) ** 2
    want = (1 - 2 * a) * np.exp(-a)
    want[t >= 10 / f0] = 0
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-6)


def _green_trace(r, c, t, f0, t0, nq=3000):
    """p(r,t) for p_tt = c^2 lap p + c^2 S(t) delta(x), 2-D:
    (1/2pi) * int_0^acosh(ct/r) S(t - (r/c) cosh u) du (S = 0 for t < 0)."""
    out = np.zeros_like(t)
    for i, tt in enumerate(t):
        if c * tt <= r:
            continue
        u = np.linspace(0.0, np.arccosh(c * tt / r), nq)
        tau = tt - (r / c) * np.cosh(u)
        a = (np.pi * f0 * (tau - t0)) ** 2
        s = (1 - 2 * a) * np.exp(-a)
        s[tau >= 10 / f0] = 0.0
        out[i] = np.trapezoid(s, u) / (2 * np.pi)
    return out


def test_greens_function_2d(oracle):
    """Homogeneous medium, point source: the FP64 oracle matches the analytic
    2-D Green's function convolved with the Ricker source (before any
    boundary reflection arrives).  Pins stencil, source scaling (c2*S) and the
    time alignment of injection (S(k-1) at step k) and recording
    (Rec(k-1) = p at step k)."""
    ny, nx, dd, dt, nt, f0, t0, v = 120, 121, 10.0, 1e-3, 520, 10.0, 0.15, 2000.0
    vp = np.full((nx, ny), v, np.float32)
    S = oracle.ricker_mcs(nt, dt, f0, t0)
    offs = np.array([15, 30])
    F, rec = oracle.solver(1, dPML=30, fs=0, nxSou=[61], nySou=[60], nxRec=61 + offs, nyRec=[60, 60], S=S,
                           dmodel=dd, dt=dt, vp=vp, store_snap=1, nt_snap=1, nt=nt, dtype=np.float64,
                           Fields=np.zeros((nt, nx, ny)), disk_mode=1)
    t = (np.arange(nt) + 1) * dt
    for i, o in enumerate(offs):
        want = _green_trace(o * dd, v, t, f0, t0)
        win = t < (o * dd + 2 * 450.0) / v  # before reflections from the PML
        err = np.linalg.norm(rec[i][win] - want[win]) / np.linalg.norm(want[win])
        assert err < 0.01, (o, err)


@pytest.mark.parametrize("fs,disk", [(1, 1), (0, 1)])
def test_mirror_symmetry_exact(oracle, fs, disk):
    """A source on the centre column of an x-symmetric model gives a wavefield
    that is mirror-symmetric to the last bit (the scheme, its C-PML profiles
    and edge rules are symmetric).  Only with the disk solvers' full-width
    padding: the RAM solvers pad the top/bottom strips for the left-most dn
    interior columns only, which breaks the symmetry."""
    ny, nx, nt = 40, 61, 160
    z = np.arange(ny)
    vel = np.where(z < 12, 1500.0, 2200.0).astype(np.float32)
    vp = np.ascontiguousarray(np.broadcast_to(vel, (nx, ny)))
    S = oracle.ricker_mcs(nt, 1e-3, 25.0)
    F, rec = oracle.solver(1, dPML=10, fs=fs, nxSou=[31], nySou=[5], nxRec=[21, 41], nyRec=[3, 3], S=S,
                           dmodel=10.0, dt=1e-3, vp=vp, store_snap=1, nt_snap=nt, nt=nt, disk_mode=disk)
    assert np.abs(F).max() > 0
    assert np.array_equal(F, F[:, ::-1, :])
    assert np.array_equal(rec[0], rec[1])


def test_fp32_matches_fp64(oracle):
    from tests.cases import make_case
    c = make_case(nt=300, fs=1, seed=9)
    kw = dict(dPML=c["dPML"], fs=1, nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"], nyRec=c["nyRec"],
              Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"], nx=c["nx"], vp_w=c["vp_w"],
              added_space=c["added_space"], store_snap=1, nt_snap=c["nt"], nt_prop2=c["nt"], nt_taper=c["nt"])
    i32 = oracle.rtm_shot(**kw)
    i64 = oracle.rtm_shot(dtype=np.float64, **kw)
    rel = np.linalg.norm(i32 - i64) / np.linalg.norm(i64)
    assert rel < 1e-4, rel


def _trace(oracle, ny, nx, sx, sz, rx, rz, disk, nt=700, dPML=20):
    S = oracle.ricker_mcs(nt, 1e-3, 15.0, 0.1)
    vp = np.full((nx, ny), 2000.0, np.float32)
    _, rec = oracle.solver(1, dPML=dPML, fs=0, nxSou=[sx], nySou=[sz], nxRec=[rx], nyRec=[rz], S=S, dmodel=10.0,
                           dt=1e-3, vp=vp, store_snap=1, nt_snap=1, nt=nt, dtype=np.float64,
                           Fields=np.zeros((nt, nx, ny)), disk_mode=disk)
    return rec[0]


def test_cpml_absorbs_with_full_padding(oracle):
    """Disk-solver padding (full width): the C-PML leaves < 2 % residual
    against a domain large enough that nothing comes back in the window."""
    small = _trace(oracle, 70, 70, 35, 45, 35, 55, disk=1)
    big = _trace(oracle, 300, 300, 150, 160, 150, 170, disk=1)
    assert np.linalg.norm(small - big) / np.linalg.norm(big) < 0.02


def test_ram_padding_reflects_at_top_and_bottom(oracle):
    """The RAM solvers pad the model in the top/bottom strips only for the
    first dn interior columns (`do j=1,dnx`, solver_ac_forward_ram.f90:288-302);
    elsewhere c = 0 there, so those strips reflect.  The oracle (and the
    engine, strategy 1) keep that behaviour of the reference."""
    small = _trace(oracle, 70, 70, 35, 45, 35, 55, disk=0)
    big = _trace(oracle, 300, 300, 150, 160, 150, 170, disk=0)
    assert np.linalg.norm(small - big) / np.linalg.norm(big) > 0.2
