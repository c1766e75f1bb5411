"""ctypes wrapper of the CPU oracle (liboracle_rtm.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, and only to check the engine against.  The CUDA engine in
psdm_b200/ never imports this module.

The oracle restates the reference's Fortran RTM solvers step by step (see the
header of rtm_oracle.cpp for the file:line list).  Parity with the reference's
own outputs is UNPINNED (no Fortran compiler exists here and the reference
ships no tests or data); known-answer tests in tests/test_oracle_*.py pin it.

Arrays follow the reference's Fortran layout: a model or image (ny, nx) is a
numpy array of shape (nx, ny) in C order (column-major (ny, nx)), traces
(nt, NumRec) are shape (NumRec, nt), Fields (ny, nx, nt_snap) is shape
(nt_snap, nx, ny).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_rtm.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_I, _F, _D = C.c_int, C.c_float, C.c_double


def build() -> str:
    """Compile liboracle_rtm.so with the oracle's Makefile (g++, no GPU)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_fd_coef_f.argtypes = [_I, _I, _f32p]
        L.orc_fd_coef_d.argtypes = [_I, _I, _f64p]
        L.orc_pml_coeffs_f.argtypes = [_I, _I, _F, _F, _I, _f32p, _f32p, _f32p]
        L.orc_pml_coeffs_d.argtypes = [_I, _I, _D, _D, _I, _f64p, _f64p, _f64p]
        L.orc_ricker_mcs.argtypes = [_I, _F, _F, _F, _f32p]
        L.orc_taper_pad_trace_f.argtypes = [_f32p, _I, _I, _I, _I]
        L.orc_dynamic_window.argtypes = [_I, _I, _i32p, _F, _I, _F, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)]
        L.orc_solver_f.argtypes = [_I, _I, _I, _I, _I, _i32p, _i32p, _i32p, _i32p, _f32p, _F, _F, _I, _I,
                                   _f32p, _I, _I, _I, _f32p, _f32p]
        L.orc_solver_dump_f.argtypes = [_I, _I, _I, _I, _I, _i32p, _i32p, _i32p, _i32p, _f32p, _F, _F, _I, _I,
                                        _f32p, _I, _I, _I, _f32p, _f32p, _f32p]
        L.orc_solver_d.argtypes = [_I, _I, _I, _I, _I, _i32p, _i32p, _i32p, _i32p, _f32p, _I, _F, _F, _I, _I,
                                   _f32p, _I, _I, _I, _f64p, _f64p]
        shot_args = [_I, _I, _I, _I, _I, _I, _i32p, _i32p, _f32p, _f32p, _F, _F, _I, _I, _I, _f32p, _F,
                     _I, _I, _I, _I, _I, _I, _I]
        L.orc_rtm_shot_f.argtypes = shot_args + [_f32p, C.c_void_p]
        L.orc_rtm_shot_d.argtypes = shot_args + [_f64p, C.c_void_p]
        L.orc_normalize_psdm.argtypes = [_I, _I, _f32p, _f32p, _f32p]
        # disk_mode .. N_zeros without nt_snap (mixed form)
        mixed_args = [_I, _I, _I, _I, _I, _I, _i32p, _i32p, _f32p, _f32p, _F, _F, _I, _I, _I, _f32p, _F,
                      _I, _I, _I, _I, _I, _I]
        L.orc_rtm_shot_mixed_f.argtypes = [_I, _I] + mixed_args + [_f32p, C.c_void_p]
        L.orc_rtm_shot_mixed_d.argtypes = mixed_args + [_f64p, C.c_void_p]
        L.orc_trace_windows.argtypes = [_I, _I, _I, _F, _F, _I, _I, _I, _i32p, _i32p, _f32p, _F, _F, _I, _i32p,
                                        _i32p, _i32p]
        L.orc_akima.argtypes = [_f32p, _I, _F, _I, _F, _f32p]
        L.orc_condition_traces.argtypes = [_I, _I, _I, _I, _f32p, _I, _F, _F, _I, _I, _I, _I, _i32p, _i32p, _f32p]
        _lib = L
    return _lib


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def fd_coef(num: int, acc: int = 3, dtype=np.float32) -> np.ndarray:
    c = np.zeros(acc + 1, dtype=dtype)
    (lib().orc_fd_coef_f if dtype == np.float32 else lib().orc_fd_coef_d)(num, acc, c)
    return c


def pml_coeffs(dPML: int, dt: float, d: float, acc: int = 3, dtype=np.float32):
    """factorA, factorB (dn,) and the corner matrices ld, rd, lu, ru (A then B),
    each shape (dn, dn) indexed [col-1, row-1] (column-major)."""
    dn = dPML + 2 * acc
    fA = np.zeros(dn, dtype=dtype)
    fB = np.zeros(dn, dtype=dtype)
    corners = np.zeros(8 * dn * dn, dtype=dtype)
    if dtype == np.float32:
        lib().orc_pml_coeffs_f(acc, dPML, dt, d, dn, fA, fB, corners)
    else:
        lib().orc_pml_coeffs_d(acc, dPML, dt, d, dn, fA, fB, corners)
    c = corners.reshape(8, dn, dn)
    names = ["ldA", "rdA", "luA", "ruA", "ldB", "rdB", "luB", "ruB"]
    return fA, fB, {n: c[q] for q, n in enumerate(names)}


def ricker_mcs(nt: int, dt: float, f0: float, t0: float = 0.0) -> np.ndarray:
    s = np.zeros(nt, dtype=np.float32)
    lib().orc_ricker_mcs(nt, dt, f0, t0, s)
    return s


def taper_pad_trace(trace, nt_prop: int, N_taper: int, N_zeros: int) -> np.ndarray:
    t = _f32(trace).copy()
    lib().orc_taper_pad_trace_f(t, nt_prop, N_taper, N_zeros, t.size)
    return t


def dynamic_window(nxSou: int, nxRec, dd: float, nx: int, dd_space: float):
    r = _i32(nxRec)
    a, b, c = _I(), _I(), _I()
    lib().orc_dynamic_window(r.size, int(nxSou), r, dd, nx, dd_space, C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value  # nx_w, x_i, x_f


def solver(iprop: int, *, dPML: int, fs: int, nxSou, nySou, nxRec, nyRec, S, dmodel: float, dt: float,
           vp, store_snap: int, nt_snap: int, nt: int, Fields=None, disk_mode: int = 0,
           dtype=np.float32):
    """One propagator call in window coordinates (solver_ac_forward_ram /
    solver_ac_backward_ram).  vp: (nx, ny) float32.  Forward (iprop=1)
    returns (Fields, Rec); backward (iprop=2) returns the image (nx, ny)."""
    vp = _f32(vp)
    nx, ny = vp.shape
    nrec = len(np.atleast_1d(nxRec))
    _check_geometry(nxSou, nySou, nxRec, nyRec, nx, ny)
    S = _f32(S).reshape(-1)
    if Fields is None:
        Fields = np.zeros((nt_snap, nx, ny), dtype=dtype)
    Fields = np.ascontiguousarray(Fields, dtype=dtype)
    if iprop == 1:
        out = np.zeros((nrec, nt), dtype=dtype)
    else:
        out = np.zeros((nx, ny), dtype=dtype)
    args = (iprop, disk_mode, dPML, fs, nrec, _i32(nxSou), _i32(nySou), _i32(nxRec), _i32(nyRec))
    if dtype == np.float32:
        lib().orc_solver_f(*args, S, dmodel, dt, ny, nx, vp, store_snap, nt_snap, nt, Fields, out)
    else:
        lib().orc_solver_d(*args, S, S.size, dmodel, dt, ny, nx, vp, store_snap, nt_snap, nt, Fields, out)
    return (Fields, out) if iprop == 1 else out


def forward_dump_p(*, dPML, fs, nxSou, nySou, nxRec, nyRec, S, dmodel, dt, vp, nt, disk_mode=0):
    """Forward propagation for nt steps; returns the padded p (nxt, nyt) after
    the last step (debugging aid for parity failures)."""
    vp = _f32(vp)
    nx, ny = vp.shape
    dn = dPML + 6
    nrec = len(np.atleast_1d(nxRec))
    F = np.zeros((max(nt, 1), nx, ny), dtype=np.float32)
    out = np.zeros((nrec, nt), dtype=np.float32)
    pd = np.zeros((nx + 2 * dn, ny + 2 * dn), dtype=np.float32)
    lib().orc_solver_dump_f(1, disk_mode, dPML, fs, nrec, _i32(nxSou), _i32(nySou), _i32(nxRec), _i32(nyRec),
                            _f32(S).reshape(-1), dmodel, dt, ny, nx, vp, 1, nt, nt, F, out, pd)
    return pd


def _check_geometry(nxSou, nySou, nxRec, nyRec, nx, ny):
    """The restatement indexes its arrays with the geometry as the reference
    does, without checks: refuse a source or receivers outside the grid
    (1-based, nx columns by ny rows) rather than read or write outside the
    arrays."""
    xs, ys = np.atleast_1d(nxSou), np.atleast_1d(nySou)
    xr, yr = np.atleast_1d(nxRec), np.atleast_1d(nyRec)
    if (xs.min() < 1 or xs.max() > nx or ys.min() < 1 or ys.max() > ny or
            (xr.size and (xr.min() < 1 or xr.max() > nx or yr.min() < 1 or yr.max() > ny))):
        raise ValueError(f"source or receivers outside the {nx} x {ny} grid")


def rtm_shot(*, dPML: int, fs: int, nxSou: int, nySou: int, nxRec, nyRec, Data_source, Data_target,
             dd: float, dt: float, nx: int, vp_w, added_space: float, store_snap: int, nt_snap: int,
             nt_prop2: int, nt_taper: int, taper_option: int = 0, N_taper: int = 1, N_zeros: int = 0,
             disk_mode: int = 0, dtype=np.float32, want_synth: bool = False):
    """calculate_PSDM_RTM.f90:395-466 for one shot.  Returns the window image
    (nx_w, ny) and, if asked, the forward receiver traces (NumRec, nt_prop2)."""
    vp_w = _f32(vp_w)
    nx_w, ny = vp_w.shape
    nrec = len(np.atleast_1d(nxRec))
    _check_geometry(nxSou, nySou, nxRec, nyRec, nx, ny)  # model coordinates
    img = np.zeros((nx_w, ny), dtype=dtype)
    synth = np.zeros((nrec, nt_prop2), dtype=dtype) if want_synth else None
    fn = lib().orc_rtm_shot_f if dtype == np.float32 else lib().orc_rtm_shot_d
    fn(disk_mode, dPML, fs, nrec, int(nxSou), int(nySou), _i32(nxRec), _i32(nyRec),
       _f32(Data_source).reshape(-1), _f32(Data_target).reshape(-1), dd, dt, ny, nx, nx_w, vp_w,
       added_space, store_snap, nt_snap, nt_prop2, nt_taper, taper_option, N_taper, N_zeros, img,
       synth.ctypes.data if synth is not None else None)
    return (img, synth) if want_synth else img


def rtm_shot_mixed(*, dPML: int, fs: int, nxSou: int, nySou: int, nxRec, nyRec, Data_source, Data_target,
                   dd: float, dt: float, nx: int, vp_w, added_space: float, store_snap: int, nt_prop2: int,
                   nt_taper: int, taper_option: int = 0, N_taper: int = 1, N_zeros: int = 0, disk_mode: int = 0,
                   q16: int = 0, kahan: int = 1, dtype=np.float32, want_fields: bool = False):
    """The engine's mixed-precision form for one shot (no reference
    counterpart): snapshots every store_snap steps, imaging at the paired
    backward steps.  float32: emulation of the engine (q16 = 1 binary16,
    2 bfloat16, 0 unrounded; Kahan image if kahan); float64: the FP64 oracle
    of the form (q16 and kahan ignored).  Returns the image (nx_w, ny) and, if
    asked, the snapshots as read back (nsnap, nx_w, ny)."""
    vp_w = _f32(vp_w)
    nx_w, ny = vp_w.shape
    _check_geometry(nxSou, nySou, nxRec, nyRec, nx, ny)  # model coordinates
    nrec = len(np.atleast_1d(nxRec))
    nsnap = (nt_prop2 - 1) // store_snap
    img = np.zeros((nx_w, ny), dtype=dtype)
    F = np.zeros((max(nsnap, 1), nx_w, ny), dtype=dtype) if want_fields else None
    args = [disk_mode, dPML, fs, nrec, int(nxSou), int(nySou), _i32(nxRec), _i32(nyRec),
            _f32(Data_source).reshape(-1), _f32(Data_target).reshape(-1), dd, dt, ny, nx, nx_w, vp_w,
            added_space, store_snap, nt_prop2, nt_taper, taper_option, N_taper, N_zeros, img,
            F.ctypes.data if F is not None else None]
    if dtype == np.float32:
        lib().orc_rtm_shot_mixed_f(q16, kahan, *args)
    else:
        lib().orc_rtm_shot_mixed_d(*args)
    return (img, F[:nsnap]) if want_fields else img


def trace_windows(*, cut_multiple, cut_sf, taper_option, T_taper, T_zeros, nxSou, nySou, nxRec, nyRec, Batmodel,
                  dmodel_prop, dt_prop, nt_prop):
    """calculate_PSDM_RTM.f90:231-291: (nt_cut, nt_sf, nt_prop2, nt_taper, N_taper, N_zeros)."""
    nxRec = _i32(nxRec)
    n = nxRec.size
    nt_cut = np.zeros(n, np.int32)
    nt_sf = np.zeros(n, np.int32)
    out = np.zeros(4, np.int32)
    lib().orc_trace_windows(cut_multiple, cut_sf, taper_option, T_taper, T_zeros, n, int(nxSou), int(nySou), nxRec,
                            _i32(nyRec), _f32(Batmodel), dmodel_prop, dt_prop, nt_prop, nt_cut, nt_sf, out)
    return nt_cut, nt_sf, int(out[0]), int(out[1]), int(out[2]), int(out[3])


def akima(y, dx: float, m: int, dt: float) -> np.ndarray:
    """Akima interpolation of y (x_k = k*dx) at t_i = i*dt, i < m."""
    y = _f32(y).reshape(-1)
    out = np.zeros(m, np.float32)
    lib().orc_akima(y, y.size, dx, m, dt, out)
    return out


def condition_traces(*, cut_multiple, cut_sf, taper_option, Field_Data, dt_data, dt_prop, nt_prop2, nt_taper,
                     N_taper, N_zeros, nt_cut, nt_sf) -> np.ndarray:
    """calculate_PSDM_RTM.f90:316-355 (no frequency filter): Data_target as (NumRec, nt_taper)."""
    F = _f32(Field_Data)
    nrec, nt_data = F.shape
    out = np.zeros((nrec, nt_taper), np.float32)
    lib().orc_condition_traces(cut_multiple, cut_sf, taper_option, nrec, F.reshape(-1), nt_data, dt_data, dt_prop,
                               nt_prop2, nt_taper, N_taper, N_zeros, _i32(nt_cut), _i32(nt_sf), out)
    return out


def butterworth_response(ts: int, fe: float, typef: int, f1: float, fc: float) -> np.ndarray:
    """The order-6 Butterworth response H[ts] of filters_function1D
    (filters.f90:50-76) and butterworth (filters.f90:129-232, even order):
    low-pass at fc (typef 1), high-pass from the fixed 40 Hz (2), band-pass
    f1..fc (3).  Evaluated like the reference, in single precision with the
    frequency accumulated by fe/ts per bin, then mirrored Hermitian."""
    f32, c64 = np.float32, np.complex64
    n, pi, fs = 6, f32(3.14159265), f32(40.0)
    f1, fc, fe = f32(f1), f32(fc), f32(fe)
    f0 = np.sqrt(f1 * fc)
    Q = f0 / (fc - f1)
    half = ts // 2 + 1
    freqs = np.zeros(half, f32)
    f = f32(0.0)
    step = fe / f32(ts)
    for j in range(half):  # f = f + fe/ts, accumulated in single precision
        freqs[j] = f
        f = f32(f + step)
    iw = (1j * freqs).astype(c64)
    with np.errstate(divide="ignore", invalid="ignore"):
        if typef == 1:
            s = iw / fc
        elif typef == 2:
            s = fs / iw
        else:
            s = Q * (iw / f0 + f0 / iw)
        Bn = np.ones(half, c64)
        for k in range(1, n // 2 + 1):
            c = np.cos(f32(2 * k + n - 1) * pi / f32(2 * n)).astype(f32)
            Bn = (Bn * (s * s - f32(2.0) * s * c + f32(1.0))).astype(c64)
        H = np.zeros(ts, c64)
        H[:half] = (1.0 / Bn).astype(c64)
    H[0] = 1.0 if typef == 1 else 0.0
    H[half:] = np.conj(H[1:ts - half + 1][::-1])
    return H


def freq_filter(Data_trace, dt: float, typef: int, f1: float, f2: float) -> np.ndarray:
    """freq_filter (auxiliar.f90:498-531) on traces (Num, nt), in float64:
    each trace that is not all zero goes to the end of a zero buffer of
    24*nt samples, is transformed forward with the 1/n scaling of FFTPACK's
    cfft1f, multiplied by the response, transformed back unscaled (cfft1b),
    and the real part of the last nt samples replaces it
    (filters.f90:78-108)."""
    D = np.array(Data_trace, dtype=np.float64, copy=True)
    num, nt = D.shape
    ts = 24 * nt
    H = butterworth_response(ts, 1.0 / np.float32(dt), typef, f1, f2).astype(np.complex128)
    for i in range(num):
        if not np.any(D[i] != 0.0):
            continue
        x = np.zeros(ts, np.float64)
        x[ts - nt:] = D[i]
        y = np.fft.ifft(np.fft.fft(x) / ts * H) * ts
        D[i] = y.real[ts - nt:]
    return D


def nav_read(text: str, cols: int, dir_boat: int, d_shot_model: float, shot_i: int = 0, shot_f: int = 0):
    """read_nav_shot_mcs (get_mcs_data.f90:30-126) on the file's text, in
    single precision: (shotID, pos_shot, pos_bat, line_i, line_f), line_i /
    line_f = 0 when the shot number is not found."""
    f32 = np.float32
    recs = text.split("\n")
    if recs and recs[-1] == "":
        recs = recs[:-1]
    nval = {11: 2, 111: 3, 1111: 4}[cols]
    ids, xs, ys, bat = [], [], [], []
    for r in recs:
        v = r.split("/")[0].replace(",", " ").split()[:nval]
        v = [w.replace("d", "e").replace("D", "e") for w in v]
        ids.append(int(v[0]))
        xs.append(f32(float(v[1])))
        ys.append(f32(float(v[2])) if nval >= 3 else f32(0))
        bat.append(f32(float(v[3])) if nval >= 4 else f32(0))
    n = len(ids)
    o = 0 if dir_boat == 1 else n - 1   # get_mcs_data.f90:68-78
    x1, y1 = xs[o], ys[o]
    si = shot_i or ids[0]
    sf = shot_f or ids[-1]
    line_i = max([k + 1 for k in range(n) if ids[k] == si], default=0)
    line_f = max([k + 1 for k in range(n) if ids[k] == sf], default=0)
    pos = np.array([f32(d_shot_model) + np.sqrt(f32(xs[k] - x1) * f32(xs[k] - x1) + f32(ys[k] - y1) * f32(ys[k] - y1))
                    for k in range(n)], np.float32)
    return np.array(ids, np.int32), pos, np.abs(np.array(bat, np.float32)), line_i, line_f


def channel_positions(pos_shot, nrec, dir_boat, offset_header, offset_unit=1.0, offsets=None, near_offset=0.0,
                      drec=0.0) -> np.ndarray:
    """get_pos_channels (get_mcs_data.f90:418-510) in single precision."""
    f32 = np.float32
    dirf = f32(dir_boat)
    out = np.zeros(nrec, np.float32)
    for i in range(nrec):
        if offset_header == 1:
            a = f32(abs(int(offsets[i])))
            off = a * f32(offset_unit) if offset_unit > 0 else a / f32(abs(offset_unit))
        else:
            off = f32(near_offset) + f32(i) * f32(drec)
        out[i] = f32(pos_shot) - dirf * f32(off)
    return out


def geometry_mcs(pos_shot, pos_rec, shot_depth, streamer_depth, dd):
    """get_geometry_mcs (get_mcs_data.f90:128-148): 1 + floor(position / dd)."""
    f32 = np.float32
    g = lambda v: 1 + int(np.floor(f32(v) / f32(dd)))
    return (g(pos_shot), g(shot_depth), np.array([g(v) for v in pos_rec], np.int32),
            np.full(len(pos_rec), g(streamer_depth), np.int32))


def _linear_1d(x1, y1, x2):
    """linear_interpolation_1D (linear_interpolation.f90:79-117) in single precision."""
    y2 = np.zeros(len(x2), np.float32)
    n1 = len(x1)
    for j, a3 in enumerate(x2):
        if a3 <= x1[0]:
            y2[j] = y1[0]
        elif a3 >= x1[n1 - 1]:
            y2[j] = y1[n1 - 1]
        else:
            for i in range(n1 - 1):
                a1, a2, b1, b2 = x1[i + 1], x1[i], y1[i + 1], y1[i]
                if a2 <= a3 <= a1 and abs(b1) > 0 and abs(b2) > 0:
                    m = np.float32(b1 - b2) / np.float32(a1 - a2)
                    y2[j] = np.float32(b2 + np.float32(np.float32(a3 - a2) * m))
                    break
    return y2


def linear_2d(vel, dmodel, nx_prop, ny_prop, dmodel_prop) -> np.ndarray:
    """linear_2D (linear_interpolation.f90:1-45): vel (nxmodel, nymodel) to (nx_prop, ny_prop)."""
    f32 = np.float32
    vel = np.asarray(vel, np.float32)
    nxm, nym = vel.shape
    xm = np.array([f32(i) * f32(dmodel) for i in range(nxm)], np.float32)
    ym = np.array([f32(i) * f32(dmodel) for i in range(nym)], np.float32)
    xp = np.array([f32(i) * f32(dmodel_prop) for i in range(nx_prop)], np.float32)
    yp = np.array([f32(i) * f32(dmodel_prop) for i in range(ny_prop)], np.float32)
    tmp = np.stack([_linear_1d(ym, vel[i], yp) for i in range(nxm)])           # (nxm, ny_prop)
    out = np.stack([_linear_1d(xm, tmp[:, j], xp) for j in range(ny_prop)], 1)  # (nx_prop, ny_prop)
    return out.astype(np.float32)


def batmodel_from_velocity(Vpmodel, dmodel_prop, water_velocity) -> np.ndarray:
    """00-main.f90:146-158: (j-2) dmodel_prop at the first 1-based row j with V > water_velocity."""
    v = np.asarray(Vpmodel, np.float32)
    out = np.zeros(v.shape[0], np.float32)
    for i in range(v.shape[0]):
        j = np.flatnonzero(v[i] > np.float32(water_velocity))
        if j.size:
            out[i] = np.float32(j[0] - 1) * np.float32(dmodel_prop)
    return out


def _records(text: str, nrec: int, nval: int):
    recs = text.split("\n")
    out = []
    for r in recs[:nrec]:
        v = r.split("/")[0].replace(",", " ").split()[:nval]
        v = [w.replace("d", "e").replace("D", "e") for w in v]
        out.append([int(v[0])] + [np.float32(float(w)) for w in v[1:]])
    return out


def nav_read_was(text: str, cols: int, num_shots: int, d_shot_model, added_space, dmodel, shot_i=0, shot_f=0):
    """read_nav_shot_was (get_was_data.f90:70-125) in single precision."""
    f32 = np.float32
    nval = {11: 2, 111: 3, 1111: 4}[cols]
    rec = _records(text, num_shots, nval)
    xs = [r[1] for r in rec]
    ys = [r[2] if nval >= 3 else f32(0) for r in rec]
    bat = [r[3] if nval >= 4 else f32(0) for r in rec]
    x1, y1 = xs[0], ys[0]
    ids = np.array([r[0] for r in rec], np.int32)
    pos = np.array([f32(d_shot_model) + np.sqrt(f32(xs[k] - x1) * f32(xs[k] - x1) + f32(ys[k] - y1) * f32(ys[k] - y1))
                    for k in range(num_shots)], np.float32)
    li = max([k + 1 for k in range(num_shots) if ids[k] == shot_i], default=0)
    lf = max([k + 1 for k in range(num_shots) if ids[k] == shot_f], default=0)
    xn = xs[-1]
    length = f32(xn + f32(f32(2) * f32(added_space)))
    with np.errstate(divide="ignore", invalid="ignore"):
        dsh = f32(abs(f32(xn - x1)) / f32(num_shots - 1))
    nxm = 1 + int(np.ceil(f32(length / f32(dmodel))))
    return ids, pos, np.abs(np.array(bat, np.float32)), (li, lf, nxm), (float(dsh), float(length))


def nav_read_obs(text: str, num_obs: int, dmodel):
    """read_nav_obs (get_was_data.f90:127-160) in single precision."""
    f32 = np.float32
    rec = _records(text, num_obs, 3)
    px = np.abs(np.array([r[1] for r in rec], np.float32))
    pz = np.abs(np.array([r[2] for r in rec], np.float32))
    g = lambda v: np.array([1 + int(np.ceil(f32(x / f32(dmodel)))) for x in v], np.int32)
    return np.array([r[0] for r in rec], np.int32), px, pz, g(px), g(pz)


def geometry_was(xobs_grid, zobs_grid, pos_shot, shot_depth, dd):
    """get_geometry_WAS (get_was_data.f90:162-189): 1 + ceiling(position / dd) for the shots."""
    f32 = np.float32
    g = lambda v: 1 + int(np.ceil(f32(v) / f32(dd)))
    return (xobs_grid, zobs_grid, np.array([g(v) for v in pos_shot], np.int32),
            np.full(len(pos_shot), g(shot_depth), np.int32))


def akima_nonuniform(x, y, u):
    """Akima's interpolant (J. ACM 17 (1970) 589-602) through (x, y), x
    strictly increasing, at the points u; single precision, in the order the
    engine evaluates it (slopes extended by two per side, node-slope weights
    |m_{i+1}-m_i| and |m_{i-1}-m_{i-2}|, end intervals continued outside)."""
    f32 = np.float32
    x = [f32(v) for v in x]
    y = [f32(v) for v in y]
    n = len(x)
    M = [f32(0)] * (n + 3)
    for i in range(n - 1):
        M[i + 2] = f32(f32(y[i + 1] - y[i]) / f32(x[i + 1] - x[i]))
    if n == 2:
        M[0] = M[1] = M[3] = M[4] = M[2]
    else:
        M[1] = f32(f32(2) * M[2] - M[3])
        M[0] = f32(f32(2) * M[1] - M[2])
        M[n + 1] = f32(f32(2) * M[n] - M[n - 1])
        M[n + 2] = f32(f32(2) * M[n + 1] - M[n])
    t = []
    for i in range(n):
        w1 = f32(abs(f32(M[i + 3] - M[i + 2])))
        w2 = f32(abs(f32(M[i + 1] - M[i])))
        w = f32(w1 + w2)
        t.append(f32(f32(M[i + 1] + M[i + 2]) * f32(0.5)) if w == 0 else
                 f32(f32(f32(w1 * M[i + 1]) + f32(w2 * M[i + 2])) / w))
    out = np.zeros(len(u), np.float32)
    for k, uu in enumerate(u):
        uu = f32(uu)
        if uu == x[-1]:
            out[k] = y[-1]
            continue
        if uu >= x[-1]:
            i = n - 2
        elif uu > x[0]:
            i = max(j for j in range(n - 1) if x[j] <= uu)
        else:
            i = 0
        h = f32(x[i + 1] - x[i])
        d = f32(uu - x[i])
        m, t0, t1 = M[i + 2], t[i], t[i + 1]
        c2 = f32(f32(f32(f32(f32(3) * m) - f32(f32(2) * t0)) - t1) / h)
        c3 = f32(f32(f32(t0 + t1) - f32(f32(2) * m)) / f32(h * h))
        out[k] = f32(y[i] + f32(d * f32(t0 + f32(d * f32(c2 + f32(d * c3))))))
    return out


def bathymetry_nav(pos_shot, pos_bat, length_model, nxmodel, dmodel) -> np.ndarray:
    """get_bathymetry_model_was / _mcs: Akima through (0, first), the shots, (length_model, last)."""
    f32 = np.float32
    x = [f32(0)] + [f32(v) for v in pos_shot] + [f32(length_model)]
    y = [f32(pos_bat[0])] + [f32(v) for v in pos_bat] + [f32(pos_bat[-1])]
    return akima_nonuniform(x, y, [f32(f32(i) * f32(dmodel)) for i in range(nxmodel)])


def relocate_obs(xgrid, bat_model, dmodel):
    """relocation_zOBS (get_was_data.f90:30-68)."""
    f32 = np.float32
    pz = np.array([bat_model[g - 1] for g in xgrid], np.float32)
    return pz, np.array([1 + int(np.ceil(f32(v / f32(dmodel)))) for v in pz], np.int32)


def normalize_psdm(psdm_sum, cov_sum) -> np.ndarray:
    a = _f32(psdm_sum)
    b = _f32(cov_sum)
    out = np.zeros_like(a)
    nx, ny = a.shape
    lib().orc_normalize_psdm(nx, ny, a, b, out)
    return out
