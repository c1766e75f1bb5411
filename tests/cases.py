"""Small seeded RTM cases shared by the parity tests (oracle-sized: seconds)."""
from __future__ import annotations

import numpy as np


def layered_model(ny: int, nx: int, dd: float, seed: int, water_m: float = 60.0) -> np.ndarray:
    """Water layer over a few layers with seeded velocities; shape (nx, ny)."""
    rng = np.random.default_rng(seed)
    z = (np.arange(ny) + 0.5) * dd
    x = np.arange(nx) * dd
    v = np.full((nx, ny), 1500.0, dtype=np.float64)
    depths = np.sort(rng.uniform(water_m + 2 * dd, ny * dd, size=3))
    vels = np.sort(rng.uniform(1800.0, 3000.0, size=3))
    for d, vv in zip(depths, vels):
        relief = 2 * dd * np.sin(2 * np.pi * x / (nx * dd) * rng.uniform(0.5, 2.0) + rng.uniform(0, 6))
        mask = z[None, :] >= (d + relief)[:, None]
        v[mask] = vv
    v[:, z < water_m] = 1500.0
    return v.astype(np.float32)


def make_case(*, ny=36, nx_model=90, dd=10.0, dt=1e-3, nt=260, dPML=8, fs=0, strategy=1, nrec=24,
              rec_step=2, near=4, sou_x=52, sou_z=3, rec_z=2, added_space=60.0, store_snap=1,
              taper_option=0, N_taper=1, N_zeros=0, seed=0, collide=False, f0=25.0, dir_boat=-1):
    """A one-shot case in model coordinates.  Receivers trail the source
    (dir_boat = -1 puts them at smaller x).  collide=True maps pairs of
    receivers to the same cell to exercise the last-write-wins injection."""
    from oracle import oracle as O
    vel = layered_model(ny, nx_model, dd, seed)
    nxSou = sou_x
    offs = near + rec_step * np.arange(nrec)
    if collide:
        offs = near + rec_step * (np.arange(nrec) // 2)
    nxRec = (nxSou + dir_boat * offs).astype(np.int32)
    nyRec = np.full(nrec, rec_z, dtype=np.int32)
    nx_w, x_i, x_f = O.dynamic_window(nxSou, nxRec, dd, nx_model, added_space)
    vp_w = np.ascontiguousarray(vel[x_i - 1:x_f, :])
    nt_prop2 = nt
    nt_taper = nt + (N_zeros if taper_option else 0)
    src = O.ricker_mcs(nt, dt, f0, 0.0)
    rng = np.random.default_rng(seed + 100)
    # Observed data: a band-limited random gather (the imaging maths does not
    # care where the data came from).
    tgt = rng.standard_normal((nrec, nt_taper)).astype(np.float32)
    k = np.exp(-0.5 * (np.arange(-6, 7) / 2.0) ** 2)
    tgt = np.stack([np.convolve(t, k / k.sum(), mode="same") for t in tgt]).astype(np.float32)
    tgt[:, nt_prop2:] = 0.0
    return dict(ny=ny, nx=nx_model, dd=dd, dt=dt, nt=nt, dPML=dPML, fs=fs, strategy=strategy,
                nxSou=nxSou, nySou=sou_z, nxRec=nxRec, nyRec=nyRec, nx_w=nx_w, x_i=x_i, x_f=x_f, vel=vel,
                vp_w=vp_w, added_space=added_space, store_snap=store_snap, nt_prop2=nt_prop2, nt_taper=nt_taper,
                taper_option=taper_option, N_taper=N_taper, N_zeros=N_zeros, src=src, tgt=tgt)
