"""Seeded synthetic marine models, acquisition geometry and shot data.

No dataset ships with the reference (its README says test data is
"forthcoming"), so the RTM workloads are built from seeded recipes with the
shapes, sizes and value ranges of the benchmark configurations:

  * config1: 200 x 600 cells at 10 m; 200 m of water at 1500 m/s over five
    layers drawn from U(1800, 3500) m/s with +-30 m smooth relief; Ricker
    15 Hz, dt 1 ms, nt 3000; CPML 40; 4 shots 500 m apart at 8 m depth;
    120-channel streamer at 12.5 m, near offset 100 m, 10 m depth.
  * config2: 1200 x 4000 cells at 6.25 m; water to 1.5 km with a +-200 m
    sinusoidal-plus-random seafloor, then a 1700 -> 4500 m/s gradient with
    5 % Gaussian-random lateral perturbations (300 m correlation); Ricker
    20 Hz, dt 0.5 ms, nt 8000; CPML 50; 200 shots 25 m apart; 480-channel
    6 km streamer at 12.5 m (near offset 100 m).
  * config4: the config-1 recipe widened to 1500 x 12000 cells at 6.25 m;
    1000 shots with windows of 800-2400 cells and records of 4000-10000
    steps drawn from a seed.
  * config5: 3000 x 16000 cells at 5 m; water over a 0.5 1/s gradient with a
    4500 m/s body under a rugose top and 3 % perturbations; Ricker 25 Hz,
    dt 0.4 ms, nt 12000; 2000 shots behind a 960-channel 12 km streamer.

Geometry indices follow get_geometry_mcs (src/get_mcs_data.f90:128-148):
nxSou = 1 + floor(pos_shot/dd), nySou = 1 + floor(shot_depth/dd), and
receivers at pos_shot - dir_boat*(near_offset + (irec-1)*drec)
(get_pos_channels, src/get_mcs_data.f90:488-496).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def _smooth_field(shape, sigma_cells, rng) -> np.ndarray:
    """Unit-variance Gaussian random field with a Gaussian correlation kernel."""
    from scipy.ndimage import gaussian_filter
    f = gaussian_filter(rng.standard_normal(shape), sigma=sigma_cells, mode="wrap")
    return f / max(f.std(), 1e-12)


def smooth_model(vel: np.ndarray, sigma_m: float, dd: float) -> np.ndarray:
    """Migration model: the true model smoothed by a Gaussian of sigma_m metres."""
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(vel.astype(np.float64), sigma=sigma_m / dd, mode="nearest").astype(np.float32)


def config1_model(seed: int = 0, ny: int = 200, nx: int = 600, dd: float = 10.0, dip: float = 0.02) -> np.ndarray:
    """Layered model of config 1; shape (nx, ny) (column-major (ny, nx)).
    Layer k dips by k * dip (m per m) about the model's centre."""
    rng = np.random.default_rng(seed)
    z = (np.arange(ny) + 0.5) * dd
    x = np.arange(nx) * dd
    vel = np.full((nx, ny), 1500.0)
    vels = np.sort(rng.uniform(1800.0, 3500.0, size=5))
    tops = np.linspace(200.0, ny * dd * 0.85, 6)[:5]
    for k in range(5):
        relief = 30.0 * _smooth_field((nx,), 40, rng)
        relief = np.clip(relief, -30.0, 30.0)
        dip_k = (k * dip) * (x - x.mean())  # flat to gently dipping
        top = tops[k] + relief + dip_k
        vel[z[None, :] >= top[:, None]] = vels[k]
    vel[:, z < 200.0] = 1500.0
    return vel.astype(np.float32)


def config2_model(seed: int = 0, ny: int = 1200, nx: int = 4000, dd: float = 6.25) -> np.ndarray:
    """Deep-water gradient model of config 2; shape (nx, ny)."""
    rng = np.random.default_rng(seed)
    z = (np.arange(ny) + 0.5) * dd
    x = np.arange(nx) * dd
    sea = 1500.0 + 120.0 * np.sin(2 * np.pi * x / 7000.0 + rng.uniform(0, 2 * np.pi))
    sea = sea + 80.0 * _smooth_field((nx,), 600.0 / dd, rng)
    sea = np.clip(sea, 1300.0, 1700.0)
    zmax = ny * dd
    frac = np.clip((z[None, :] - sea[:, None]) / np.maximum(zmax - sea[:, None], 1.0), 0.0, 1.0)
    grad = 1700.0 + (4500.0 - 1700.0) * frac
    pert = 0.05 * _smooth_field((nx, ny), 300.0 / dd, rng)
    vel = grad * (1.0 + pert)
    vel = np.where(z[None, :] < sea[:, None], 1500.0, np.clip(vel, 1600.0, 4500.0))
    return vel.astype(np.float32)


def config4_model(seed: int = 0, ny: int = 1500, nx: int = 12000, dd: float = 6.25) -> np.ndarray:
    """Config 4: the config-1 recipe widened to 1500 x 12000 cells at 6.25 m
    (200 m of water over five layers, +-30 m relief), with dips scaled to
    the 75 km line."""
    return config1_model(seed=seed, ny=ny, nx=nx, dd=dd, dip=0.0015)


def config5_model(seed: int = 0, ny: int = 3000, nx: int = 16000, dd: float = 5.0, water_m: float = 1000.0,
                  x0_m: float = 0.0) -> np.ndarray:
    """Config 5: 1500 m/s water over sediments with a 0.5 1/s velocity
    gradient (from 1700 m/s, capped at 4500 m/s), a seeded irregular
    high-velocity body at 4500 m/s whose top is a random polygon with +-150 m
    rugosity, and 3 % Gaussian-random perturbations.  nx columns starting at
    x0_m (a window of the 80 km line); shape (nx, ny)."""
    rng = np.random.default_rng(seed)
    z = (np.arange(ny) + 0.5) * dd
    x = x0_m + np.arange(nx) * dd
    zs = z[None, :] - water_m
    vel = np.clip(1700.0 + 0.5 * zs, 1700.0, 4500.0) * np.ones((nx, 1))
    pert = 0.03 * _smooth_field((nx, ny), 200.0 / dd, rng)
    vel = vel * (1.0 + pert)
    # high-velocity body: polygon top near 5-6 km depth between 15 and 65 km
    knots_x = np.linspace(15000.0, 65000.0, 26)
    knots_top = 6000.0 - 1000.0 * np.sin(np.linspace(0, np.pi, 26)) + rng.uniform(-150.0, 150.0, 26)
    top = np.interp(x, knots_x, knots_top, left=np.inf, right=np.inf)
    base = 9000.0 + 300.0 * np.sin(x / 7000.0)
    body = (z[None, :] >= top[:, None]) & (z[None, :] <= base[:, None])
    vel = np.where(body, 4500.0, vel)
    vel = np.where(zs < 0.0, 1500.0, np.clip(vel, 1500.0, 4500.0))
    return vel.astype(np.float32)


@dataclass
class Survey:
    """Marine streamer geometry in model coordinates (1-based indices)."""
    dd: float
    nxSou: np.ndarray            # (nshots,)
    nySou: np.ndarray            # (nshots,)
    nxRec: np.ndarray            # (nshots, nrec)
    nyRec: np.ndarray            # (nshots, nrec)
    pos_shot: np.ndarray = field(default=None)
    pos_rec: np.ndarray = field(default=None)

    @property
    def nshots(self) -> int:
        return int(self.nxSou.size)

    @property
    def nrec(self) -> int:
        return int(self.nxRec.shape[1])


def streamer_survey(dd: float, nshots: int, first_shot_m: float, shot_spacing_m: float, nrec: int,
                    drec: float, near_offset: float, shot_depth: float, streamer_depth: float,
                    dir_boat: int = 1) -> Survey:
    pos_shot = first_shot_m + shot_spacing_m * np.arange(nshots)
    pos_rec = pos_shot[:, None] - dir_boat * (near_offset + drec * np.arange(nrec))[None, :]
    nxSou = (1 + np.floor(pos_shot / dd)).astype(np.int32)
    nySou = np.full(nshots, 1 + int(np.floor(shot_depth / dd)), dtype=np.int32)
    nxRec = (1 + np.floor(pos_rec / dd)).astype(np.int32)
    nyRec = np.full((nshots, nrec), 1 + int(np.floor(streamer_depth / dd)), dtype=np.int32)
    return Survey(dd, nxSou, nySou, nxRec, nyRec, pos_shot, pos_rec)


def config4_shots(nshots: int = 1000, seed: int = 4, nx: int = 12000, dd: float = 6.25,
                  added_space: float = 500.0, near_offset: float = 100.0, drec: float = 12.5,
                  shot_depth: float = 8.0, streamer_depth: float = 10.0):
    """Config 4's uneven shot list: per shot a migration window of 800-2400
    cells drawn from a seed (the streamer's span varies with feathering and
    offset, so the channel count follows from the window) and a record of
    4000-10000 steps; shots spread along the line.  Returns a list of dicts
    (nxSou, nySou, nxRec, nyRec, pos_shot, pos_rec, nt)."""
    rng = np.random.default_rng(seed)
    ddx = 1 + int(np.floor(added_space / dd))
    out = []
    widths = rng.integers(800, 2401, size=nshots)
    nts = rng.integers(4000, 10001, size=nshots)
    for i in range(nshots):
        span = int(widths[i]) - 2 * ddx  # cells from the last receiver to the source
        nrec = max(2, 1 + int((span * dd - near_offset) // drec))
        lo = (span + ddx + 2) * dd
        hi = (nx - ddx - 2) * dd
        pos = float(rng.uniform(lo, hi))
        pos_rec = pos - (near_offset + drec * np.arange(nrec))
        nxRec = (1 + np.floor(pos_rec / dd)).astype(np.int32)
        nyRec = np.full(nrec, 1 + int(np.floor(streamer_depth / dd)), np.int32)
        out.append(dict(nxSou=int(1 + np.floor(pos / dd)), nySou=1 + int(np.floor(shot_depth / dd)), nxRec=nxRec,
                        nyRec=nyRec, pos_shot=pos, pos_rec=pos_rec, nt=int(nts[i])))
    return out


def config5_survey(nshots: int = 2000, dd: float = 5.0) -> Survey:
    # 2000 shots 25 m apart behind a 960-channel, 12 km streamer at 12.5 m.
    return streamer_survey(dd, nshots, 13000.0, 25.0, 960, 12.5, 100.0, 8.0, 10.0, dir_boat=1)


def config1_survey() -> Survey:
    # 4 shots 500 m apart; the streamer trails the boat (dir_boat = 1).
    return streamer_survey(10.0, 4, 2300.0, 500.0, 120, 12.5, 100.0, 8.0, 10.0, dir_boat=1)


def config2_survey(nshots: int = 200) -> Survey:
    # 200 shots 25 m apart; first shot leaves room for the 6 km streamer and
    # the 500 m added space inside the 25 km model.
    return streamer_survey(6.25, nshots, 7000.0, 25.0, 480, 12.5, 100.0, 8.0, 10.0, dir_boat=1)


def mute_direct(traces: np.ndarray, offsets_m: np.ndarray, dt: float, v_water: float = 1500.0,
                t_pad: float = 0.15, taper_s: float = 0.05) -> np.ndarray:
    """Top mute removing the direct arrival: zero before offset/v_water + t_pad,
    cosine ramp of taper_s seconds.  traces: (nrec, nt)."""
    nrec, nt = traces.shape
    t = np.arange(nt) * dt
    out = traces.copy()
    for r in range(nrec):
        t0 = abs(offsets_m[r]) / v_water + t_pad
        w = np.clip((t - t0) / taper_s, 0.0, 1.0)
        out[r] *= (0.5 - 0.5 * np.cos(np.pi * w)).astype(np.float32)
    return out
