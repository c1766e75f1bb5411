"""Per-shot inputs of a marine (MCS) line or a wide-angle (OBS) line, read
from their files the way the reference prepares them before migrating a shot
(wide-angle: `WasLine`, `load_was`, `was_inputs`, after get_was_data.f90).

At start-up the reference reads the shot navigation (read_nav_shot_mcs,
src/get_mcs_data.f90:30-126) and, for every shot, its channel positions and
grid indices (get_geom_mcs_data -> get_pos_channels, get_geometry_mcs,
:9-28,128-148,418-510); per shot it then reads the SU gather with the
optional delay shift (get_shot_data, :150-214; calculate_PSDM_RTM.f90:
204-220).  `McsLine` holds the parfile values these routines read, and
`load_line` / `shot_inputs` return the same arrays through the library's C
ABI (psdm_nav_read, psdm_su_read_header_i32, psdm_channel_positions,
psdm_geometry_mcs, psdm_su_read_shot).  Everything here runs on the host;
the migration of the shot (Engine.rtm_shot) is the GPU step that follows.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import rtm


@dataclass
class McsLine:
    """Parfile values of an MCS line (src/modules.f90 names in comments)."""
    nav_path: str                      # folder_input_mcs // nav_shot_mcs
    su_paths: List[str]                # one SU file per navigation record (shot gather)
    num_rec: int                       # NumRec_MCS
    ns_max: int                        # nt_mcs_max: samples per stored trace
    nt: int                            # nt_mcs: samples used
    dt: float                          # dt_mcs
    dd: float                          # dmodel_prop: grid step of the propagation
    cols: int = 1111                   # nav_mcs_cols
    dir_boat: int = 1                  # dir_boat
    d_shot_model: float = 0.0          # d_shot_model
    shot_i: int = 0                    # shot_i (0: first record)
    shot_f: int = 0                    # shot_f (0: last record)
    shot_depth: float = 0.0            # shot_depth_mcs
    streamer_depth: float = 0.0        # streamer_depth
    offset_header: int = 0             # offset_header: 1 reads offsets from the trace headers
    offset_unit: float = 1.0           # offset_unit
    byte_offset: int = 37              # byte_offset (1-based; the SU 'offset' word)
    near_offset: float = 0.0           # near_offset (offset_header = 0)
    drec: float = 0.0                  # drec (offset_header = 0)
    delay_time: float = 0.0            # delay_time_data
    big_endian: bool = False           # endianness_data


@dataclass
class LineGeometry:
    shot_id: np.ndarray
    pos_shot: np.ndarray
    pos_bat: np.ndarray
    line_i: int
    line_f: int
    pos_rec: List[np.ndarray] = field(default_factory=list)
    nxSou: List[int] = field(default_factory=list)
    nySou: List[int] = field(default_factory=list)
    nxRec: List[np.ndarray] = field(default_factory=list)
    nyRec: List[np.ndarray] = field(default_factory=list)


def load_line(cfg: McsLine, shots: Optional[List[int]] = None) -> LineGeometry:
    """Navigation of the line and the geometry of its shots (1-based record
    numbers `shots`; default line_i..line_f)."""
    ids, pos, bat, li, lf = rtm.nav_read(cfg.nav_path, cfg.cols, cfg.dir_boat, cfg.d_shot_model, cfg.shot_i,
                                         cfg.shot_f)
    g = LineGeometry(ids, pos, bat, li, lf)
    for icount in (shots if shots is not None else range(li, lf + 1)):
        offsets = None
        if cfg.offset_header == 1:
            offsets = rtm.su_read_header_i32(cfg.su_paths[icount - 1], cfg.num_rec, cfg.ns_max, cfg.byte_offset,
                                             cfg.big_endian)
        pr = rtm.channel_positions(float(pos[icount - 1]), cfg.num_rec, cfg.dir_boat, cfg.offset_header,
                                   cfg.offset_unit, offsets, cfg.near_offset, cfg.drec)
        nxs, nys, nxr, nyr = rtm.geometry_mcs(float(pos[icount - 1]), pr, cfg.shot_depth, cfg.streamer_depth, cfg.dd)
        g.pos_rec.append(pr)
        g.nxSou.append(nxs)
        g.nySou.append(nys)
        g.nxRec.append(nxr)
        g.nyRec.append(nyr)
    return g


def delay_samples(cfg: McsLine) -> int:
    """id = delay_time_data / dt_mcs, truncated as the integer assignment does
    (get_mcs_data.f90:186)."""
    return int(np.float32(cfg.delay_time) / np.float32(cfg.dt))


def shot_inputs(cfg: McsLine, geom: LineGeometry, k: int, icount: int) -> dict:
    """Field_Data (NumRec, nt) and the geometry of record `icount`, the k-th
    shot loaded by load_line: the raw gather, or the delayed one when
    delay_time_data is not zero (calculate_PSDM_RTM.f90:213-217)."""
    d = delay_samples(cfg)
    raw, delayed = rtm.su_read_shot(cfg.su_paths[icount - 1], cfg.num_rec, cfg.ns_max, cfg.nt, cfg.big_endian, d)
    return dict(shot_id=int(geom.shot_id[icount - 1]), nxSou=geom.nxSou[k], nySou=geom.nySou[k],
                nxRec=geom.nxRec[k], nyRec=geom.nyRec[k], Field_Data=delayed if cfg.delay_time != 0 else raw)


# ---- wide-angle (OBS) data -------------------------------------------------

@dataclass
class WasLine:
    """Parfile values of a wide-angle line: OBS gathers, in which by
    reciprocity the OBSs act as sources and the shots as receivers."""
    nav_shot_path: str                 # folder_input_was // nav_shot_was
    nav_obs_path: str                  # folder_input_was // nav_obs
    su_paths: List[str]                # one SU gather per OBS (su_file_was)
    num_shots: int                     # NumShots_was (= NumRec_WAS)
    num_obs: int                       # NumOBS
    ns_max: int                        # nt_was_max
    nt: int                            # nt_was
    dd: float                          # dmodel_prop
    dmodel: float                      # dmodel: grid of the model and of the OBS indices
    length_model: float                # length_model
    nxmodel: int                       # nxmodel
    cols: int = 1111                   # nav_was_cols
    d_shot_model: float = 0.0          # d_shot_model
    added_space: float = 0.0           # added_space
    shot_i: int = 0
    shot_f: int = 0
    shot_depth: float = 0.0            # shot_depth_was
    big_endian: bool = False


@dataclass
class WasGeometry:
    shot_id: np.ndarray
    pos_shot: np.ndarray
    pos_bat: np.ndarray
    lines: tuple                       # (line_i, line_f, nxmodel_was)
    spacing: tuple                     # (dshots_was, length_model_was)
    obs_id: np.ndarray
    pos_xobs: np.ndarray
    pos_zobs: np.ndarray
    xgrid: np.ndarray
    zgrid: np.ndarray
    bat_model: np.ndarray
    nxSou: List[int] = field(default_factory=list)
    nySou: List[int] = field(default_factory=list)
    nxRec: List[np.ndarray] = field(default_factory=list)
    nyRec: List[np.ndarray] = field(default_factory=list)


def load_was(cfg: WasLine) -> WasGeometry:
    """read_nav_shot_was, read_nav_obs and get_bathymetry_model_was (the last
    only with depths in the navigation, cols 1111; the bathymetry is zero
    otherwise), then per OBS get_geometry_WAS followed by relocation_zOBS
    (src/00-main.f90:62-71,195-204; get_was_data.f90:9-28).  In that order
    the first OBS takes its source row from the navigation depth and the
    others from the relocated one, which this reproduces."""
    ids, pos, bat, lines, spacing = rtm.nav_read_was(cfg.nav_shot_path, cfg.cols, cfg.num_shots, cfg.d_shot_model,
                                                     cfg.added_space, cfg.dmodel, cfg.shot_i, cfg.shot_f)
    oid, px, pz, gx, gz = rtm.nav_read_obs(cfg.nav_obs_path, cfg.num_obs, cfg.dmodel)
    if cfg.cols == 1111:
        bm = rtm.bathymetry_nav(pos, bat, cfg.length_model, cfg.nxmodel, cfg.dmodel)
    else:
        bm = np.zeros(cfg.nxmodel, np.float32)
    g = WasGeometry(ids, pos, bat, lines, spacing, oid, px, pz, gx, gz, bm)
    for i in range(cfg.num_obs):
        nxs, nys, nxr, nyr = rtm.geometry_was(int(g.xgrid[i]), int(g.zgrid[i]), pos, cfg.shot_depth, cfg.dd)
        g.nxSou.append(nxs)
        g.nySou.append(nys)
        g.nxRec.append(nxr)
        g.nyRec.append(nyr)
        g.pos_zobs, g.zgrid = rtm.relocate_obs(g.xgrid, bm, cfg.dmodel)
    return g


def was_inputs(cfg: WasLine, geom: WasGeometry, iobs: int) -> dict:
    """Field_Data (NumShots, nt) and the geometry of OBS `iobs` (1-based),
    read as get_obs_data does (get_was_data.f90:191-227: num_shots traces, no
    delay shift)."""
    raw, _ = rtm.su_read_shot(cfg.su_paths[iobs - 1], cfg.num_shots, cfg.ns_max, cfg.nt, cfg.big_endian, 0)
    k = iobs - 1
    return dict(obs_id=int(geom.obs_id[k]), nxSou=geom.nxSou[k], nySou=geom.nySou[k], nxRec=geom.nxRec[k],
                nyRec=geom.nyRec[k], Field_Data=raw)
