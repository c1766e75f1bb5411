"""Python face of the RTM engine, mirroring the reference's solver interface.

Names, argument meaning and order follow the Fortran routines they replace
(src/dynamic_window.f90:54-183, src/calculate_PSDM_RTM.f90:395-466), so
a driver written against the reference reads the same.  Everything runs
through the C ABI of libpsdm_rtm.so (include/psdm_rtm.h).

Array layout is the reference's column-major order expressed as C-order numpy
arrays: a model or image (ny, nx) is an array of shape (nx, ny); traces
(nt, NumRec) are shape (NumRec, nt); Fields (ny, nx_w, nt_snap) is shape
(nt_snap, nx_w, ny).  Geometry indices are 1-based model coordinates.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))


@dataclass
class Params:
    """Module globals of mod_parfile read by the solvers, plus the strategy
    switch and the engine precision (PSDM_PREC_*)."""
    dPML: int = 20
    fs: int = 1
    strategy: int = 1
    precision: int = L.PREC_FP32

    def c(self) -> L.Params:
        return L.Params(self.dPML, self.fs, self.strategy, self.precision)


class Engine:
    """One RTM engine bound to a CUDA device (owns device memory)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        L.check(L.lib().psdm_engine_create(device, C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            L.lib().psdm_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        """Queue work on a caller's cudaStream_t (e.g. torch's current stream)."""
        L.check(L.lib().psdm_engine_set_stream(self._h, stream_ptr))

    def set_profiling(self, on: bool):
        L.check(L.lib().psdm_engine_set_profiling(self._h, int(on)))

    def stats(self) -> dict:
        st = L.Stats()
        L.check(L.lib().psdm_engine_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in L.Stats._fields_}

    def reset_stats(self):
        L.check(L.lib().psdm_engine_reset_stats(self._h))

    def device_bytes(self) -> int:
        return int(L.lib().psdm_engine_device_bytes(self._h))

    def trim(self):
        L.check(L.lib().psdm_engine_trim(self._h))

    # ---- reference-named entry points ------------------------------------
    def dynamic_window_solver_forward_ram(self, prm: Params, nxSou, nySou, nxRec, nyRec, Data_source, dd, dt,
                                          ny, nx, nx_w, Vp_w, dd_space, store_snap, nt_snap, nt,
                                          Fields=None, Data_synth=None):
        """src/dynamic_window.f90:54-96.  Fills Fields (nt_snap, nx_w, ny) and
        Data_synth (NumRec, nt) in place if given; returns (Fields, Data_synth)."""
        nxRec = _i32(nxRec)
        nrec = nxRec.size
        Vp_w = _f32(Vp_w)
        assert Vp_w.shape == (nx_w, ny)
        S = _f32(Data_source).reshape(-1)
        assert S.size >= nt
        fptr = synptr = None
        if Fields is not None:
            assert Fields.dtype == np.float32 and Fields.flags.c_contiguous and Fields.size >= nt_snap * nx_w * ny
            fptr = Fields.ctypes.data
        if Data_synth is not None:
            assert Data_synth.dtype == np.float32 and Data_synth.flags.c_contiguous and Data_synth.size >= nrec * nt
            synptr = Data_synth.ctypes.data
        L.check(L.lib().psdm_dynamic_window_solver_forward_ram(
            self._h, C.byref(prm.c()), nrec, _i32(nxSou), _i32(nySou), nxRec, _i32(nyRec), S, dd, dt, ny, nx,
            nx_w, Vp_w, dd_space, store_snap, nt_snap, nt, fptr, synptr))
        return Fields, Data_synth

    def dynamic_window_solver_backward_ram(self, prm: Params, nxSou, nySou, nxRec, nyRec, AdjSource, dd, dt,
                                           ny, nx, nx_w, Vp_w, dd_space, store_snap, nt_snap, nt, Fields,
                                           PSDM_thread):
        """src/dynamic_window.f90:143-183.  PSDM_thread (nx_w, ny) is updated in place."""
        nxRec = _i32(nxRec)
        adj = _f32(AdjSource)
        assert adj.size >= nxRec.size * nt
        assert PSDM_thread.dtype == np.float32 and PSDM_thread.flags.c_contiguous
        F = _f32(Fields) if Fields is not None else None
        L.check(L.lib().psdm_dynamic_window_solver_backward_ram(
            self._h, C.byref(prm.c()), nxRec.size, _i32(nxSou), _i32(nySou), nxRec, _i32(nyRec), adj.reshape(-1),
            dd, dt, ny, nx, nx_w, _f32(Vp_w), dd_space, store_snap, nt_snap, nt,
            F.ctypes.data if F is not None else None, PSDM_thread))
        return PSDM_thread

    def rtm_shot(self, prm: Params, nxSou: int, nySou: int, nxRec, nyRec, Data_source, Data_target, dd, dt, ny,
                 nx, nx_w, Vp_w, added_space, store_snap, nt_snap, nt_prop2, nt_taper, taper_option=0, N_taper=1,
                 N_zeros=0, PSDM_w=None):
        """src/calculate_PSDM_RTM.f90:395-466 for one shot; returns PSDM_w (nx_w, ny)."""
        nxRec = _i32(nxRec)
        if PSDM_w is None:
            PSDM_w = np.zeros((nx_w, ny), dtype=np.float32)
        tgt = _f32(Data_target)
        assert tgt.size == nxRec.size * nt_taper
        L.check(L.lib().psdm_rtm_shot(
            self._h, C.byref(prm.c()), nxRec.size, int(nxSou), int(nySou), nxRec, _i32(nyRec),
            _f32(Data_source).reshape(-1), tgt.reshape(-1), dd, dt, ny, nx, nx_w, _f32(Vp_w), added_space,
            store_snap, nt_snap, nt_prop2, nt_taper, taper_option, N_taper, N_zeros, PSDM_w))
        return PSDM_w

    def rtm_shot_device(self, prm: Params, nxSou: int, nySou: int, nxRec, nyRec, d_Data_source: int,
                        d_Data_target: int, dd, dt, ny, nx, nx_w, d_Vp_w: int, added_space, store_snap, nt_snap,
                        nt_prop2, nt_taper, taper_option, N_taper, N_zeros, d_PSDM_w: int):
        """psdm_rtm_shot_device: d_* are device pointers (ints); asynchronous."""
        nxRec = _i32(nxRec)
        L.check(L.lib().psdm_rtm_shot_device(
            self._h, C.byref(prm.c()), nxRec.size, int(nxSou), int(nySou), nxRec, _i32(nyRec), d_Data_source,
            d_Data_target, dd, dt, ny, nx, nx_w, d_Vp_w, added_space, store_snap, nt_snap, nt_prop2, nt_taper,
            taper_option, N_taper, N_zeros, d_PSDM_w))

    def rtm_batch(self, prm: Params, shots, Data_source, dd, dt, ny, nx, added_space, store_snap=1,
                  taper_option=0, N_taper=1, N_zeros=0, max_slots=0):
        """psdm_rtm_batch over host arrays.  `shots` is a list of dicts with keys
        nxSou, nySou, nxRec, nyRec, nx_w, nt_prop2, nt_taper, Vp_w (nx_w, ny),
        Data_target (NumRec, nt_taper); returns the window images (nx_w, ny)."""
        keep, descs, outs = [], [], []
        for sh in shots:
            nxr, nyr = _i32(sh["nxRec"]), _i32(sh["nyRec"])
            vp, tgt = _f32(sh["Vp_w"]), _f32(sh["Data_target"])
            nx_w = int(sh["nx_w"])
            assert vp.shape == (nx_w, ny) and tgt.size == nxr.size * int(sh["nt_taper"])
            out = np.zeros((nx_w, ny), dtype=np.float32)
            keep += [nxr, nyr, vp, tgt]
            outs.append(out)
            descs.append(L.Shot(nxr.size, int(sh["nxSou"]), int(sh["nySou"]), nxr.ctypes.data, nyr.ctypes.data,
                                nx_w, int(sh["nt_prop2"]), int(sh["nt_taper"]), vp.ctypes.data, tgt.ctypes.data,
                                out.ctypes.data))
        arr = (L.Shot * max(len(descs), 1))(*descs)
        L.check(L.lib().psdm_rtm_batch(self._h, C.byref(prm.c()), len(descs), arr, _f32(Data_source).reshape(-1),
                                       dd, dt, ny, nx, added_space, store_snap, taper_option, N_taper, N_zeros,
                                       max_slots))
        return outs

    def rtm_batch_device(self, prm: Params, shots, d_Data_source: int, dd, dt, ny, nx, added_space, store_snap=1,
                         taper_option=0, N_taper=1, N_zeros=0, max_slots=0):
        """psdm_rtm_batch_device: each shot dict carries device pointers (ints)
        d_Vp_w, d_Data_target, d_PSDM_w besides its geometry."""
        keep, descs = [], []
        for sh in shots:
            nxr, nyr = _i32(sh["nxRec"]), _i32(sh["nyRec"])
            keep += [nxr, nyr]
            descs.append(L.Shot(nxr.size, int(sh["nxSou"]), int(sh["nySou"]), nxr.ctypes.data, nyr.ctypes.data,
                                int(sh["nx_w"]), int(sh["nt_prop2"]), int(sh["nt_taper"]), int(sh["d_Vp_w"]),
                                int(sh["d_Data_target"]), int(sh["d_PSDM_w"])))
        arr = (L.Shot * max(len(descs), 1))(*descs)
        L.check(L.lib().psdm_rtm_batch_device(self._h, C.byref(prm.c()), len(descs), arr, int(d_Data_source), dd,
                                              dt, ny, nx, added_space, store_snap, taper_option, N_taper, N_zeros,
                                              max_slots))

    def condition_traces(self, cond, Field_Data, dt_data, dt_prop, nt_cut, nt_sf, lens):
        """psdm_condition_traces: Data_target (NumRec, nt_taper) from Field_Data (NumRec, nt_data)."""
        F = _f32(Field_Data)
        nrec, nt_data = F.shape
        out = np.zeros((nrec, int(lens[1])), dtype=np.float32)
        L.check(L.lib().psdm_condition_traces(self._h, C.byref(cond), nrec, F.reshape(-1), nt_data, dt_data, dt_prop,
                                              _i32(nt_cut), _i32(nt_sf), _i32(lens), out))
        return out

    def condition_traces_device(self, cond, nrec, d_Field_Data: int, nt_data, dt_data, dt_prop, nt_cut, nt_sf, lens,
                                d_Data_target: int):
        """psdm_condition_traces_device (device pointers; asynchronous)."""
        L.check(L.lib().psdm_condition_traces_device(self._h, C.byref(cond), nrec, d_Field_Data, nt_data, dt_data,
                                                     dt_prop, _i32(nt_cut), _i32(nt_sf), _i32(lens), d_Data_target))

    def freq_filter(self, traces, dt, typef, f1, f2):
        """psdm_freq_filter on a copy of traces (Num, nt); returns the filtered traces."""
        out = np.array(_f32(traces), dtype=np.float32, copy=True, order="C")
        num, nt = out.shape
        L.check(L.lib().psdm_freq_filter(self._h, out.reshape(-1), nt, dt, num, typef, f1, f2))
        return out

    def freq_filter_device(self, d_traces: int, nt: int, dt: float, num: int, typef: int, f1: float, f2: float):
        """psdm_freq_filter_device: filters device traces (num, nt) in place (asynchronous)."""
        L.check(L.lib().psdm_freq_filter_device(self._h, d_traces, nt, dt, num, typef, f1, f2))

    def set_pass_launch(self, on):
        """psdm_engine_set_pass_launch: one launch per step (0 / False), one cooperative launch per pass
        with tiles (1 / True) or with regions resident in shared memory (2)."""
        L.check(L.lib().psdm_engine_set_pass_launch(self._h, int(on)))

    def set_steps_per_launch(self, steps: int):
        """psdm_engine_set_steps_per_launch: 2 (default) time steps per kernel launch, or 1."""
        L.check(L.lib().psdm_engine_set_steps_per_launch(self._h, int(steps)))

    def autotune(self, prm: Params, ny: int, nx_w: int, nt_prop2: int, nt_taper: int, store_snap: int, nrec: int,
                 budget_bytes: int = 0, max_slots: int = 0, probe: bool = True) -> dict:
        """psdm_engine_autotune: plan against the budget (0 = free device memory), probe the launch form, apply."""
        p = L.Plan()
        L.check(L.lib().psdm_engine_autotune(self._h, C.byref(prm.c()), ny, nx_w, nt_prop2, nt_taper, store_snap,
                                             nrec, int(budget_bytes), max_slots, int(bool(probe)), C.byref(p)))
        return _plan_dict(p)

    def set_reconstruction(self, on: bool):
        """psdm_engine_set_reconstruction: rebuild the source wavefield from a saved band (FP32, store_snap 1)."""
        L.check(L.lib().psdm_engine_set_reconstruction(self._h, int(bool(on))))

    def set_checkpointing(self, interval: int):
        """psdm_engine_set_checkpointing: K > 0 keeps states every K steps instead of all snapshots."""
        L.check(L.lib().psdm_engine_set_checkpointing(self._h, int(interval)))

    def check_wait_timeout(self):
        """psdm_engine_check_wait_timeout: raises PsdmError when the failure path works."""
        L.check(L.lib().psdm_engine_check_wait_timeout(self._h))

    def dt_quotients(self, dt: float, x):
        """psdm_engine_dt_quotients: (the interior tiles' x / dt, the general form's x / dt), float32."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        q = np.zeros(2 * x.size, dtype=np.float32)
        L.check(L.lib().psdm_engine_dt_quotients(self._h, float(dt), x, int(x.size), q))
        return q[:x.size], q[x.size:]

    def batch_slots(self) -> int:
        return int(L.lib().psdm_engine_batch_slots(self._h))

    def model_shot(self, prm: Params, nxSou: int, nySou: int, nxRec, nyRec, Data_source, dd, dt, ny, nx, nx_w,
                   Vp_w, dd_space, nt):
        """Forward modelling (Rec_point of solver_ac_forward_ram); returns (NumRec, nt)."""
        nxRec = _i32(nxRec)
        out = np.zeros((nxRec.size, nt), dtype=np.float32)
        L.check(L.lib().psdm_model_shot(
            self._h, C.byref(prm.c()), nxRec.size, int(nxSou), int(nySou), nxRec, _i32(nyRec),
            _f32(Data_source).reshape(-1), dd, dt, ny, nx, nx_w, _f32(Vp_w), dd_space, nt, out))
        return out


def _plan_dict(p) -> dict:
    return {"steps_per_launch": p.steps_per_launch, "slots": p.slots, "checkpoint_interval": p.checkpoint_interval,
            "fits": bool(p.fits), "bytes_per_slot": p.bytes_per_slot, "budget_bytes": p.budget_bytes,
            "probe_us": [float(p.probe_us[0]), float(p.probe_us[1])]}


def plan_memory(prm: Params, ny: int, nx_w: int, nt_prop2: int, nt_taper: int, store_snap: int, nrec: int,
                budget_bytes: int, max_slots: int = 0) -> dict:
    """psdm_plan_memory: slots and checkpoint interval against an HBM budget (host arithmetic only)."""
    p = L.Plan()
    L.check(L.lib().psdm_plan_memory(C.byref(prm.c()), ny, nx_w, nt_prop2, nt_taper, store_snap, nrec,
                                     int(budget_bytes), max_slots, C.byref(p)))
    return _plan_dict(p)


def rtm_shot_fp64(device: int, prm: Params, nxSou: int, nySou: int, nxRec, nyRec, Data_source, Data_target, dd, dt,
                  ny, nx, nx_w, Vp_w, added_space, store_snap, nt_prop2, nt_taper, taper_option=0, N_taper=1,
                  N_zeros=0, want_fields=False):
    """psdm_rtm_shot_fp64: the FP64 build of one shot on `device` (the error
    reference of the FP32 and mixed forms).  Returns the image (nx_w, ny)
    float64 and, if asked, the snapshots (nsnap, nx_w, ny) float64."""
    nxRec = _i32(nxRec)
    img = np.zeros((nx_w, ny), dtype=np.float64)
    nsnap = (nt_prop2 - 1) // store_snap
    F = np.zeros((max(nsnap, 1), nx_w, ny), dtype=np.float64) if want_fields else None
    L.check(L.lib().psdm_rtm_shot_fp64(
        device, C.byref(prm.c()), nxRec.size, int(nxSou), int(nySou), nxRec, _i32(nyRec),
        _f32(Data_source).reshape(-1), _f32(Data_target).reshape(-1), dd, dt, ny, nx, nx_w, _f32(Vp_w), added_space,
        store_snap, nt_prop2, nt_taper, taper_option, N_taper, N_zeros, img,
        F.ctypes.data if F is not None else None))
    return (img, F[:nsnap]) if want_fields else img


# ---- host helpers (reference set-up arithmetic, run in the library) --------

def fd_coef(num: int, acc: int = 3) -> np.ndarray:
    c = np.zeros(acc + 1, dtype=np.float32)
    L.lib().psdm_fd_coef(num, acc, c)
    return c


def pml_coeffs(dPML: int, dt: float, d: float, acc: int = 3, corners: bool = False):
    dn = dPML + 2 * acc
    fA = np.zeros(dn, dtype=np.float32)
    fB = np.zeros(dn, dtype=np.float32)
    cm = np.zeros(8 * dn * dn, dtype=np.float32) if corners else None
    L.lib().psdm_pml_coeffs(acc, dPML, dt, d, dn, fA, fB, cm.ctypes.data if cm is not None else None)
    if not corners:
        return fA, fB
    c = cm.reshape(8, dn, dn)
    names = ["ldA", "rdA", "luA", "ruA", "ldB", "rdB", "luB", "ruB"]
    return fA, fB, {n: c[q] for q, n in enumerate(names)}


def ricker_mcs(nt: int, dt: float, f0: float, t0: float = 0.0) -> np.ndarray:
    s = np.zeros(nt, dtype=np.float32)
    L.lib().psdm_ricker_mcs(nt, dt, f0, t0, s)
    return s


def dynamic_window(nxSou: int, nxRec, dd: float, nx: int, dd_space: float):
    """Returns (nx_w, x_i, x_f) (src/dynamic_window.f90:1-52)."""
    r = _i32(nxRec)
    a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
    L.lib().psdm_dynamic_window(r.size, int(nxSou), r, dd, nx, dd_space, C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


def taper_pad_trace(trace, nt_prop: int, N_taper: int, N_zeros: int) -> np.ndarray:
    t = _f32(trace).copy()
    L.lib().psdm_taper_pad_trace(t, nt_prop, N_taper, N_zeros, t.size)
    return t


def optimization_dt(dmodel_prop: float, vmax: float, tfin: float, store_snap: int = 1):
    """Returns (dt_prop, nt_prop, nt_snap) (src/optimization.f90:24-32)."""
    dt, ntp, nts = C.c_float(), C.c_int32(), C.c_int32()
    L.lib().psdm_optimization_dt(dmodel_prop, vmax, tfin, store_snap, C.byref(dt), C.byref(ntp), C.byref(nts))
    return dt.value, ntp.value, nts.value


def trace_windows(cond, nxSou, nySou, nxRec, nyRec, Batmodel, dmodel_prop, dt_prop, nt_prop):
    """psdm_trace_windows: (nt_cut, nt_sf, lens = [nt_prop2, nt_taper, N_taper, N_zeros])."""
    nxRec = _i32(nxRec)
    n = nxRec.size
    nt_cut = np.zeros(n, np.int32)
    nt_sf = np.zeros(n, np.int32)
    lens = np.zeros(4, np.int32)
    L.lib().psdm_trace_windows(C.byref(cond), n, int(nxSou), int(nySou), nxRec, _i32(nyRec), _f32(Batmodel),
                               dmodel_prop, dt_prop, nt_prop, nt_cut, nt_sf, lens)
    return nt_cut, nt_sf, lens


def su_write_image(path: str, model, di: float, dj: float, trid: int = 200, big_endian: bool = False):
    """psdm_su_write_image: model (ni, nj) in C order (the reference's (nj, ni)) as ni SU traces."""
    m = _f32(model)
    ni, nj = m.shape
    L.check(L.lib().psdm_su_write_image(str(path).encode(), ni, nj, di, dj, trid, m.reshape(-1), int(big_endian)))


def su_read_shot(path: str, nrec: int, ns_max: int, nt: int, big_endian: bool = False, delay_samples: int = 0):
    """psdm_su_read_shot: (raw, delayed), each (nrec, nt)."""
    raw = np.zeros((nrec, nt), np.float32)
    delayed = np.zeros((nrec, nt), np.float32)
    L.check(L.lib().psdm_su_read_shot(str(path).encode(), nrec, ns_max, nt, int(big_endian), delay_samples, raw,
                                      delayed.ctypes.data))
    return raw, delayed


def su_read_header_i32(path: str, nrec: int, ns_max: int, byte_pos: int, big_endian: bool = False):
    """psdm_su_read_header_i32: the int32 word at 1-based byte byte_pos of each trace."""
    out = np.zeros(nrec, np.int32)
    L.check(L.lib().psdm_su_read_header_i32(str(path).encode(), nrec, ns_max, byte_pos, int(big_endian), out))
    return out


def butterworth_response(ts: int, fe: float, typef: int, f1: float, f2: float) -> np.ndarray:
    """psdm_butterworth_response: the frequency filter's response H (ts,) complex64."""
    out = np.zeros(2 * ts, np.float32)
    L.check(L.lib().psdm_butterworth_response(ts, fe, typef, f1, f2, out))
    return out.view(np.complex64)


def nav_read(path: str, cols: int, dir_boat: int, d_shot_model: float, shot_i: int = 0, shot_f: int = 0):
    """psdm_nav_read: (shotID, pos_shot, pos_bat, line_i, line_f) of a shot navigation file."""
    out = np.zeros(3, np.int32)
    L.lib().psdm_nav_read(str(path).encode(), cols, dir_boat, d_shot_model, shot_i, shot_f, 0, None, None, None,
                          out)
    n = int(out[0])
    if n <= 0:
        L.check(L.lib().psdm_nav_read(str(path).encode(), cols, dir_boat, d_shot_model, shot_i, shot_f, 0, None,
                                      None, None, out))
    ids = np.zeros(n, np.int32)
    pos = np.zeros(n, np.float32)
    bat = np.zeros(n, np.float32)
    L.check(L.lib().psdm_nav_read(str(path).encode(), cols, dir_boat, d_shot_model, shot_i, shot_f, n,
                                  ids.ctypes.data, pos.ctypes.data, bat.ctypes.data, out))
    return ids, pos, bat, int(out[1]), int(out[2])


def channel_positions(pos_shot: float, nrec: int, dir_boat: int, offset_header: int, offset_unit: float = 1.0,
                      offsets=None, near_offset: float = 0.0, drec: float = 0.0):
    """psdm_channel_positions: pos_rec (nrec,) of one shot."""
    out = np.zeros(nrec, np.float32)
    off = None if offsets is None else _i32(offsets)
    L.check(L.lib().psdm_channel_positions(pos_shot, nrec, dir_boat, offset_header, offset_unit,
                                           None if off is None else off.ctypes.data, near_offset, drec, out))
    return out


def geometry_mcs(pos_shot: float, pos_rec, shot_depth: float, streamer_depth: float, dd: float):
    """psdm_geometry_mcs: (nxSou, nySou, nxRec, nyRec), 1-based grid indices."""
    pr = _f32(pos_rec).reshape(-1)
    nxs, nys = C.c_int32(), C.c_int32()
    nxr = np.zeros(pr.size, np.int32)
    nyr = np.zeros(pr.size, np.int32)
    L.check(L.lib().psdm_geometry_mcs(pos_shot, pr.size, pr, shot_depth, streamer_depth, dd, C.byref(nxs),
                                      C.byref(nys), nxr, nyr))
    return nxs.value, nys.value, nxr, nyr


def linear_2d(vel, dmodel: float, nx_prop: int, ny_prop: int, dmodel_prop: float) -> np.ndarray:
    """psdm_linear_2d: vel (nxmodel, nymodel) resampled to (nx_prop, ny_prop)."""
    v = _f32(vel)
    nxm, nym = v.shape
    out = np.zeros((nx_prop, ny_prop), np.float32)
    L.check(L.lib().psdm_linear_2d(nxm, nym, dmodel, v.reshape(-1), nx_prop, ny_prop, dmodel_prop,
                                   out.reshape(-1)))
    return out


def batmodel_from_velocity(Vpmodel, dmodel_prop: float, water_velocity: float) -> np.ndarray:
    """psdm_batmodel_from_velocity: sea-floor depth (nx_prop,) from Vpmodel (nx_prop, ny_prop)."""
    v = _f32(Vpmodel)
    nx, ny = v.shape
    out = np.zeros(nx, np.float32)
    L.check(L.lib().psdm_batmodel_from_velocity(nx, ny, dmodel_prop, water_velocity, v.reshape(-1), out))
    return out


def nav_read_was(path: str, cols: int, num_shots: int, d_shot_model: float, added_space: float, dmodel: float,
                 shot_i: int = 0, shot_f: int = 0):
    """psdm_nav_read_was: (shotID, pos_shot, pos_bat, (line_i, line_f, nxmodel_was),
    (dshots_was, length_model_was))."""
    ids = np.zeros(num_shots, np.int32)
    pos = np.zeros(num_shots, np.float32)
    bat = np.zeros(num_shots, np.float32)
    oi = np.zeros(3, np.int32)
    of = np.zeros(2, np.float32)
    L.check(L.lib().psdm_nav_read_was(str(path).encode(), cols, num_shots, d_shot_model, added_space, dmodel,
                                      shot_i, shot_f, ids, pos, bat, oi, of))
    return ids, pos, bat, tuple(int(v) for v in oi), (float(of[0]), float(of[1]))


def nav_read_obs(path: str, num_obs: int, dmodel: float):
    """psdm_nav_read_obs: (obsID, pos_xobs, pos_zobs, xgrid, zgrid)."""
    ids = np.zeros(num_obs, np.int32)
    px = np.zeros(num_obs, np.float32)
    pz = np.zeros(num_obs, np.float32)
    gx = np.zeros(num_obs, np.int32)
    gz = np.zeros(num_obs, np.int32)
    L.check(L.lib().psdm_nav_read_obs(str(path).encode(), num_obs, dmodel, ids, px, pz, gx, gz))
    return ids, px, pz, gx, gz


def geometry_was(xobs_grid: int, zobs_grid: int, pos_shot, shot_depth: float, dd: float):
    """psdm_geometry_was: (nxSou, nySou, nxRec, nyRec)."""
    ps = _f32(pos_shot).reshape(-1)
    nxs, nys = C.c_int32(), C.c_int32()
    nxr = np.zeros(ps.size, np.int32)
    nyr = np.zeros(ps.size, np.int32)
    L.check(L.lib().psdm_geometry_was(xobs_grid, zobs_grid, ps.size, ps, shot_depth, dd, C.byref(nxs), C.byref(nys),
                                      nxr, nyr))
    return nxs.value, nys.value, nxr, nyr


def bathymetry_nav(pos_shot, pos_bat, length_model: float, nxmodel: int, dmodel: float) -> np.ndarray:
    """psdm_bathymetry_nav: sea-floor depth (nxmodel,) along the line."""
    ps, pb = _f32(pos_shot).reshape(-1), _f32(pos_bat).reshape(-1)
    out = np.zeros(nxmodel, np.float32)
    L.check(L.lib().psdm_bathymetry_nav(ps.size, ps, pb, length_model, nxmodel, dmodel, out))
    return out


def relocate_obs(xgrid, bat_model, dmodel: float):
    """psdm_relocate_obs: (pos_zobs, zgrid) of the OBSs moved to the sea floor."""
    gx = _i32(xgrid)
    bm = _f32(bat_model).reshape(-1)
    pz = np.zeros(gx.size, np.float32)
    gz = np.zeros(gx.size, np.int32)
    L.check(L.lib().psdm_relocate_obs(gx.size, gx, bm, bm.size, dmodel, pz, gz))
    return pz, gz


def normalize_psdm(psdm_sum, cov_sum) -> np.ndarray:
    a, b = _f32(psdm_sum), _f32(cov_sum)
    out = np.zeros_like(a)
    nx, ny = a.shape
    L.lib().psdm_normalize_psdm(nx, ny, a, b, out)
    return out
