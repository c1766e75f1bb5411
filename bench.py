#!/usr/bin/env python
"""RTM throughput benchmark (shots/s) for the B200 engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One step = one RTM shot of the production-size drop-in configuration
(config 2: 1200 x 4000 cells at 6.25 m, window 1200 x 1136, CPML 50, free
surface, dt 0.5 ms, nt 8000, 480 receivers): forward propagation with all
8000 FP32 snapshots kept in HBM (43.6 GB), backward propagation with the
imaging condition, and the window stacked into the full image.  Inputs are
seeded synthetic data (see psdm_b200/synth.py): smoothed migration model,
Ricker source, observed data forward-modelled by the engine on the true model
with the direct arrival muted.

`value` is timed with CUDA events around K shots whose inputs are already in
HBM; `e2e` times K shots through the C-ABI call psdm_rtm_shot with pinned
host buffers (H2D of model + traces and D2H of the image inside the timed
region).  Each shot streams 87 GB of snapshots through HBM, so every timed
step is far larger than L2 (no explicit flush needed).

Under torchrun (N > 1) every rank migrates its own shots (round-robin, as
calculate_PSDM_RTM.f90:168) and the per-round images are summed with one
all-reduce per round (the reference's MPI_ALLREDUCE, :493-494).

--impl reference times the reference's CPU algorithm on the host cores: the
reference is Fortran and cannot be compiled here (no Fortran compiler), so
its step-by-step C++ restatement (oracle/) stands in, one shot per process
as the reference runs one shot per MPI rank.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# ---- workload (config 2) --------------------------------------------------
NY, NX, DD, DT, NT, DPML, F0 = 1200, 4000, 6.25, 5e-4, 8000, 50, 20.0
CPU_SAMPLE_STEPS = 200  # forward and backward steps per CPU shot sample
ADDED_SPACE = 500.0
WORKLOAD = "rtm_config2_1200x4000_dx6.25_nt8000_cpml50_480ch_fp32"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def grid_cells(ny, nx_w, dpml, fs=1):
    dn = dpml + 6
    nyt, nxt = ny + 2 * dn, nx_w + 2 * dn
    rows = nyt - dn if fs else nyt
    return dict(dn=dn, nyt=nyt, nxt=nxt, n_pad=nyt * nxt, n_act=rows * nxt, n_int=ny * nx_w,
                n_xpml=2 * dn * rows, n_zpml=(dn if fs else 2 * dn) * nxt)


def algorithmic_bytes(ny, nx_w, dpml, fs=1):
    """Compulsory bytes of one fused step (per launch), plain FP32:
    16 B per updated cell (read p, read+write p1/p3, read c2), 16 B per PML
    cell per direction (phi in/out, chi read+write), snapshot 4 B per interior
    cell (forward write / backward read) and the image read+write (8 B per
    interior cell, backward)."""
    g = grid_cells(ny, nx_w, dpml, fs)
    base = 16 * g["n_act"] + 16 * (g["n_xpml"] + g["n_zpml"])
    return base + 4 * g["n_int"], base + 12 * g["n_int"], g


def algorithmic_bytes_mixed(ny, nx_w, dpml, fs, ks):
    """Compulsory bytes of one step of the mixed-precision form: the FP32
    propagation's 16 B per updated cell and C-PML bytes, and per interior
    cell every ks steps the staged FP32 snapshot (written, read back) and its
    16-bit copy (forward), or the 16-bit snapshot and the image and
    compensation read-modify-writes (backward)."""
    g = grid_cells(ny, nx_w, dpml, fs)
    base = 16 * g["n_act"] + 16 * (g["n_xpml"] + g["n_zpml"])
    return base + 10 * g["n_int"] / ks, base + 18 * g["n_int"] / ks, g


def profiled_traffic(which: str):
    """DRAM bytes (read + write) per launch of the step kernel from the ncu
    capture summarised in profiles/ (a `traffic_bytes_per_launch:` line), or
    None if there is none."""
    import re
    p = os.path.join(ROOT, "profiles", "step_kernel_config2_ncu_full.md")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        m = re.search(r"traffic_bytes_per_launch:\s*fwd=(\d+)\s+bwd=(\d+)", f.read())
    if not m:
        return None
    return int(m.group(1) if which == "fwd" else m.group(2))


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                smax = float(r[1])
                for n, v in zip(names, r[4:8]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


# ---- CPU arm (oracle restatement) -------------------------------------------

def _cpu_worker(args):
    """One process = one shot sample of the CPU restatement: the first nt_s
    forward and nt_s backward steps of a config-2 shot on the config-2
    migration model window (1200 x 1136 cells)."""
    nt_s, seed = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from psdm_b200 import synth
    sv = synth.config2_survey(4)
    s = seed % sv.nshots
    nx_w, x_i, x_f = O.dynamic_window(int(sv.nxSou[s]), sv.nxRec[s], DD, NX, ADDED_SPACE)
    vp = np.ascontiguousarray(synth.smooth_model(synth_model_cached(), 100.0, DD)[x_i - 1:x_f])
    src = O.ricker_mcs(nt_s, DT, F0)
    tgt = np.random.default_rng(seed).standard_normal((sv.nrec, nt_s)).astype(np.float32)
    t0 = time.perf_counter()
    O.rtm_shot(dPML=DPML, fs=1, nxSou=int(sv.nxSou[s]), nySou=int(sv.nySou[s]), nxRec=sv.nxRec[s],
               nyRec=sv.nyRec[s], Data_source=src, Data_target=tgt, dd=DD, dt=DT, nx=NX, vp_w=vp,
               added_space=ADDED_SPACE, store_snap=1, nt_snap=nt_s, nt_prop2=nt_s, nt_taper=nt_s)
    return time.perf_counter() - t0, nx_w


def cpu_sample(procs: int, nt_s: int):
    """Run `procs` shot samples in parallel; extrapolate to full shots/s."""
    from oracle import oracle as O
    O.build() if not os.path.exists(O._LIB_PATH) else None
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(nt_s, i) for i in range(procs)])
    wall = time.perf_counter() - t0
    per_sample = max(r[0] for r in res)
    per_shot = per_sample * (2 * (NT - 1)) / (2 * (nt_s - 1))
    return {"shots_per_s": procs / per_shot, "sec_per_shot": per_shot, "sample_s": per_sample, "wall_s": wall,
            "nx_w": res[0][1]}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_procs(max_procs: int) -> int:
    n = host_cores()
    try:
        import psutil
        n = min(n, max(1, int(psutil.virtual_memory().available / (1.2 * 2 ** 30))))
    except Exception:
        pass
    return max(1, min(n, max_procs))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    procs = cpu_procs(64)
    nt_s = CPU_SAMPLE_STEPS
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_sample(procs, nt_s)
        if i >= args.warmup:
            vals.append(r)
    v = statistics.median([r["shots_per_s"] for r in vals])
    sample = (f"{procs} processes x one config-2 shot sample each ({nt_s} forward + {nt_s} backward steps on "
              f"the {NY}x{vals[0]['nx_w']} window of the migration model), extrapolated to nt={NT}; "
              f"{host_cores()} host cores")
    line = {"impl": "reference", "metric": "rtm_shots_per_s", "value": v, "unit": "shots/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cpu": "reference algorithm, C++ restatement (oracle/)",
                       "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": v, "unit": "shots/s", "cores": procs, "kind": "port", "sample": sample,
                             "host_cores": host_cores(), "processes": procs},
            "e2e": {"value": v, "unit": "shots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---- GPU arm -----------------------------------------------------------------

# The engine's other forms, timed after the drop-in on the same shots.
# slots = 0 is one shot at a time through psdm_rtm_shot_device, otherwise
# psdm_rtm_batch_device with that many shots in flight; precision 1 / 2 =
# binary16 / bfloat16 snapshots every ks steps; ckpt = checkpoint interval of
# FP32 shots; spl = time steps per kernel launch.
FORMS = [
    dict(name="fp32_two_steps", precision=0, ks=1, slots=0, spl=2),
    dict(name="fp32_resident", precision=0, ks=1, slots=0, pass_form=2),
    dict(name="fp16_ks4", precision=1, ks=4, slots=0),
    dict(name="batch_fp16_ks4", precision=1, ks=4, slots=8),
    dict(name="batch_bf16_ks4", precision=2, ks=4, slots=8),
    dict(name="batch_fp16_ks4_two_steps", precision=1, ks=4, slots=8, spl=2),
    dict(name="batch_fp32", precision=0, ks=1, slots=2),
    dict(name="fp32_checkpoint_k100", precision=0, ks=1, slots=0, ckpt=100),
    dict(name="fp32_reconstruct", precision=0, ks=1, slots=0, recon=True),
]


def time_conditioning(engine, torch, dev, stream, survey, nshot_traces=480):
    """Device time of the trace conditioning of one shot (480 traces of 2 s at
    2 ms resampled to the 0.5 ms propagation step, sea-floor and multiple cuts,
    taper), against the CPU restatement on one core."""
    from psdm_b200 import rtm
    from psdm_b200._lib import Conditioning
    from oracle import oracle as O
    vel = synth_model_cached()
    bat = np.zeros(NX, np.float32)
    for i in range(NX):
        j = np.flatnonzero(vel[i] > 1500.0)
        bat[i] = np.float32(j[0] - 1) * np.float32(DD) if j.size else 0.0
    cond = Conditioning(1, 1, 1, 0.05, 0.2)
    s = 0
    cut, sf, lens = rtm.trace_windows(cond, survey.nxSou[s], survey.nySou[s], survey.nxRec[s], survey.nyRec[s], bat,
                                      DD, DT, NT)
    dt_data = 4 * DT
    nt_data = NT // 4 + 4
    F = np.cumsum(np.random.default_rng(3).standard_normal((len(cut), nt_data)), axis=1).astype(np.float32)
    d_in = torch.from_numpy(F).to(dev)
    d_out = torch.zeros((len(cut), int(lens[1])), dtype=torch.float32, device=dev)
    run = lambda: engine.condition_traces_device(cond, len(cut), d_in.data_ptr(), nt_data, dt_data, DT, cut, sf, lens,
                                                 d_out.data_ptr())
    for _ in range(3):
        run()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    e0.record(stream)
    for _ in range(reps):
        run()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    gpu_ms = e0.elapsed_time(e1) / reps
    t0 = time.perf_counter()
    O.condition_traces(cut_multiple=1, cut_sf=1, taper_option=1, Field_Data=F, dt_data=dt_data, dt_prop=DT,
                       nt_prop2=int(lens[0]), nt_taper=int(lens[1]), N_taper=int(lens[2]), N_zeros=int(lens[3]),
                       nt_cut=cut, nt_sf=sf)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    # the band-pass filter that precedes it (freq_filter, 24x zero-padded FFT per trace)
    d_f = d_in.clone()
    filt = lambda: engine.freq_filter_device(d_f.data_ptr(), nt_data, dt_data, len(cut), 3, 3.0, 40.0)
    for _ in range(3):
        filt()
    torch.cuda.synchronize(dev)
    e0.record(stream)
    for _ in range(reps):
        filt()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    filt_gpu_ms = e0.elapsed_time(e1) / reps
    t0 = time.perf_counter()
    O.freq_filter(F, dt_data, 3, 3.0, 40.0)
    filt_cpu_ms = (time.perf_counter() - t0) * 1e3
    return {"gpu_ms_per_shot": gpu_ms, "cpu_ms_per_shot": cpu_ms, "cpu_cores": 1, "traces": len(cut),
            "samples_in": nt_data, "samples_out": int(lens[1]), "api": "psdm_condition_traces_device",
            "filter_gpu_ms_per_shot": filt_gpu_ms, "filter_cpu_ms_per_shot": filt_cpu_ms,
            "filter_api": "psdm_freq_filter_device"}


_VEL = None


def synth_model_cached():
    global _VEL
    if _VEL is None:
        from psdm_b200 import synth
        _VEL = synth.config2_model(seed=2)
    return _VEL


def time_forms(engine, torch, dev, stream, d_src, items, names, ref_value):
    """Shots/s of each named form on the workload's shots (inputs in HBM)."""
    from psdm_b200 import rtm
    out = {}
    outs = [torch.zeros((it["nx_w"], NY), dtype=torch.float32, device=dev) for it in items]
    for f in FORMS:
        name, precision, ks, slots = f["name"], f["precision"], f["ks"], f["slots"]
        if name not in names:
            continue
        prm = rtm.Params(dPML=DPML, fs=1, strategy=1, precision=precision)
        ckpt = f.get("ckpt", 0)
        n = 2 * slots if slots else 4
        engine.set_checkpointing(ckpt)
        engine.set_reconstruction(f.get("recon", False))
        engine.set_steps_per_launch(f.get("spl", 1))
        engine.set_pass_launch(f.get("pass_form", 0))
        sel = [(items[i % len(items)], outs[i % len(outs)]) for i in range(n)]

        def run(k):
            if slots == 0:
                for it, o in sel[:k]:
                    engine.rtm_shot_device(prm, it["nxSou"], it["nySou"], it["nxRec"], it["nyRec"], d_src.data_ptr(),
                                           it["d_obs"].data_ptr(), DD, DT, NY, NX, it["nx_w"], it["d_vp"].data_ptr(),
                                           ADDED_SPACE, ks, NT, NT, NT, 0, 1, 0, o.data_ptr())
            else:
                descs = [dict(nxSou=it["nxSou"], nySou=it["nySou"], nxRec=it["nxRec"], nyRec=it["nyRec"],
                              nx_w=it["nx_w"], nt_prop2=NT, nt_taper=NT, d_Vp_w=it["d_vp"].data_ptr(),
                              d_Data_target=it["d_obs"].data_ptr(), d_PSDM_w=o.data_ptr()) for it, o in sel[:k]]
                engine.rtm_batch_device(prm, descs, d_src.data_ptr(), DD, DT, NY, NX, ADDED_SPACE, store_snap=ks,
                                        max_slots=slots)

        run(max(slots, 1))  # warm-up: buffers, graphs
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run(n)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        engine.set_checkpointing(0)
        engine.set_reconstruction(False)
        engine.set_steps_per_launch(1)
        engine.set_pass_launch(0)
        v = n / (e0.elapsed_time(e1) / 1e3)
        out[name] = {"shots_per_s": v, "vs_plain": v / ref_value, "shots": n,
                     "slots": engine.batch_slots() if slots else 1, "precision": ["f32", "fp16", "bf16"][precision],
                     "store_snap": ks}
        if ckpt:
            out[name]["checkpoint_interval"] = ckpt
        if f.get("spl", 1) != 1:
            out[name]["steps_per_launch"] = f["spl"]
        if f.get("recon"):
            out[name]["source_wavefield"] = "reconstructed from a saved 3-cell band"
        if f.get("pass_form"):
            out[name]["launch"] = "one cooperative launch per pass, regions resident in shared memory"
    return out


def _shot_rate(torch, dev, stream, run, nshots):
    """Shots/s of run() (warm-up call first), CUDA events on `stream`."""
    run()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    return nshots / (e0.elapsed_time(e1) / 1e3)


def _config_line(name, rate, shots, cells_steps, bytes_per_shot, peak, **extra):
    """A config entry: shots/s, Gcell-updates/s and the achieved HBM rate on
    the algorithmic bytes, against the measured copy bandwidth."""
    gbs = bytes_per_shot * rate / 1e9
    d = {"shots_per_s": rate, "shots": shots, "gcell_upd_per_s": cells_steps * rate / 1e9,
         "achieved_gbs": gbs, "frac_of_peak": gbs / peak}
    d.update(extra)
    return d


def time_config1(engine, torch, dev, stream, peak, with_cpu, mixed=False):
    """Config 1 in full: its 4 shots (200 x 600 at 10 m, CPML 40, nt 3000,
    120 channels), plain FP32 one shot at a time and all 4 in flight; and the
    CPU restatement running the 4 shots in parallel processes.  With mixed,
    also the mixed-precision form on the same shots (binary16 and bfloat16
    snapshots every 4 steps, Kahan image), one at a time and all 4 in flight;
    returned as a second entry."""
    from oracle import oracle as O
    from psdm_b200 import rtm, synth
    ny, nx, dd, dt, nt, dpml, f0 = 200, 600, 10.0, 1e-3, 3000, 40, 15.0
    sv = synth.config1_survey()
    vt = synth.config1_model(seed=1)
    vm = synth.smooth_model(vt, 100.0, dd)
    prm = rtm.Params(dPML=dpml, fs=0, strategy=1)
    src = rtm.ricker_mcs(nt, dt, f0)
    d_src = torch.from_numpy(src).to(dev)
    items = []
    for s in range(sv.nshots):
        nxS, nyS, nxR, nyR = int(sv.nxSou[s]), int(sv.nySou[s]), sv.nxRec[s], sv.nyRec[s]
        nx_w, x_i, x_f = rtm.dynamic_window(nxS, nxR, dd, nx, ADDED_SPACE)
        obs = engine.model_shot(prm, nxS, nyS, nxR, nyR, src, dd, dt, ny, nx, nx_w,
                                np.ascontiguousarray(vt[x_i - 1:x_f]), ADDED_SPACE, nt)
        obs = synth.mute_direct(obs, sv.pos_rec[s] - sv.pos_shot[s], dt)
        vmw = np.ascontiguousarray(vm[x_i - 1:x_f])
        items.append(dict(nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, nx_w=nx_w, vm=vmw, obs=obs,
                          d_vp=torch.from_numpy(vmw).to(dev), d_obs=torch.from_numpy(obs).to(dev),
                          d_img=torch.zeros((nx_w, ny), dtype=torch.float32, device=dev)))

    def one_at_a_time(prm=prm, ks=1):
        for it in items:
            engine.rtm_shot_device(prm, it["nxSou"], it["nySou"], it["nxRec"], it["nyRec"], d_src.data_ptr(),
                                   it["d_obs"].data_ptr(), dd, dt, ny, nx, it["nx_w"], it["d_vp"].data_ptr(),
                                   ADDED_SPACE, ks, nt, nt, nt, 0, 1, 0, it["d_img"].data_ptr())

    def batched(prm=prm, ks=1):
        descs = [dict(nxSou=it["nxSou"], nySou=it["nySou"], nxRec=it["nxRec"], nyRec=it["nyRec"], nx_w=it["nx_w"],
                      nt_prop2=nt, nt_taper=nt, d_Vp_w=it["d_vp"].data_ptr(), d_Data_target=it["d_obs"].data_ptr(),
                      d_PSDM_w=it["d_img"].data_ptr()) for it in items]
        engine.rtm_batch_device(prm, descs, d_src.data_ptr(), dd, dt, ny, nx, ADDED_SPACE, store_snap=ks,
                                max_slots=len(items))

    fb, bb, g = algorithmic_bytes(ny, items[0]["nx_w"], dpml, 0)
    cells = 2 * (nt - 1) * g["n_pad"]
    out = {"workload": "rtm_config1_200x600_dx10_nt3000_cpml40_120ch_fp32_4shots"}
    out["gpu_one_at_a_time"] = _config_line("config1", _shot_rate(torch, dev, stream, one_at_a_time, len(items)),
                                            len(items), cells, (fb + bb) * (nt - 1), peak)
    out["gpu_batched_4"] = _config_line("config1", _shot_rate(torch, dev, stream, batched, len(items)), len(items),
                                        cells, (fb + bb) * (nt - 1), peak)
    engine.set_pass_launch(2)  # each pass one launch, regions resident in shared memory
    try:
        out["gpu_resident_one_at_a_time"] = _config_line(
            "config1", _shot_rate(torch, dev, stream, one_at_a_time, len(items)), len(items), cells,
            (fb + bb) * (nt - 1), peak, launch="one cooperative launch per pass, regions resident in shared memory")
    finally:
        engine.set_pass_launch(0)
    if with_cpu:
        ctx = mp.get_context("spawn")
        t0 = time.perf_counter()
        with ctx.Pool(len(items)) as pool:
            pool.map(_cpu_config1_worker, [(it["nxSou"], it["nySou"], it["nxRec"], it["nyRec"], it["vm"], it["obs"])
                                           for it in items])
        wall = time.perf_counter() - t0
        out["cpu"] = {"shots_per_s": len(items) / wall, "processes": len(items), "host_cores": host_cores(),
                      "kind": "port", "sample": "the 4 shots in full, one process each (includes process start)"}
    if not mixed:
        return out, None
    mx = {"workload": "rtm_config3_config1_shots_fp16_bf16_snapshots_ks4_kahan_image"}
    mb, mbb, _ = algorithmic_bytes_mixed(ny, items[0]["nx_w"], dpml, 0, 4)
    for kind, name in ((1, "fp16"), (2, "bf16")):
        pm = rtm.Params(dPML=dpml, fs=0, strategy=1, precision=kind)
        for form, fn in (("one_at_a_time", one_at_a_time), ("batched_4", batched)):
            r = _shot_rate(torch, dev, stream, lambda: fn(pm, 4), len(items))
            base = out["gpu_" + form]["shots_per_s"]
            mx[f"{name}_ks4_{form}"] = _config_line("config3", r, len(items), cells, (mb + mbb) * (nt - 1), peak,
                                                    vs_plain_fp32=r / base)
    return out, mx


def _cpu_config1_worker(args):
    nxS, nyS, nxR, nyR, vm, obs = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    nt = obs.shape[1]
    src = O.ricker_mcs(nt, 1e-3, 15.0)
    O.rtm_shot(dPML=40, fs=0, nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, Data_source=src, Data_target=obs, dd=10.0,
               dt=1e-3, nx=600, vp_w=vm, added_space=ADDED_SPACE, store_snap=1, nt_snap=nt, nt_prop2=nt, nt_taper=nt)
    return 0


def time_config4(engine, torch, dev, stream, peak, nshots=24):
    """Config 4: a seeded subset of the 1000 uneven shots (windows of 800-2400
    cells, records of 4000-10000 steps) on the 1500 x 12000 model, batched
    with binary16 snapshots every 4 steps (psdm_rtm_batch_device, slots sized
    to the free device memory)."""
    from psdm_b200 import rtm, synth
    ny, nx, dd, dt, dpml, f0 = 1500, 12000, 6.25, 5e-4, 50, 20.0
    shots = synth.config4_shots()[:nshots]
    vt = synth.config4_model(seed=4)
    vm = synth.smooth_model(vt, 100.0, dd)
    ntmax = max(s["nt"] for s in shots)
    src = rtm.ricker_mcs(ntmax, dt, f0)
    d_src = torch.from_numpy(src).to(dev)
    prm32 = rtm.Params(dPML=dpml, fs=1, strategy=1)
    descs, keep, cells, nbytes = [], [], 0, 0.0
    for s in shots:
        nx_w, x_i, x_f = rtm.dynamic_window(s["nxSou"], s["nxRec"], dd, nx, ADDED_SPACE)
        obs = engine.model_shot(prm32, s["nxSou"], s["nySou"], s["nxRec"], s["nyRec"], src[:s["nt"]], dd, dt, ny, nx,
                                nx_w, np.ascontiguousarray(vt[x_i - 1:x_f]), ADDED_SPACE, s["nt"])
        obs = synth.mute_direct(obs, s["pos_rec"] - s["pos_shot"], dt)
        d_vp = torch.from_numpy(np.ascontiguousarray(vm[x_i - 1:x_f])).to(dev)
        d_obs = torch.from_numpy(obs).to(dev)
        d_img = torch.zeros((nx_w, ny), dtype=torch.float32, device=dev)
        keep += [d_vp, d_obs, d_img]
        descs.append(dict(nxSou=s["nxSou"], nySou=s["nySou"], nxRec=s["nxRec"], nyRec=s["nyRec"], nx_w=nx_w,
                          nt_prop2=s["nt"], nt_taper=s["nt"], d_Vp_w=d_vp.data_ptr(), d_Data_target=d_obs.data_ptr(),
                          d_PSDM_w=d_img.data_ptr()))
        fb, bb, g = algorithmic_bytes_mixed(ny, nx_w, dpml, 1, 4)
        cells += 2 * (s["nt"] - 1) * g["n_pad"]
        nbytes += (fb + bb) * (s["nt"] - 1)
    engine.trim()
    prm = rtm.Params(dPML=dpml, fs=1, strategy=1, precision=1)
    run = lambda: engine.rtm_batch_device(prm, descs, d_src.data_ptr(), dd, dt, ny, nx, ADDED_SPACE, store_snap=4,
                                          max_slots=16)
    rate = _shot_rate(torch, dev, stream, run, len(descs))
    widths = [d["nx_w"] for d in descs]
    line = _config_line("config4", rate, len(descs), cells / len(descs), nbytes / len(descs), peak,
                        form="batched, binary16 snapshots every 4 steps", slots=engine.batch_slots(),
                        nx_w_range=[min(widths), max(widths)], nt_range=[min(s["nt"] for s in shots),
                                                                        max(s["nt"] for s in shots)])
    del keep
    engine.trim()
    return {"workload": f"rtm_config4_1500x12000_dx6.25_{len(descs)}_of_1000_uneven_shots", "batch_fp16_ks4": line}


def time_config5(engine, torch, dev, stream, peak):
    """Config 5: one shot of the 3000 x 16000 model at 5 m (dt 0.4 ms, nt
    12000, 960 channels, 12 km streamer): FP32 snapshots (377 GB) do not fit,
    so the forms are binary16 snapshots every 4 steps, FP32 with checkpoints
    every 100 steps, and FP32 with the source wavefield reconstructed from a
    saved band, one shot at a time; and batched binary16 with every snapshot
    and with checkpoints."""
    from psdm_b200 import rtm, synth
    ny, nx, dd, dt, nt, dpml, f0 = 3000, 16000, 5.0, 4e-4, 12000, 50, 25.0
    sv = synth.config5_survey(1)
    nxS, nyS, nxR, nyR = int(sv.nxSou[0]), int(sv.nySou[0]), sv.nxRec[0], sv.nyRec[0]
    nx_w, x_i, x_f = rtm.dynamic_window(nxS, nxR, dd, nx, ADDED_SPACE)
    vt = synth.config5_model(seed=5, nx=x_f)
    vm = synth.smooth_model(vt, 100.0, dd)
    src = rtm.ricker_mcs(nt, dt, f0)
    d_src = torch.from_numpy(src).to(dev)
    prm32 = rtm.Params(dPML=dpml, fs=1, strategy=1)
    engine.trim()
    obs = engine.model_shot(prm32, nxS, nyS, nxR, nyR, src, dd, dt, ny, nx, nx_w,
                            np.ascontiguousarray(vt[x_i - 1:x_f]), ADDED_SPACE, nt)
    obs = synth.mute_direct(obs, sv.pos_rec[0] - sv.pos_shot[0], dt)
    d_vp = torch.from_numpy(np.ascontiguousarray(vm[x_i - 1:x_f])).to(dev)
    d_obs = torch.from_numpy(obs).to(dev)
    d_img = torch.zeros((nx_w, ny), dtype=torch.float32, device=dev)
    out = {"workload": f"rtm_config5_3000x16000_dx5_nt12000_cpml50_960ch_window{nx_w}"}
    for name, precision, ks, ckpt in (("fp16_ks4", 1, 4, 0), ("fp32_checkpoint_k100", 0, 1, 100),
                                      ("fp32_reconstruct", 0, 1, -1)):
        prm = rtm.Params(dPML=dpml, fs=1, strategy=1, precision=precision)
        engine.set_checkpointing(max(ckpt, 0))
        engine.set_reconstruction(ckpt < 0)
        run = lambda: engine.rtm_shot_device(prm, nxS, nyS, nxR, nyR, d_src.data_ptr(), d_obs.data_ptr(), dd, dt, ny,
                                             nx, nx_w, d_vp.data_ptr(), ADDED_SPACE, ks, nt, nt, nt, 0, 1, 0,
                                             d_img.data_ptr())
        try:
            rate = _shot_rate(torch, dev, stream, run, 1)
        finally:
            engine.set_checkpointing(0)
            engine.set_reconstruction(False)
        if precision:
            fb, bb, g = algorithmic_bytes_mixed(ny, nx_w, dpml, 1, ks)
            nbytes = (fb + bb) * (nt - 1)
        elif ckpt > 0:  # the forward pass runs twice
            fb, bb, g = algorithmic_bytes(ny, nx_w, dpml, 1)
            nbytes = (2 * fb + bb) * (nt - 1)
        else:  # forward without snapshot writes; the reverse step reads p, p1, c2 and writes p and a snapshot
            fb, bb, g = algorithmic_bytes(ny, nx_w, dpml, 1)
            nbytes = (fb - 4 * g["n_int"] + bb + 20 * g["n_int"]) * (nt - 1)
        cells = 2 * (nt - 1) * g["n_pad"]
        out[name] = _config_line("config5", rate, 1, cells, nbytes, peak)
        engine.trim()
    out["fp32_all_snapshots"] = {"fits": False, "snapshot_gb": round(4.0 * ny * nx_w * (nt - 1) / 1e9, 1)}
    # Batched binary16 every 4 steps: every snapshot kept (as many shots in
    # flight as fit), and with checkpoints at the planner's interval (more
    # shots in flight, the forward pass twice).  The shots repeat shot 0's
    # geometry and data.
    prm = rtm.Params(dPML=dpml, fs=1, strategy=1, precision=1)
    fb, bb, g = algorithmic_bytes_mixed(ny, nx_w, dpml, 1, 4)
    fb32, _, _ = algorithmic_bytes(ny, nx_w, dpml, 1)
    cells = 2 * (nt - 1) * g["n_pad"]
    engine.trim()
    torch.cuda.synchronize(dev)
    free, _ = torch.cuda.mem_get_info(dev)
    for name, force_ckpt in (("batch_fp16_ks4", False), ("batch_fp16_ks4_checkpoint", True)):
        budget = free if not force_ckpt else min(free, 40 * 10 ** 9)  # 40 GB per shot: below its 47 GB of snapshots
        plan = rtm.plan_memory(prm, ny, nx_w, nt, nt, 4, len(nxR), budget)
        if not plan["fits"]:
            continue
        K = plan["checkpoint_interval"]
        slots = plan["slots"] if not force_ckpt else min(8, int((free - 2 ** 30) // plan["bytes_per_slot"]))
        if slots < 1:
            continue
        descs = [dict(nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, nx_w=nx_w, nt_prop2=nt, nt_taper=nt,
                      d_Vp_w=d_vp.data_ptr(), d_Data_target=d_obs.data_ptr(), d_PSDM_w=d_img.data_ptr())] * slots
        engine.set_checkpointing(K)
        run = lambda: engine.rtm_batch_device(prm, descs, d_src.data_ptr(), dd, dt, ny, nx, ADDED_SPACE, store_snap=4,
                                              max_slots=slots)
        try:
            rate = _shot_rate(torch, dev, stream, run, slots)
        finally:
            engine.set_checkpointing(0)
        nbytes = (fb + bb + (fb32 - 4 * g["n_int"] if K else 0)) * (nt - 1)  # checkpoints: the forward pass twice
        out[name] = _config_line("config5", rate, slots, cells, nbytes, peak, slots=engine.batch_slots(),
                                 checkpoint_interval=K, gb_per_shot=round(plan["bytes_per_slot"] / 1e9, 1))
        engine.trim()
    return out


def build_inputs(engine, torch, dev, shots, survey, vel_true, vel_mig, prm):
    """Device-resident inputs of each shot (model window, source, observed data)."""
    from psdm_b200 import rtm, synth
    src = rtm.ricker_mcs(NT, DT, F0)
    d_src = torch.from_numpy(src).to(dev)
    items = []
    for s in shots:
        nxS, nyS = int(survey.nxSou[s]), int(survey.nySou[s])
        nxR, nyR = survey.nxRec[s], survey.nyRec[s]
        nx_w, x_i, x_f = rtm.dynamic_window(nxS, nxR, DD, NX, ADDED_SPACE)
        vt = np.ascontiguousarray(vel_true[x_i - 1:x_f])
        vm = np.ascontiguousarray(vel_mig[x_i - 1:x_f])
        obs = engine.model_shot(prm, nxS, nyS, nxR, nyR, src, DD, DT, NY, NX, nx_w, vt, ADDED_SPACE, NT)
        obs = synth.mute_direct(obs, survey.pos_rec[s] - survey.pos_shot[s], DT)
        items.append(dict(nxSou=nxS, nySou=nyS, nxRec=nxR, nyRec=nyR, nx_w=nx_w, x_i=x_i, x_f=x_f,
                          vp_h=vm, obs_h=np.ascontiguousarray(obs, dtype=np.float32),
                          d_vp=torch.from_numpy(vm).to(dev), d_obs=torch.from_numpy(obs).to(dev)))
    return d_src, src, items


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from psdm_b200 import driver, rtm, synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    engine = rtm.Engine(local)
    # One non-default stream for torch ops, NCCL and the engine (handle 0
    # would mean "the engine's own stream" to psdm_engine_set_stream).
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    engine.set_stream(stream.cuda_stream)
    prm = rtm.Params(dPML=DPML, fs=1, strategy=1)

    survey = synth.config2_survey(200)
    vel_true = synth_model_cached()
    vel_mig = synth.smooth_model(vel_true, 100.0, DD)
    n_total = args.warmup + args.steps
    # round-robin shots (0-based lines, wrapping over the survey)
    my_shots = [(driver.shot_of(i + 1, world, rank, 1) - 1) % survey.nshots for i in range(n_total)]
    uniq = sorted(set(my_shots))
    d_src, h_src, items_u = build_inputs(engine, torch, dev, uniq, survey, vel_true, vel_mig, prm)
    by_shot = dict(zip(uniq, items_u))
    items = [by_shot[s] for s in my_shots]

    # window images embedded, summed over ranks once per round and stacked
    # (calculate_PSDM_RTM.f90:471-497)
    stack = driver.ImageStack(NY, NX, device=dev)
    d_img = torch.zeros((max(it["nx_w"] for it in items), NY), dtype=torch.float32, device=dev)

    def one_round(it):
        nx_w = it["nx_w"]
        engine.rtm_shot_device(prm, it["nxSou"], it["nySou"], it["nxRec"], it["nyRec"], d_src.data_ptr(),
                               it["d_obs"].data_ptr(), DD, DT, NY, NX, nx_w, it["d_vp"].data_ptr(), ADDED_SPACE, 1,
                               NT, NT, NT, 0, 1, 0, d_img.data_ptr())
        stack.add_round(d_img, it["x_i"], it["x_f"])

    for i in range(args.warmup):
        one_round(items[i])
    torch.cuda.synchronize(dev)
    engine.reset_stats()
    engine.set_profiling(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for i in range(args.warmup, n_total):
            one_round(items[i])
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    st = engine.stats()
    engine.set_profiling(False)
    ms_t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = world * args.steps / (ms_max / 1e3)

    # roofline of the dominant kernel (per-launch time from CUDA events)
    nx_w0 = items[args.warmup]["nx_w"]
    fwd_b, bwd_b, g = algorithmic_bytes(NY, nx_w0, DPML, 1)
    fwd_us = st["fwd_ms"] * 1e3 / max(st["fwd_steps"], 1)
    bwd_us = st["bwd_ms"] * 1e3 / max(st["bwd_steps"], 1)
    dom = "bwd" if st["bwd_ms"] >= st["fwd_ms"] else "fwd"
    peak, peak_kind = _peaks()
    bytes_dom = bwd_b if dom == "bwd" else fwd_b
    us_dom = bwd_us if dom == "bwd" else fwd_us
    achieved = bytes_dom / (us_dom * 1e-6) / 1e9
    traffic = profiled_traffic(dom)

    # end-to-end through the C ABI with pinned host buffers
    e2e = None
    if rank == 0 or world > 1:
        pin = [(torch.from_numpy(it["vp_h"]).pin_memory(), torch.from_numpy(it["obs_h"]).pin_memory(),
                torch.empty((it["nx_w"], NY), dtype=torch.float32).pin_memory()) for it in items[args.warmup:]]
        h_src = torch.from_numpy(h_src).pin_memory()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for it, (vp_p, obs_p, img_p) in zip(items[args.warmup:], pin):
            engine.rtm_shot(prm, it["nxSou"], it["nySou"], it["nxRec"], it["nyRec"], h_src.numpy(), obs_p.numpy(),
                            DD, DT, NY, NX, it["nx_w"], vp_p.numpy(), ADDED_SPACE, 1, NT, NT, NT, 0, 1, 0,
                            PSDM_w=img_p.numpy())
        torch.cuda.synchronize(dev)
        el = torch.tensor([time.perf_counter() - t0], device=dev)
        if world > 1:
            dist.all_reduce(el, op=dist.ReduceOp.MAX)
        it0 = items[args.warmup]
        h2d = 4 * (NY * it0["nx_w"] + NT + it0["obs_h"].size) + 8 * it0["obs_h"].shape[0]
        d2h = 4 * NY * it0["nx_w"]
        e2e = {"value": world * args.steps / float(el.item()), "unit": "shots/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "api": "psdm_rtm_shot (C ABI, pinned host buffers)"}

    forms = None
    names = [f["name"] for f in FORMS] if args.forms == "all" else [n for n in args.forms.split(",") if n and n != "none"]
    if world == 1 and names:
        forms = time_forms(engine, torch, dev, stream, d_src, items_u, names, value)
    configs = None
    cnames = ["config1", "config3", "config4", "config5"] if args.configs == "all" else \
        [n for n in args.configs.split(",") if n and n != "none"]
    if world == 1 and cnames:
        peak_c, _ = _peaks()
        configs = {}
        if "config1" in cnames or "config3" in cnames:
            c1, c3 = time_config1(engine, torch, dev, stream, peak_c, not args.no_cpu and "config1" in cnames,
                                  mixed="config3" in cnames)
            if "config1" in cnames:
                configs["config1"] = c1
            if c3 is not None:
                configs["config3"] = c3
        if "config4" in cnames:
            configs["config4"] = time_config4(engine, torch, dev, stream, peak_c)
        if "config5" in cnames:
            configs["config5"] = time_config5(engine, torch, dev, stream, peak_c)
    conditioning = None
    if rank == 0 and world == 1 and not args.no_cpu:
        conditioning = time_conditioning(engine, torch, dev, stream, survey)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        procs = cpu_procs(32)
        r = cpu_sample(procs, CPU_SAMPLE_STEPS)
        cpu = {"value": r["shots_per_s"], "unit": "shots/s", "cores": procs, "kind": "port",
               "host_cores": host_cores(), "processes": procs,
               "sample": f"{procs} processes x one config-2 shot sample each ({CPU_SAMPLE_STEPS} forward + "
                         f"{CPU_SAMPLE_STEPS} backward steps of the C++ restatement on the migration model), "
                         f"extrapolated to nt={NT}; {r['sec_per_shot']:.0f} s/shot"}

    if rank == 0:
        gcell = world * args.steps * 2 * (NT - 1) * g["n_pad"] / (ms_max / 1e3) / 1e9
        line = {"metric": "rtm_shots_per_s", "value": value, "unit": "shots/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": WORKLOAD, "engine": "plain FP32 drop-in (bit-exact)", "nx_w": nx_w0,
                           "cells_padded": g["n_pad"], "snapshots_gb": round(4 * g["n_int"] * (NT - 1) / 1e9, 1),
                           "l2": "inputs larger than L2 (87 GB of snapshots streamed per step)",
                           "parallelism": f"shots x{world}"},
                "gcell_upd_per_s": gcell,
                "kernel": {"fwd_us_per_step": fwd_us, "bwd_us_per_step": bwd_us, "fwd_bytes": fwd_b,
                           "bwd_bytes": bwd_b},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "kernel": f"step_kernel<{dom}>",
                             "peak_kind": peak_kind},
                "gpu_launches": int(st["launches"]),
                "clocks": clk.summary(),
                "e2e": e2e,
                "forms": forms,
                "configs": configs,
                "conditioning": conditioning,
                "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--forms", default="all",
                    help="other engine forms to time after the drop-in: all, none or a comma list of " +
                         ", ".join(f["name"] for f in FORMS))
    ap.add_argument("--configs", default="all",
                    help="other benchmark configurations to time: all, none or a comma list of config1, config3, "
                         "config4, config5")
    ap.add_argument("--nt", type=int, default=None,
                    help="override the record length (small cases for ncu captures only; not a bench value)")
    args = ap.parse_args()
    if args.nt:
        global NT, WORKLOAD
        NT = args.nt
        WORKLOAD = WORKLOAD.replace("nt8000", f"nt{NT}")
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
