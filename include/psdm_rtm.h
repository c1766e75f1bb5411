/*
 * psdm_rtm.h -- C ABI of the B200 reverse-time-migration (RTM) engine.
 *
 * Drop-in boundary for the RTM propagators of PSDM (ejimeneztejero/PSDM).
 * Every entry point takes plain pointers and sizes; arrays use the
 * reference's Fortran layout (column-major, 1-based geometry indices):
 *   model / image (ny, nx)            -> float[nx][ny]
 *   traces (nt, NumRec)               -> float[NumRec][nt]
 *   snapshots Fields(ny, nx_w, nslot) -> float[nslot][nx_w][ny]
 * The caller owns host buffers; the engine owns device memory.  Calls are
 * synchronous (results are in the caller's buffers on return), return
 * PSDM_OK (0) on success and a negative code on failure, never exit, and
 * leave a message for psdm_last_error().  One engine serves one host thread
 * at a time; separate engines are independent.
 *
 * There is no CPU fallback: an engine on a machine without a usable CUDA
 * device fails at psdm_engine_create with PSDM_ERR_CUDA.
 */
#ifndef PSDM_RTM_H
#define PSDM_RTM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PSDM_OK = 0,
    PSDM_ERR_ARG = -1,   /* invalid argument or geometry outside the padded grid */
    PSDM_ERR_CUDA = -2,  /* CUDA runtime error (no device, launch failure, ...) */
    PSDM_ERR_NOMEM = -3, /* device allocation failed (HBM budget) */
    PSDM_ERR_STATE = -4  /* engine misuse (null engine, ...) */
};

/*
 * Snapshot storage precision of the engine (psdm_params.precision).  The
 * 16-bit forms propagate in FP32, keep an FP32 image with Kahan compensation,
 * and set up their FD coefficients and C-PML profiles in double precision,
 * rounded once to FP32; PSDM_PREC_FP32 keeps the reference's single-precision
 * set-up (src/solver_FD_coeffs.f90, src/solver_PML_coeffs.f90).
 */
enum {
    PSDM_PREC_FP32 = 0,  /* plain FP32: the reference's arithmetic, bit for bit */
    PSDM_PREC_FP16 = 1,  /* FP16 snapshots with per-snapshot power-of-two scale */
    PSDM_PREC_BF16 = 2   /* BF16 snapshots with per-snapshot power-of-two scale */
};

/*
 * Values the reference solvers read from module mod_parfile
 * (src/solver_ac_forward_ram.f90:8 `USE mod_parfile, ONLY: dPML, fs`) and
 * the strategy switch of calculate_PSDM_RTM (src/calculate_PSDM_RTM.f90:395,411,435).
 */
typedef struct psdm_params {
    int32_t dPML;       /* C-PML thickness in cells (parfile `dPML`, default 20) */
    int32_t fs;         /* 0 = absorbing top; otherwise free surface (parfile `free_surface`, default 1) */
    int32_t strategy;   /* 1 = RAM solvers' statement order, 2 = disk solvers' order (strategy_num) */
    int32_t precision;  /* PSDM_PREC_*; the *_ram drop-in entry points require PSDM_PREC_FP32 */
} psdm_params;

typedef struct psdm_engine psdm_engine;

/* Last error message of the calling thread ("" if none). */
const char* psdm_last_error(void);

/* Create an engine bound to CUDA device `device`. */
int psdm_engine_create(int32_t device, psdm_engine** out);
int psdm_engine_destroy(psdm_engine* e);
/* Device bytes currently held by the engine's buffer cache. */
int64_t psdm_engine_device_bytes(const psdm_engine* e);
/* Release the engine's cached device buffers. */
int psdm_engine_trim(psdm_engine* e);
/*
 * Run the engine's work on the caller's CUDA stream (a cudaStream_t passed as
 * void*); NULL restores the engine's own stream.  No reference counterpart:
 * lets a host framework order the engine with its own device work.
 */
int psdm_engine_set_stream(psdm_engine* e, void* stream);

/* Counters of the engine (no reference counterpart; the reference only prints). */
typedef struct psdm_stats {
    int64_t launches;   /* kernels launched by the engine */
    int64_t fwd_steps;  /* forward time steps */
    int64_t bwd_steps;  /* backward time steps */
    int64_t shots;      /* shots timed while profiling was on */
    double fwd_ms;      /* device time of the forward passes of those shots */
    double bwd_ms;      /* device time of the backward passes of those shots */
} psdm_stats;
/* Turn per-shot CUDA-event timing of the forward and backward passes on/off. */
int psdm_engine_set_profiling(psdm_engine* e, int32_t on);
int psdm_engine_stats(psdm_engine* e, psdm_stats* out);
int psdm_engine_reset_stats(psdm_engine* e);

/*
 * Replaces dynamic_window_solver_forward_ram (src/dynamic_window.f90:54-96),
 * which calls solver_ac_forward_ram (src/solver_ac_forward_ram.f90:4-637).
 * Geometry in model coordinates; the window is recomputed from dd_space as
 * the reference does.  Writes Fields(ny, nx_w, nt_snap) (slots
 * 1..(nt-1)/store_snap; other slots untouched) and Data_synth(nt, NumRec).
 * Fields or Data_synth may be NULL to skip that output.
 */
int psdm_dynamic_window_solver_forward_ram(
    psdm_engine* e, const psdm_params* prm, int32_t NumRec,
    const int32_t* nxSou, const int32_t* nySou, const int32_t* nxRec, const int32_t* nyRec,
    const float* Data_source /* nt */, float dd, float dt, int32_t ny, int32_t nx, int32_t nx_w,
    const float* Vp_w /* (ny, nx_w) */, float dd_space, int32_t store_snap, int32_t nt_snap,
    int32_t nt, float* Fields /* (ny, nx_w, nt_snap) or NULL */,
    float* Data_synth /* (nt, NumRec) or NULL */);

/*
 * Replaces dynamic_window_solver_backward_ram (src/dynamic_window.f90:143-183),
 * which calls solver_ac_backward_ram (src/solver_ac_backward_ram.f90:4-598).
 * AdjSource(nt, NumRec) is injected at the receivers; the imaging condition
 * is accumulated into PSDM_thread(ny, nx_w) (read, then updated in place).
 */
int psdm_dynamic_window_solver_backward_ram(
    psdm_engine* e, const psdm_params* prm, int32_t NumRec,
    const int32_t* nxSou, const int32_t* nySou, const int32_t* nxRec, const int32_t* nyRec,
    const float* AdjSource /* (nt, NumRec) */, float dd, float dt, int32_t ny, int32_t nx,
    int32_t nx_w, const float* Vp_w /* (ny, nx_w) */, float dd_space, int32_t store_snap,
    int32_t nt_snap, int32_t nt, const float* Fields /* (ny, nx_w, nt_snap) */,
    float* PSDM_thread /* (ny, nx_w), in/out */);

/*
 * One shot of RTM: replaces the per-shot block of calculate_PSDM_RTM
 * (src/calculate_PSDM_RTM.f90:395-466) -- forward propagation, the optional
 * half-cosine taper of the snapshot series (taper_pad_trace,
 * src/filters.f90:20-48), time reversal of the conditioned data, backward
 * propagation with the imaging condition.  The snapshots stay in device
 * memory.  prm->strategy selects the RAM (1) or disk (2) solvers' statement
 * order; prm->precision selects FP32 snapshots (bit-exact drop-in) or the
 * mixed-precision form.  PSDM_w(ny, nx_w) is overwritten.
 */
int psdm_rtm_shot(
    psdm_engine* e, const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
    const int32_t* nxRec, const int32_t* nyRec, const float* Data_source /* nt_prop2 */,
    const float* Data_target /* (nt_taper, NumRec), conditioned, not reversed */,
    float dd, float dt, int32_t ny, int32_t nx, int32_t nx_w, const float* Vp_w /* (ny, nx_w) */,
    float added_space, int32_t store_snap, int32_t nt_snap, int32_t nt_prop2, int32_t nt_taper,
    int32_t taper_option, int32_t N_taper, int32_t N_zeros, float* PSDM_w /* (ny, nx_w) out */);

/*
 * psdm_rtm_shot with every array already in device memory (d_* pointers are
 * device pointers; nxRec/nyRec stay on the host).  Asynchronous: work is
 * queued on the engine's stream and the call returns without waiting.  Same
 * arithmetic as psdm_rtm_shot; for host frameworks that keep models, data
 * and images resident in HBM across shots.
 */
int psdm_rtm_shot_device(
    psdm_engine* e, const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
    const int32_t* nxRec, const int32_t* nyRec, const float* d_Data_source,
    const float* d_Data_target, float dd, float dt, int32_t ny, int32_t nx, int32_t nx_w,
    const float* d_Vp_w, float added_space, int32_t store_snap, int32_t nt_snap, int32_t nt_prop2,
    int32_t nt_taper, int32_t taper_option, int32_t N_taper, int32_t N_zeros, float* d_PSDM_w);

/*
 * One shot of a batched call.  Geometry in model coordinates as for
 * psdm_rtm_shot; nxRec/nyRec are host arrays.  Vp_w, Data_target and PSDM_w
 * are host pointers for psdm_rtm_batch and device pointers for
 * psdm_rtm_batch_device.
 */
typedef struct psdm_shot {
    int32_t NumRec, nxSou, nySou;
    const int32_t* nxRec;
    const int32_t* nyRec;
    int32_t nx_w;                /* window width (dynamic_window of this geometry) */
    int32_t nt_prop2, nt_taper;  /* forward steps, data length (>= nt_prop2) */
    const float* Vp_w;           /* (ny, nx_w) migration model of the window */
    const float* Data_target;    /* (nt_taper, NumRec), conditioned, not reversed */
    float* PSDM_w;               /* (ny, nx_w) out, overwritten */
} psdm_shot;

/*
 * Many shots through the per-shot block of calculate_PSDM_RTM
 * (src/calculate_PSDM_RTM.f90:395-466), several at a time: each time step is
 * one launch that advances every shot in flight (its forward pass, then its
 * backward pass with the imaging condition), and a finished shot's place is
 * taken by the next one, so windows and record lengths may differ from shot
 * to shot.  Up to max_slots shots (at most 16; <= 0 = as many as fit) are in
 * flight, limited by the free device memory (each holds its FP32 snapshots).
 * Every PSDM_w equals what psdm_rtm_shot returns for that shot, bit for bit.
 * Data_source (>= max nt_prop2 samples) is shared by all shots, as in the
 * reference (one Ricker wavelet per run).  The reference has no batched
 * interface: it runs one shot per MPI rank at a time.
 */
int psdm_rtm_batch(
    psdm_engine* e, const psdm_params* prm, int32_t nshots, const psdm_shot* shots,
    const float* Data_source, float dd, float dt, int32_t ny, int32_t nx, float added_space,
    int32_t store_snap, int32_t taper_option, int32_t N_taper, int32_t N_zeros, int32_t max_slots);
/* Same with device pointers (Data_source too); returns when all images are written. */
int psdm_rtm_batch_device(
    psdm_engine* e, const psdm_params* prm, int32_t nshots, const psdm_shot* shots,
    const float* d_Data_source, float dd, float dt, int32_t ny, int32_t nx, float added_space,
    int32_t store_snap, int32_t taper_option, int32_t N_taper, int32_t N_zeros, int32_t max_slots);
/*
 * Checkpointing (psdm_rtm_shot, psdm_rtm_batch and their device variants,
 * FP32 and mixed precision): interval K > 0 keeps the propagation state every
 * K forward steps and recomputes each K-step segment of the forward pass
 * during the backward pass, in place of holding all snapshots of the pass
 * (the role of the reference's disk strategy,
 * solver_ac_forward_disk.f90:469-517).  Mixed-precision segments are staged
 * and converted to 16 bits as in the pass without checkpoints.  Same image
 * bit for bit; the forward pass runs twice.  0 (default) = off.
 * Reconstruction (psdm_engine_set_reconstruction) takes precedence for
 * single FP32 shots.
 */
int psdm_engine_set_checkpointing(psdm_engine* e, int32_t interval);
/*
 * Boundary-saved reconstruction for FP32 shots (psdm_rtm_shot,
 * psdm_rtm_shot_device) with store_snap 1: 1 saves
 * the 3 C-PML cells next to the interior on each side at every forward step
 * (4 B x (6 ny + 6 nx_w) per step) and rebuilds the source wavefield
 * backwards in time on the interior during the backward pass, in place of
 * holding nt_prop2 snapshots (the role of the reference's disk strategy,
 * solver_ac_forward_disk.f90:469-517).  The image equals the plain shot's
 * to rounding level (the reverse recursion is not bit-exact).  Its passes
 * run two steps per launch.  0 (default) = off; takes precedence over
 * checkpointing.
 */
int psdm_engine_set_reconstruction(psdm_engine* e, int32_t on);
/*
 * Launch form of one shot's passes (psdm_rtm_shot, psdm_model_shot and their
 * device variants): 1 runs a pass whose steps allow it as one cooperative
 * launch in which each tile advances as soon as its neighbours finished the
 * previous step; 2 runs each forward and plain backward pass as one
 * cooperative launch of one block per region of the grid, each block keeping
 * its region's wavefield in shared memory for the whole pass and exchanging
 * only the ring with its neighbours (grids that fit the device's blocks;
 * others fall back to one launch per step); 0 (default) launches one kernel
 * per time step (replayed from a CUDA graph).  Same results bit for bit.
 * Passes with the mixed-precision snapshots always use one launch per step.
 * Values other than 0, 1 and 2 return PSDM_ERR_ARG.
 */
int psdm_engine_set_pass_launch(psdm_engine* e, int32_t on);
/*
 * Time steps per kernel launch for every pass of the engine (no reference
 * counterpart; the reference advances its arrays one step at a time,
 * solver_ac_forward_ram.f90:344-573): 1 (default) launches one kernel per
 * step; 2 advances each tile two steps per launch, level n+1 computed on the
 * tile and a 3-cell ring in shared memory, so that the wavefield crosses HBM
 * and the launch queue half as often.  Same results bit for bit.  On the
 * B200 the one-step form is currently the faster (see psdm_engine_autotune,
 * which times both).  The cooperative pass launch
 * (psdm_engine_set_pass_launch) and checkpointed shots use one step per
 * launch; reconstruction (psdm_engine_set_reconstruction) uses two.
 */
int psdm_engine_set_steps_per_launch(psdm_engine* e, int32_t steps);

/*
 * Planning against an HBM budget (the role of the reference's rtm_strategy,
 * optimization.f90:114-188, which picks RAM, disk or checkpoint strategies
 * from the memory per rank).
 */
typedef struct psdm_plan {
    int32_t steps_per_launch;     /* launch form chosen (1 or 2) */
    int32_t slots;                /* shots in flight for the batched calls (1: one shot at a time) */
    int32_t checkpoint_interval;  /* 0: all snapshots in HBM; K > 0: checkpoints every K steps */
    int32_t fits;                 /* 1 if the plan fits the budget */
    int64_t bytes_per_slot;       /* device bytes of one shot in flight under the plan */
    int64_t budget_bytes;         /* the budget planned against */
    float probe_us[2];            /* per-step device time measured with 1 and 2 steps per launch (0: not probed) */
} psdm_plan;

/*
 * Memory plan of shots of a window ny x nx_w with nt_prop2 / nt_taper steps
 * (host arithmetic only, no device needed): the device bytes of one shot in
 * flight for the snapshot form that prm->precision selects; slots =
 * min(max_slots, what fits in budget_bytes less a 1 GiB reserve); for shots
 * whose snapshots do not fit, the checkpoint interval K that minimises their
 * memory, and the slots that fit with it.  Returns PSDM_ERR_NOMEM, with
 * the sizes in psdm_last_error(), when not even that fits.  The plan's
 * steps_per_launch is 1 and probe_us zero.
 */
int psdm_plan_memory(const psdm_params* prm, int32_t ny, int32_t nx_w, int32_t nt_prop2, int32_t nt_taper,
                     int32_t store_snap, int32_t NumRec, int64_t budget_bytes, int32_t max_slots, psdm_plan* out);
/*
 * psdm_plan_memory against budget_bytes (0: the device's free memory plus
 * what the engine holds), then, if probe != 0, a timed probe of the launch
 * form: a 40-step forward pass of the window with one and with two steps per
 * launch; the faster is kept.  The plan is applied to the engine (steps per
 * launch, checkpoint interval); pass plan->slots as max_slots to the batched
 * calls.
 */
int psdm_engine_autotune(psdm_engine* e, const psdm_params* prm, int32_t ny, int32_t nx_w, int32_t nt_prop2,
                         int32_t nt_taper, int32_t store_snap, int32_t NumRec, int64_t budget_bytes,
                         int32_t max_slots, int32_t probe, psdm_plan* out);

/* Shots in flight at a time in the last batched call. */
int32_t psdm_engine_batch_slots(const psdm_engine* e);

/*
 * Exercise the engine's failure path without a GPU fault (no reference
 * counterpart): one kernel waits, with the step kernels' time limit (about
 * 1 s), for copies that are never issued, gives up and reports through the
 * engine's error word.  Returns PSDM_ERR_CUDA with the step kernels' timeout
 * message when the path works; the engine stays usable afterwards.
 */
int psdm_engine_check_wait_timeout(psdm_engine* e);

/*
 * The snapshot quotient of the forward kernels, x / dt, for n host inputs (no
 * counterpart: the reference divides in FP32 when it stores a snapshot,
 * src/solver_ac_forward_ram.f90:485): q[i] as the interior tiles compute it (a branch-free
 * form, with the general one for a float4 holding a rare input), q[n + i] by
 * the general form alone.  Both must equal the IEEE quotient x / dt rounded
 * to nearest, subnormal results and signed zeros included.  n is a positive
 * multiple of 4; q holds 2 n floats.
 */
int psdm_engine_dt_quotients(psdm_engine* e, float dt, const float* x, int32_t n, float* q);

/*
 * Forward modelling only (the receiver output Rec_point of
 * solver_ac_forward_ram, src/solver_ac_forward_ram.f90:567-577) without
 * storing snapshots: synthetic shot gathers for least-squares or QC.
 */
int psdm_model_shot(
    psdm_engine* e, const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
    const int32_t* nxRec, const int32_t* nyRec, const float* Data_source /* nt */, float dd,
    float dt, int32_t ny, int32_t nx, int32_t nx_w, const float* Vp_w, float dd_space,
    int32_t nt, float* Data_synth /* (nt, NumRec) out */);

/*
 * psdm_model_shot without any device allocation; no counterpart in the
 * reference.  For callers that cannot allocate device memory when they model
 * a shot: applications whose device memory belongs to their own pool or to
 * a fixed budget, and plugins that must not touch their host's device heap.
 * Needs no engine.  The scratch (wavefield, model, C-PML variables, ...)
 * is one fixed static device array of about 19 MB per GPU that loads this
 * library, kept until exit.  Limits: rows x columns <= 2^19 cells, where
 * rows = ny + 2*(dPML+6) plus up to 3 alignment rows, rounded up to a
 * multiple of 32 (at most 4096) and columns = nx_w + 2*(dPML+6) (at most
 * 4096); NumRec <= 8192.  Larger shots return PSDM_ERR_ARG with the sizes
 * in psdm_last_error().
 * d_Data_source (nt), d_Vp_w (ny, nx_w) and d_Data_synth ((nt, NumRec),
 * overwritten) are device pointers owned by the caller; nxRec/nyRec are host
 * arrays.  Work is queued on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) and the call returns when it has finished.  Every call
 * looks up the scratch's device address in the context current at the call
 * (the first call on a device also prepares the kernels).  The call copies
 * from pageable host memory and waits for `stream`, so it must not be made
 * while `stream`, or any other stream of the device, is being captured into
 * a CUDA graph.  All calls on a device share the one scratch: calls that
 * overlap on the GPU (other host threads, or other streams) race and corrupt
 * each other's results.
 */
int psdm_model_shot_noalloc(
    const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
    const int32_t* nxRec, const int32_t* nyRec, const float* d_Data_source, float dd, float dt,
    int32_t ny, int32_t nx, int32_t nx_w, const float* d_Vp_w, float dd_space, int32_t nt,
    float* d_Data_synth, void* stream);

/*
 * FP64 build of one shot of the mixed-precision form's schedule on the GPU:
 * the error reference of the FP32 and FP16/BF16 forms (no counterpart in the
 * reference, whose solvers are FP32).  The same per-cell update as the FP32
 * kernels in double precision (FD coefficients, C-PML profiles and c2 set up
 * in double from the FP32 inputs), snapshots every store_snap forward steps
 * kept in FP64, imaging at the paired backward steps (for store_snap 1 the
 * reference's pairing, solver_ac_backward_ram.f90:455-470).  Host arrays in
 * the layouts of psdm_rtm_shot; PSDM_w (ny, nx_w) and, if not NULL,
 * Fields_out (ny, nx_w, (nt_prop2-1)/store_snap) receive doubles.  Runs on
 * `device` with its own device allocations, one launch per step; meant for
 * accuracy checks, not speed.
 */
int psdm_rtm_shot_fp64(
    int32_t device, const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
    const int32_t* nxRec, const int32_t* nyRec, const float* Data_source, const float* Data_target,
    float dd, float dt, int32_t ny, int32_t nx, int32_t nx_w, const float* Vp_w, float added_space,
    int32_t store_snap, int32_t nt_prop2, int32_t nt_taper, int32_t taper_option, int32_t N_taper,
    int32_t N_zeros, double* PSDM_w, double* Fields_out);

/* ---- host helpers: the reference's set-up arithmetic, same FP32 order ---- */

/* finite_difference_coef (src/solver_FD_coeffs.f90:1-73); coef[acc+1]. */
void psdm_fd_coef(int32_t num, int32_t accuracy, float* coef);

/*
 * PML_coeffs (src/solver_PML_coeffs.f90:1-75): factorA/B[dn] with dn =
 * dPML + 2*acc (zero for the first acc cells), and the corner matrices
 * ld, rd, lu, ru (A then B) as 8 consecutive (dn, dn) column-major blocks.
 */
void psdm_pml_coeffs(int32_t acc, int32_t dPML, float dt, float d, int32_t dn, float* factorA,
                     float* factorB, float* corners /* 8*dn*dn or NULL */);

/* Ricker_mcs (src/get_mcs_data.f90:318-351). */
void psdm_ricker_mcs(int32_t nt, float dt, float f0, float t0, float* S0);

/* dynamic_window (src/dynamic_window.f90:1-52) for one shot. */
void psdm_dynamic_window(int32_t NumRec, int32_t nxSou, const int32_t* nxRec, float dd, int32_t nx,
                         float dd_space, int32_t* nx_w, int32_t* x_i, int32_t* x_f);

/* taper_pad_trace (src/filters.f90:20-48), in place on trace[nt_new]. */
void psdm_taper_pad_trace(float* trace, int32_t nt_prop, int32_t N_taper, int32_t N_zeros,
                          int32_t nt_new);

/* optimization's time step (src/optimization.f90:24-32): dt_prop, nt_prop, nt_snap. */
void psdm_optimization_dt(float dmodel_prop, float vmax, float tfin, int32_t store_snap,
                          float* dt_prop, int32_t* nt_prop, int32_t* nt_snap);

/* ---- trace conditioning (src/calculate_PSDM_RTM.f90:231-355) ---------------- */

/* Parfile switches of the conditioning (modules.f90: cut_multiple, cut_sf,
 * taper_option, T_taper, T_zeros; T_taper after the reader's default rule
 * T_taper = T_zeros/4 when it is 0, modules.f90:556). */
typedef struct psdm_conditioning {
    int32_t cut_multiple;
    int32_t cut_sf;
    int32_t taper_option;
    float T_taper, T_zeros; /* seconds */
} psdm_conditioning;

/*
 * Time windows of one shot (calculate_PSDM_RTM.f90:231-291), the reference's
 * FP32 arithmetic: per trace nt_cut (before the sea-floor multiple) and nt_sf
 * (after the direct water wave), from the sea-floor depth Batmodel (nx_prop
 * values, metres) at the source-receiver midpoint; then lens = {nt_prop2,
 * nt_taper, N_taper, N_zeros}.
 */
void psdm_trace_windows(const psdm_conditioning* c, int32_t NumRec, int32_t nxSou, int32_t nySou,
                        const int32_t* nxRec, const int32_t* nyRec, const float* Batmodel,
                        float dmodel_prop, float dt_prop, int32_t nt_prop, int32_t* nt_cut,
                        int32_t* nt_sf, int32_t* lens /* 4 */);

/*
 * Data_target (nt_taper, NumRec) from Field_Data (nt_data, NumRec) on the GPU
 * (calculate_PSDM_RTM.f90:316-355): resampling from dt_data to dt_prop by
 * Akima's local cubic interpolation when they differ (in place of the
 * reference's vendored TOMS-433 routine, interpolation_akima.f90), the
 * sea-floor cut, the multiple cut and the taper with zero padding.  The
 * frequency filter (freq_filter) is not part of it: filter Field_Data first.
 * nt_cut, nt_sf and lens come from psdm_trace_windows.
 */
int psdm_condition_traces(psdm_engine* e, const psdm_conditioning* c, int32_t NumRec,
                          const float* Field_Data, int32_t nt_data, float dt_data, float dt_prop,
                          const int32_t* nt_cut, const int32_t* nt_sf, const int32_t* lens,
                          float* Data_target);
/* Same with device pointers for Field_Data and Data_target (nt_cut, nt_sf and
 * lens stay on the host); asynchronous on the engine's stream. */
int psdm_condition_traces_device(psdm_engine* e, const psdm_conditioning* c, int32_t NumRec,
                                 const float* d_Field_Data, int32_t nt_data, float dt_data,
                                 float dt_prop, const int32_t* nt_cut, const int32_t* nt_sf,
                                 const int32_t* lens, float* d_Data_target);

/*
 * The frequency filter of the data preparation (freq_filter, src/auxiliar.f90:
 * 498-531, with filters_function1D and butterworth, src/filters.f90:50-232) on
 * the GPU, in place on traces (nt, Num): order-6 Butterworth low-pass
 * (typef 1, cut-off f2), high-pass (2, from 40 Hz as the reference fixes it)
 * or band-pass (3, f1..f2), applied through a 24-times zero-padded FFT;
 * all-zero traces are left as they are.  The transforms are cuFFT's, so the
 * result matches the reference's FFTPACK arithmetic to FP32 rounding.
 */
int psdm_freq_filter(psdm_engine* e, float* traces, int32_t nt, float dt, int32_t Num, int32_t typef,
                     float f1, float f2);
/* The filter's response H (ts complex values, interleaved re/im) for sampling
 * frequency fe = 1/dt and zero-padded length ts (24 nt), as butterworth
 * computes it (src/filters.f90:129-232); host only. */
int psdm_butterworth_response(int32_t ts, float fe, int32_t typef, float f1, float f2, float* H);
/* Same on a device array; asynchronous on the engine's stream. */
int psdm_freq_filter_device(psdm_engine* e, float* d_traces, int32_t nt, float dt, int32_t Num,
                            int32_t typef, float f1, float f2);

/* ---- SU trace files without the SU tools ---------------------------------- */

/*
 * Write model(nj, ni) as ni SU traces of nj samples with the headers the
 * reference's write_psdm / write_vel pipelines set (src/auxiliar.f90:275-353,
 * a2b | suaddhead | sushw | suchw): tracl = tracr = 1..ni, ns = nj, d1 = dj,
 * f1 = 0, d2 = di, f2 = 0, cdp = -di + di*tracl, trid.  big_endian != 0
 * writes big-endian words.
 */
int psdm_su_write_image(const char* path, int32_t ni, int32_t nj, float di, float dj, int32_t trid,
                        const float* model, int32_t big_endian);
/*
 * Read NumRec fixed-length SU traces (240-byte header + ns_max samples) as
 * get_shot_data does (src/get_mcs_data.f90:150-214): raw (nt, NumRec) gets
 * samples 1..nt of each trace; delayed (nt, NumRec, or NULL) gets them shifted
 * by delay_samples (later for > 0), zero where nothing lands.
 */
int psdm_su_read_shot(const char* path, int32_t NumRec, int32_t ns_max, int32_t nt, int32_t big_endian,
                      int32_t delay_samples, float* raw, float* delayed);
/* The int32 header word at 1-based byte position byte_pos of each of NumRec
 * fixed-length traces (shot number, offset: get_mcs_data.f90:449-470). */
int psdm_su_read_header_i32(const char* path, int32_t NumRec, int32_t ns_max, int32_t byte_pos,
                            int32_t big_endian, int32_t* out);

/* ---- Survey geometry (host) ------------------------------------------------ */
/*
 * read_nav_shot_mcs (src/get_mcs_data.f90:30-126): the shot navigation file,
 * one record per shot, list-directed: "shotID x" (cols 11), "shotID x y"
 * (111) or "shotID x y depth" (1111).  pos_shot = d_shot_model + distance
 * from the line's origin (the first shot for dir_boat = 1, the last for -1),
 * pos_bat = |depth|.  shot_i / shot_f = 0 select the first / last record's
 * shot; out = {nlines, line_i, line_f} (1-based records of shot_i, shot_f;
 * the last record with the number wins).  out[0] is set even when max_lines
 * is too small (then PSDM_ERR_ARG); a shot number not found is PSDM_ERR_ARG.
 */
int psdm_nav_read(const char* path, int32_t cols, int32_t dir_boat, float d_shot_model, int32_t shot_i,
                  int32_t shot_f, int32_t max_lines, int32_t* shotID, float* pos_shot, float* pos_bat,
                  int32_t* out /* 3 */);
/*
 * get_pos_channels (src/get_mcs_data.f90:418-510): channel positions of one
 * shot, pos_rec = pos_shot - dir_boat * offset, the offset from the trace
 * headers (offset_header = 1: |offset| * offset_unit, or |offset| /
 * |offset_unit| when offset_unit < 0; read them with
 * psdm_su_read_header_i32) or from the spread (offset_header = 0:
 * near_offset + (i-1) drec).
 */
int psdm_channel_positions(float pos_shot, int32_t NumRec, int32_t dir_boat, int32_t offset_header,
                           float offset_unit, const int32_t* offsets, float near_offset, float drec,
                           float* pos_rec);
/* get_geometry_mcs (src/get_mcs_data.f90:128-148): 1-based grid indices
 * 1 + floor(position / dd) of the source and the channels. */
int psdm_geometry_mcs(float pos_shot, int32_t NumRec, const float* pos_rec, float shot_depth,
                      float streamer_depth, float dd, int32_t* nxSou, int32_t* nySou, int32_t* nxRec,
                      int32_t* nyRec);
/* linear_2D (src/linear_interpolation.f90:1-45, with linear_interpolation_1D
 * :79-117): the model vel (nymodel, nxmodel) at dmodel resampled to Vpmodel
 * (ny_prop, nx_prop) at dmodel_prop, along depth then along x. */
int psdm_linear_2d(int32_t nxmodel, int32_t nymodel, float dmodel, const float* vel, int32_t nx_prop,
                   int32_t ny_prop, float dmodel_prop, float* Vpmodel);
/* Sea-floor depth per column (src/00-main.f90:146-158): (j-2) dmodel_prop for
 * the first 1-based row j whose velocity exceeds water_velocity, else 0. */
int psdm_batmodel_from_velocity(int32_t nx_prop, int32_t ny_prop, float dmodel_prop, float water_velocity,
                                const float* Vpmodel, float* Batmodel);

/*
 * Wide-angle (OBS) data: by reciprocity the OBSs are the sources and the shots
 * the receivers.  read_nav_shot_was (src/get_was_data.f90:70-125): the first
 * NumShots records "shotID x [y [depth]]" (cols 11 / 111 / 1111);
 * pos_shot = d_shot_model + distance from the first shot, pos_bat = |depth|;
 * out_i = {line_i, line_f (0 when the number is absent), nxmodel_was =
 * 1 + ceiling(length_model_was / dmodel)}, out_f = {dshots_was,
 * length_model_was = last shot's x + 2 added_space}.
 */
int psdm_nav_read_was(const char* path, int32_t cols, int32_t NumShots, float d_shot_model, float added_space,
                      float dmodel, int32_t shot_i, int32_t shot_f, int32_t* shotID, float* pos_shot,
                      float* pos_bat, int32_t* out_i /* 3 */, float* out_f /* 2 */);
/* read_nav_obs (src/get_was_data.f90:127-160): NumOBS records "obsID x z";
 * positions |x|, |z| and their grid indices 1 + ceiling(position / dmodel). */
int psdm_nav_read_obs(const char* path, int32_t NumOBS, float dmodel, int32_t* obsID, float* pos_xobs,
                      float* pos_zobs, int32_t* xgrid, int32_t* zgrid);
/* get_geometry_WAS (src/get_was_data.f90:162-189): the OBS's grid indices as
 * the source, 1 + ceiling(position / dd) of the shots as the receivers. */
int psdm_geometry_was(int32_t xobs_grid, int32_t zobs_grid, int32_t NumRec, const float* pos_shot,
                      float shot_depth, float dd, int32_t* nxSou, int32_t* nySou, int32_t* nxRec,
                      int32_t* nyRec);
/* get_bathymetry_model_was / _mcs (src/get_was_data.f90:500-549,
 * src/get_mcs_data.f90:353-415): sea-floor depth at x = (i-1) dmodel along
 * the line, Akima's interpolant through (0, first depth), the shots
 * (pos_shot, pos_bat) and (length_model, last depth).  Positions must
 * increase strictly. */
int psdm_bathymetry_nav(int32_t NumShots, const float* pos_shot, const float* pos_bat, float length_model,
                        int32_t nxmodel, float dmodel, float* bat_model);
/* relocation_zOBS (src/get_was_data.f90:30-68): each OBS moved to the sea
 * floor under it, pos_zobs = bat_model(xgrid), zgrid = 1 + ceiling(pos_zobs /
 * dmodel). */
int psdm_relocate_obs(int32_t NumOBS, const int32_t* xgrid, const float* bat_model, int32_t nxmodel,
                      float dmodel, float* pos_zobs, int32_t* zgrid);

/* normalize_psdm (src/auxiliar_PSDM.f90:1-20): PSDM = sum/fold where fold > 0. */
void psdm_normalize_psdm(int32_t nx, int32_t ny, const float* PSDM_sum, const float* Cov_sum,
                         float* PSDM);

#ifdef __cplusplus
}
#endif

#endif /* PSDM_RTM_H */
