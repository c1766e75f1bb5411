// Internal declarations shared by the host code and the CUDA translation
// units of the RTM engine.  Not part of the C ABI.
#pragma once

#include <complex>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace psdm {

constexpr int kAcc = 3;  // FD half-width (acc=3, src/solver_ac_forward_ram.f90:95)

void pml_profiles_f32(int acc, int dPML, float dt, float d, int dn, float* fA, float* fB);
void pml_profiles_f64(int acc, int dPML, double dt, double d, int dn, double* fA, double* fB);
void fd_coef_f64(int num, double* c);  // acc = 3
float taper_weight(int n, int N_taper);
// True if x/y may be computed as RN(q0 + (x - q0*y)*r), q0 = RN(x*r),
// r = RN(1/y), for |x| in [lo, hi] (exhaustive check over one binade).
bool fast_div_exact(float y, float* r, float* lo, float* hi, float* tiny);

// Padded propagation grid of one shot (0-based, column-major, z fastest):
//   logical z in [0, nyt), x in [0, nxt); element (z, x) is stored at device
//   row zd = z + zoff, i.e. at x*ldz + zd.  zoff in [0, 3] makes the first
//   interior row dn start on a 16-byte boundary.
// Interior rows [dn, dn+ny), interior columns [dn, dn+nx); dn = dPML+2*acc
// (src/solver_ac_forward_ram.f90:103-127).
// Snapshots and images of the interior are stored column by column with the
// pitch ldf = ny rounded up to 4: interior cell (j, i) at i*ldf + j.
struct Grid {
    int ny = 0, nx = 0, dPML = 0, dn = 0, nyt = 0, nxt = 0, ldz = 0, zoff = 0, ldf = 0;
    size_t cells() const { return (size_t)ldz * (size_t)nxt; }
    size_t field_cells() const { return (size_t)ldf * (size_t)nx; }
};

// The layout above for an ny x nx window and a C-PML of dPML cells (ny, nx,
// dPML >= 1).  Every path that builds a padded grid uses this one function.
inline Grid make_grid(int dPML, int ny, int nx) {
    Grid g;
    g.ny = ny;
    g.nx = nx;
    g.dPML = dPML;
    g.dn = dPML + 2 * kAcc;
    g.nyt = g.dn + ny + g.dn;
    g.nxt = nx + 2 * g.dn;
    g.zoff = (4 - g.dn % 4) % 4;
    g.ldz = (g.zoff + g.nyt + 31) / 32 * 32;
    g.ldf = (ny + 3) / 4 * 4;
    return g;
}

// Message for a nonzero value of a step kernel's error word: 1 = a bounded
// wait for the tile's shared-memory copies ran out, 2 = the tile plan was
// made for another launch form, 3 = a pass kernel gave up waiting for its
// neighbouring tiles.
inline const char* step_error_message(int code) {
    switch (code) {
        case 2: return "a step kernel was given a tile plan for another launch form";
        case 3: return "a pass kernel timed out waiting for neighbouring tiles";
        default: return "a step kernel timed out waiting for its shared-memory copies";
    }
}

// Arguments of one fused time step.  Pointers are device pointers.
struct StepArgs {
    // wavefield: p = level n (read only); pm = level n-1 in, level n+1 out
    const float* p;
    float* pm;
    const float* c2;
    // C-PML memory variables on the padded grid (only PML cells touched)
    const float* phix_in;
    float* phix_out;
    float* chix;
    const float* phiz_in;
    float* phiz_out;
    float* chiz;
    // strip-private histories of the free-surface row in the x-strip columns
    // (RAM ordering with a free surface): side_p = level n, side_pm = n-1 -> n+1
    const float* side_p;
    float* side_pm;
    // C-PML profiles factorA/B[dn] (index k-1, k = 1 next to the interior)
    const float* fA;
    const float* fB;
    // FD coefficients (finite_difference_coef, acc = 3)
    float cf1[4];
    float cf2[4];
    // grid
    int nyt, nxt, ldz, ny, nx, dn, zoff, ldf;
    int fs;     // free surface on
    int disk;   // disk solvers' statement order
    // injection (sources / adjoint sources): row_slot[zd] = -1 or a row slot
    // (indexed by device row, ldz entries);
    // inj_cols[slot*nxt + x] = trace index or -1; value inj_trace[j*inj_ld + inj_t]
    const int* row_slot;
    const int* inj_cols;
    const float* inj_trace;
    int inj_ld, inj_t;
    // forward snapshot (write) or backward snapshot (read); null = none this step
    float* field;
    float dt;
    // snapshot division by dt: reciprocal + one FMA correction when exact
    float inv_dt, div_lo, div_hi, div_tiny;
    int fast_div;
    // backward imaging: image[(x-dn)*ldf + (z-dn)] += 0.5*(p3-p1)*field*w*ss
    float* image;
    float field_w;   // taper weight of this snapshot slot
    float ss;        // float(store_snap)
    // deferred receiver gather (forward): rec_out[i*rec_ld + rec_t] = p[rec_cell[i]]
    const int* rec_cell;
    float* rec_out;
    int nrec, rec_ld, rec_t;  // rec_t < 0: no gather this step
    // block decomposition (plan_tiles): rect r of type r_type (0 interior
    // band, 1 C-PML x-strip band, 2 z-strip, 3 corner, 4 interior rows with
    // injection or the free surface) covers device rows
    // [r_zd0, r_zd0+r_h) x columns [r_x0, r_x0+r_w); its tiles are blocks
    // [r_first[r], r_first[r+1]) with r_tz tiles along z.
    int nrect;
    int itx;  // interior tile columns the plan was made for (one-shot or batched launches)
    int ixb;  // C-PML x-strip tile columns the plan was made for (one-shot or batched launches)
    int r_type[16], r_zd0[16], r_x0[16], r_h[16], r_w[16], r_tz[16], r_first[17];
    // persistent scheduling: tile_counter[counter_sel] starts at 0 (cleared
    // by the previous step); num_sms = multiprocessor count of the device
    int* tile_counter;
    int counter_sel;
    int num_sms;
    int* err;  // set to 1 if a bulk copy did not complete
    // Mixed-precision form: snapshots kept as binary16 / bfloat16 scaled by a
    // power of two per snapshot, image summed with Kahan compensation.
    unsigned int* field_amax;   // forward: max |snapshot| of this step (float bits), or null
    const void* field16;        // backward (mode 2): this step's 16-bit snapshot, pitched like field
    const float* field_iscale;  // its inverse scale 2^-k
    float* comp;                // backward (mode 2): Kahan compensation of the image
    int kind16;                 // 1 = binary16, 2 = bfloat16
    // Quantization of an earlier snapshot, done by this launch's blocks
    // before their tiles: q_dst[i] = round16(q_src[i] * 2^k) for i < q_n and
    // *q_iscale = 2^-k, with k from *q_amax.  q_src = null: none.
    int q_n;
    const float* q_src;
    const unsigned int* q_amax;
    void* q_dst;
    float* q_iscale;
};

// One launch advancing several shots ("slots") by one time step each:
// slot s runs pass mode[s] (0 forward, 1 backward, 2 mixed backward) with the step arguments
// at args[s] (device memory); its tiles are [first[s], first[s+1]) of the
// launch's work list, first[s+1] - first[s] = that step's r_first[nrect].
// counter[counter_sel] starts at 0; the launch clears the other one.
constexpr int kMaxSlots = 16;
struct BatchParams {
    int nslots;
    int counter_sel;
    int* counter;
    int mode[kMaxSlots];
    int first[kMaxSlots + 1];
    const StepArgs* args[kMaxSlots];
};

// ---- Two time steps per launch (rtm_pair.cu) ------------------------------
//
// A pair launch advances the grid from levels (n-1, n) to (n+1, n+2): each
// tile loads level n on itself plus a 6-cell ring, computes level n+1 on
// itself plus a 3-cell ring in shared memory (the ring is recomputed,
// bit-identically, by the neighbouring tiles), then level n+2 on itself.
// Inputs are only read and outputs go to other buffers, so the wavefield
// rotates through four buffers, the C-PML variables through two each and
// the free-surface histories through four.

// Per-step values of one sub-step of a pair launch.
struct SubStep {
    float* field;               // forward: snapshot written (FP32, or the mixed form's staging buffer);
                                // backward: FP32 snapshot read; null = none at this sub-step
    const void* field16;        // mixed backward: 16-bit snapshot read, or null
    const float* field_iscale;  // its inverse scale 2^-k
    unsigned int* field_amax;   // mixed forward: largest |snapshot| (float bits), or null
    float field_w;              // taper weight of the snapshot slot
    int inj_t;                  // injection sample index of this step
    int rec_t;                  // forward: receiver sample taken from this sub-step's level, or -1
    int pad_;
    float* band;                // forward: this level's band (band_index) written, or null
};

// The band of a padded grid: the 3 C-PML cells next to the interior on each
// side (x strips over the interior rows, z strips over the interior
// columns), nband = 6*ny + 6*nx values, at index
//   x strips: col * ny + (z - dn), col 0..2 left (x = dn-3..dn-1), 3..5 right;
//   z strips: 6*ny + (x - dn) * 6 + row, row 0..2 bottom, 3..5 top.
// With it every interior cell's stencil has its operands: the interior and
// the band.
inline int band_count(int ny, int nx) { return 6 * ny + 6 * nx; }

// Reverse time step of the interior (boundary-saved reconstruction of the
// source wavefield): pn = level L+2 in, level L out, pc = level L+1
// (interior and band filled).  snap = (P(L+2) - P(L)) * 0.5 / dt on the
// interior; band_L = the saved band of level L, written into pn's band.
struct ReconArgs {
    const float* pc;
    float* pn;
    const float* c2;
    const float* band_L;
    float* snap;
    float cf2[4];
    int nyt, nxt, ldz, ny, nx, dn, zoff, ldf, fs;
    const int* row_slot;
    const int* inj_cols;
    const float* inj_trace;
    int inj_t;
    float dt, inv_dt, div_lo, div_hi, div_tiny;
    int fast_div;
};
int launch_reconstruct(const ReconArgs& r, void* stream);

constexpr int kPairRects = 48;

struct PairArgs {
    // Common fields.  a.p = level n (read on tile + 6), a.pm = level n-1
    // (read on tile + 3), a.phix_in / a.phiz_in = phi at level n, a.phix_out
    // / a.phiz_out = phi at level n + nsub, a.chix / a.chiz = chi at level
    // n + nsub (written), a.side_p / a.side_pm = free-surface histories at
    // levels n / n-1, a.q_* = the first snapshot conversion of the launch's
    // prologue.  a's per-step fields and tile plan are not used.
    StepArgs a;
    const float* chix_in;  // chi at level n
    const float* chiz_in;
    float* p_out[2];       // levels n+1, n+2
    float* side_out[2];    // free-surface histories at levels n+1, n+2
    SubStep sub[2];
    int nsub;              // 2: two steps; 1: one step (outputs at level n+1 only)
    int txc;               // columns of the clean interior tiles the plan was made for
    // second conversion of the prologue (two snapshots per launch)
    int q_n2;
    const float* q_src2;
    const unsigned int* q_amax2;
    void* q_dst2;
    float* q_iscale2;
    // receivers whose cell lies in tile b: rec_idx[rec_first[b] .. rec_first[b+1])
    const int* rec_first;
    const int* rec_idx;
    // Tile plan: rect r of type r_type (0 clean interior, 1 generic) covers
    // device rows [r_zd0, r_zd0 + r_h) x columns [r_x0, r_x0 + r_w), split
    // into r_tz x r_tx tiles, blocks [r_first[r], r_first[r+1]).
    int nrect;
    int r_type[kPairRects], r_zd0[kPairRects], r_x0[kPairRects], r_h[kPairRects], r_w[kPairRects];
    int r_tz[kPairRects], r_tx[kPairRects], r_first[kPairRects + 1];
};

// Plan the tiles of a pair launch from P->a's grid fields and the host copy
// of the injection row map (ldz entries or null).  Returns false if the plan
// needs more than kPairRects rectangles.
bool plan_pair(PairArgs* P, const int* row_slot_host);
// Cell rectangle [z0, z1) x [x0, x1) (device rows, columns) of tile b.
void pair_tile_rect(const PairArgs& P, int b, int* z0, int* z1, int* x0, int* x1);
// Receivers (linear cells x * ldz + device row) held by each tile, as offsets.
void pair_rec_lists(const PairArgs& P, int nrec, const int* h_rec_cell, std::vector<int>* first,
                    std::vector<int>* idx);
int prepare_pair_kernels();
// One pair launch of pass `mode` (0 forward, 1 backward, 2 mixed backward).
int launch_pair(int mode, const PairArgs& P, void* stream);

// Several shots per pair launch: slot s runs pass mode[s] with the arguments
// at args[s] (device memory), tiles [first[s], first[s+1]).
struct PairBatchParams {
    int nslots;
    int counter_sel;
    int* counter;
    int mode[kMaxSlots];
    int first[kMaxSlots + 1];
    const PairArgs* args[kMaxSlots];
};
int launch_pair_batch(const PairBatchParams& bp, int num_sms, void* stream);

// Fill the block decomposition of `a` from its grid fields (nyt, nxt, ny,
// nx, dn, zoff, fs) and the host copy of the injection row map (ldz
// entries, or null when nothing is injected).  `batched` plans the interior
// tiles of batch_step_kernel, otherwise those of step_kernel.
// forward: the plan of a one-shot forward pass (its interior tiles are narrower).
void plan_tiles(StepArgs* a, const int* row_slot_host, bool batched = false, bool forward = false);

// Set kernel attributes (shared memory carve-out, occupancy); call once per
// device before the first launch.  Returns a cudaError_t value.
int prepare_step_kernels();
// Launch one fused forward (mode 0), backward (mode 1) or mixed-precision
// backward (mode 2: 16-bit snapshots, Kahan image) step on `stream`.
int launch_step(int mode, const StepArgs& a, void* stream);
// Quantize one snapshot outside a step launch (see StepArgs::q_*).
int launch_quantize(const float* src, const unsigned int* amax, void* dst, float* iscale, int n, int kind16,
                    void* stream);
// Trace conditioning (rtm_condition.cu): Data_target (nt_taper per trace)
// from Field_Data (nt_data per trace); w = taper weights (N_taper).
struct CondArgs {
    const float* field;
    float* out;
    const int* nt_cut;
    const int* nt_sf;
    const float* w;
    int nrec, nt_data, nt_prop2, nt_taper, N_taper, N_zeros;
    int cut_multiple, cut_sf, taper_option, resample;
    float dt_data, dt_prop;
};
int launch_condition(const CondArgs& c, void* stream);

// Frequency filter (rtm_filter.cu): Butterworth response of length ts on the
// host, and the filtering of num traces of nt samples in place on `stream`
// with a batched length-ts cuFFT plan (an int handle stored at plan_ptr).
void butterworth_response(int ts, float fe, int typef, float f1, float fc, std::complex<float>* H);
int make_fft_plans(int ts, int num, int* plans);  // plans[0] real-to-complex, plans[1] complex-to-real
void destroy_fft_plans(int* plans);
size_t filter_work_floats(int ts, int num);
int filter_traces(float* d_tr, int nt, int num, const void* d_H, float* d_x, int* d_keep, int ts, const int* plans,
                  void* stream);

// ---- One launch per pass (dataflow form) --------------------------------
// A pass of one shot as a single cooperative launch: every tile of the plan
// is owned by one resident block, which advances it step after step as soon
// as the tiles whose cells its stencils read (its neighbours) have finished
// the previous step.  Tiles publish their completed step count in `flags`;
// waits are bounded and report through err.  Step arguments are the two
// parity bases with the per-step values of PassVar patched in.
struct PassVar {
    float* field;
    const void* field16;
    const float* field_iscale;
    float field_w;
    int inj_t;
    int rec_t;
    int par;
    int pad_;
};
static_assert(sizeof(PassVar) % 16 == 0, "PassVar is fetched in 16-byte pieces");

struct PassParams {
    const StepArgs* base;  // [2], by step parity
    const PassVar* var;    // [nsteps]
    int nsteps;
    int ntiles;
    const int* nbr_first;  // [ntiles + 1]
    const int* nbr;        // neighbour tiles of each tile
    const int* rec_first;  // [ntiles + 1]
    const int* rec_idx;    // receivers whose cell lies in each tile
    int* flags;            // [ntiles] steps completed, zero at launch
    int* abort;            // device word, zero at launch: set when a block gives up
    int* err;              // the engine's error word (host memory mapped into the device)
};

// Cell rectangle [z0, z1) x [x0, x1) (device rows, columns) of tile b of a plan.
void tile_rect(const StepArgs& a, int b, int* z0, int* z1, int* x0, int* x1);
// Halo (cells) within which a tile's reads of p, phi and the snapshot lie.
constexpr int kTileReadHalo = 12;
// Neighbour lists of a plan (tiles within kTileReadHalo cells of each other)
// and the receivers (linear cells x * ldz + row) held by each tile, both as
// offset arrays.
void pass_lists(const StepArgs& a, int nrec, const int* h_rec_cell, std::vector<int>* nbr_first,
                std::vector<int>* nbr, std::vector<int>* rec_first, std::vector<int>* rec_idx);
// Resident blocks per multiprocessor of the pass kernel (0 on failure).
int pass_blocks_per_sm(int mode);
// Launch one pass (modes 0, 1, 2) with `grid` co-resident blocks.
int launch_pass(int mode, const PassParams& pp, int grid, void* stream);

// ---- resident pass kernel (rtm_resident.cu) --------------------------------
// One cooperative launch per pass with one block per region of the grid; a
// block keeps its region's two wavefield levels in shared memory for the
// whole pass and exchanges only the 3-cell ring with its neighbours through
// the global wavefield buffers, waiting on their step counters.
constexpr int kResWarps = 16;
constexpr int kResThreads = 32 * kResWarps;
constexpr int kResRows = 384;             // most rows of a region (a multiple of 4)
constexpr int kResPitch = kResRows + 8;   // shared rows per column (4-row ring above and below)
constexpr int kResMinSide = 8;            // fewest rows and columns of a region
// Work item kinds of a warp (items[2k+1] = first quad or row
// (region-relative) << 16 | first column (region-relative)):
//   0  interior float4s: items[2k] = 0 | ncols << 4 | lanes << 8, lane l the
//      float4 of quad first+l over ncols columns
//   1  C-PML x-strip float4s (interior band rows): as 0, the x-strip update
//   3  C-PML z-strip float4s (interior columns, rows away from the strip and
//      grid edges): as 0, the z-strip update
//   2  generic cells: items[2k] = 2 | groups << 4 | rows << 8 | span << 16,
//      lane l row first + l % rows, columns [span*g/groups,
//      span*(g+1)/groups) of the item with g = l / rows
constexpr int kResFast = 0, kResXpml = 1, kResGen = 2, kResZpml = 3;
struct ResRegion {
    int zr0, nrows, x0, w;  // device rows [zr0, zr0+nrows) (multiples of 4) x columns [x0, x0+w)
    int nbr0, nnbr;         // neighbour regions nbr[nbr0 ..)
    int rec0, nrec;         // receivers rec[rec0 ..) (forward gather)
};
struct ResParams {
    const StepArgs* base;   // [2], by step parity
    const PassVar* var;     // [nsteps]
    int nsteps;
    int nreg;
    int sw;                 // shared columns per level buffer (widest region + 6)
    const ResRegion* reg;   // [nreg]
    const int* nbr;
    const int* rec;
    const int* warp_first;  // [nreg * kResWarps + 1] offsets into items (pairs)
    const int* items;       // [2 * nitems]
    int* flags;             // [nreg] steps completed, zero at launch
    int* abort;             // device word, zero at launch
    int* err;               // the engine's error word
};
struct ResPlan {
    std::vector<ResRegion> reg;
    std::vector<int> nbr, rec, warp_first, items;
    int sw = 0;
};
// Regions, neighbour lists, receiver lists and per-warp work items of the
// resident form for the step plan `a` (plan_tiles) with at most max_regions
// regions of at most max_sw - 6 columns.  False if the grid does not fit.
bool plan_resident(const StepArgs& a, int max_regions, int max_sw, int nrec, const int* h_rec_cell, ResPlan* plan);
// Widest shared-memory window (columns) of a resident block on this device,
// and how many resident blocks fit per multiprocessor (0 on failure).
int resident_max_sw();
int resident_blocks_per_sm(int mode, int sw);
// Launch one pass (modes 0 and 1) of the resident kernel, rp.nreg blocks.
int launch_resident(int mode, const ResParams& rp, void* stream);

// One kernel whose bounded copy wait runs out (nothing is copied); sets *err.
int launch_wait_timeout_probe(int* err, void* stream);
int launch_dt_quotients(float dt, float inv_dt, float div_lo, float div_hi, int fast_div, const float* x, float* q,
                        int n, void* stream);
// Launch one batched step (batch_step_kernel) on `stream`.
int launch_batch_step(const BatchParams& bp, int num_sms, void* stream);
// Receiver gather after the last forward step (Rec(nt-1) and Rec(nt)).
int launch_rec_final(const int* rec_cell, const float* p, float* rec_out, int nrec, int rec_ld, int nt, void* stream);
// Padded c2 = c^2 dt^2 / d^2 from the window model (edge replication;
// ram_padding = 1 reproduces the RAM solvers' partial top/bottom padding).
int launch_pad_c2(const float* vp, int ny, int nx, int dn, int nyt, int nxt, int ldz, int zoff, float dt, float dd,
                  int ram_padding, float* c2, void* stream);

// Record the message that psdm_last_error returns on this thread.
void set_last_error(const char* msg);

}  // namespace psdm
