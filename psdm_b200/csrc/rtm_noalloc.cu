// Forward modelling of one shot without allocating device memory
// (psdm_model_shot_noalloc).
//
// Who needs it: a caller that cannot call cudaMalloc or take memory from an
// allocator at the time it models a shot -- a host application whose device
// memory is owned by its own pool or capped by a fixed budget (a solver or
// inversion framework that hands out every byte itself), or a plugin that
// must leave the device heap of its host process untouched.
// psdm_model_shot needs an engine, and the engine allocates its buffers on
// demand; this entry point needs neither.
//
// How: every scratch array of the pass (wavefield levels, padded model,
// C-PML memory variables, free-surface histories, injection map, receiver
// cells, tile counters, error word) is carved out of one file-scope
// __device__ array, g_noalloc_scratch, of kScratchBytes (about 19 MB).  Each
// GPU that loads this library holds that array until the process exits.
// The caller passes its inputs (model, source trace) and its output (the
// receiver traces) in device memory it owns; the receiver coordinates are
// host arrays.  The time steps run the same step kernels as the engine
// (rtm_step.cu), so the traces are identical to psdm_model_shot's.
//
// In host code the name g_noalloc_scratch stands for the host-side shadow
// of the variable, not for device memory: every call looks its device
// address up with cudaGetSymbolAddress, with the caller's device current,
// and hands that address to the kernels.  The address belongs to the CUDA
// context current at the call, so a device reset or another context
// between calls is harmless.  The first call on a device also sets the
// step kernels' attributes.  The call copies from pageable host memory and
// waits for its stream, so it must not be made while any stream of the
// device is being captured into a CUDA graph.

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/psdm_rtm.h"
#include "rtm_internal.h"

namespace {

using namespace psdm;

// Limits of one call: a padded grid of at most kMaxCells cells (device rows
// times columns, rows counted with their 32-row alignment), at most
// kMaxRows device rows and kMaxCols columns, and at most kMaxRec receivers.
constexpr size_t kMaxCells = size_t(1) << 19;
constexpr int kMaxRows = 4096;
constexpr int kMaxCols = 4096;
constexpr int kMaxRec = 8192;
constexpr int kMaxDn = 1024;    // dPML + 6
constexpr int kGridArrays = 9;  // p (two levels), c2, phix (two), chix, phiz (two), chiz
constexpr size_t kAlign = 256;
// Every carve is rounded up to kAlign; 24 carves at most.
constexpr size_t kScratchBytes = kGridArrays * kMaxCells * sizeof(float) +
                                 (2 * size_t(kMaxCols) + 2 * size_t(kMaxDn)) * sizeof(float) +
                                 (size_t(kMaxRows) + size_t(kMaxCols) + 3 * size_t(kMaxRec) + 3) * sizeof(int) +
                                 24 * kAlign;

// Shared by every call on a device; keeps the last call's contents.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

int nfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_last_error(buf);
    return code;
}

#define NA_CUDA(expr)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (expr);                                                                       \
        if (e_ != cudaSuccess) return nfail(PSDM_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

// Kernel attributes are set once per device; the scratch's device address
// is looked up on every call (a cheap driver query), so that it always
// belongs to the context current at the call.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
bool g_prepared[kMaxDevices] = {false};

int scratch_address(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return nfail(PSDM_ERR_ARG, "device ordinal %d not supported", dev);
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_prepared[dev]) {
            const int rc = prepare_step_kernels();
            if (rc)
                return nfail(PSDM_ERR_CUDA, "preparing the step kernels: %s", cudaGetErrorString((cudaError_t)rc));
            g_prepared[dev] = true;
        }
    }
    // The look-up also loads this library's device code into the current
    // context if that has not happened yet.
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
        return nfail(PSDM_ERR_CUDA, "cudaGetSymbolAddress of the scratch array: %s", cudaGetErrorString(e));
    *out = static_cast<unsigned char*>(ptr);
    return PSDM_OK;
}

// Consecutive kAlign-aligned pieces of the scratch.
struct Carve {
    unsigned char* base;
    size_t off;
    template <class T>
    T* take(size_t count) {
        off = (off + kAlign - 1) / kAlign * kAlign;
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

// Injection map of the source (row slot 0, one column) and the receiver
// cells, from the receivers' window coordinates (rec_xy: nxRec then nyRec).
__global__ void noalloc_geometry_kernel(int* row_slot, int* inj_cols, int zs_dev, int xs, int src_interior,
                                        const int* rec_xy, int* rec_cell, int nrec, int dn, int x_i, int ldz,
                                        int zoff) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && src_interior) {
        row_slot[zs_dev] = 0;
        inj_cols[xs] = 0;
    }
    if (i < nrec) {
        const int zr = dn + rec_xy[nrec + i] - 1;
        const int xr = dn + (rec_xy[i] - x_i + 1) - 1;
        rec_cell[i] = xr * ldz + zr + zoff;
    }
}

// Host copy of the injection row map handed to plan_tiles.
thread_local int t_row_slot[kMaxRows];

}  // namespace

extern "C" int psdm_model_shot_noalloc(const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
                                       const int32_t* nxRec, const int32_t* nyRec, const float* d_Data_source,
                                       float dd, float dt, int32_t ny, int32_t nx, int32_t nx_w,
                                       const float* d_Vp_w, float dd_space, int32_t nt, float* d_Data_synth,
                                       void* stream) {
    if (!prm || !nxRec || !nyRec || !d_Data_source || !d_Vp_w || !d_Data_synth)
        return nfail(PSDM_ERR_ARG, "null argument");
    if (prm->dPML < 2) return nfail(PSDM_ERR_ARG, "dPML must be >= 2 (got %d)", prm->dPML);
    if (prm->strategy != 1 && prm->strategy != 2)
        return nfail(PSDM_ERR_ARG, "strategy must be 1 (RAM) or 2 (disk) (got %d)", prm->strategy);
    if (NumRec < 1 || nt < 2 || ny < 1 || nx_w < 1)
        return nfail(PSDM_ERR_ARG, "need NumRec >= 1, nt >= 2 and a non-empty window");

    // Padded grid of the window, laid out as the engine lays it out.
    if (prm->dPML > kMaxDn - 2 * kAcc)
        return nfail(PSDM_ERR_ARG, "dPML %d too large for the fixed scratch (max %d)", prm->dPML, kMaxDn - 2 * kAcc);
    const Grid g = make_grid(prm->dPML, ny, nx_w);
    if (prm->strategy == 1 && nx_w < g.dn)
        return nfail(PSDM_ERR_ARG, "RAM ordering needs nx_w >= dPML+6 (nx_w=%d, dPML=%d)", nx_w, prm->dPML);
    if (g.dn > kMaxDn || g.cells() > kMaxCells || g.ldz > kMaxRows || g.nxt > kMaxCols || NumRec > kMaxRec)
        return nfail(PSDM_ERR_ARG,
                     "shot too large for the fixed scratch of the allocation-free modelling: padded grid %d x %d "
                     "(%zu cells incl. row alignment, max %zu; rows max %d, columns max %d), %d receivers (max %d), "
                     "dPML %d (max %d)",
                     g.ldz, g.nxt, g.cells(), kMaxCells, kMaxRows, kMaxCols, NumRec, kMaxRec, prm->dPML,
                     kMaxDn - 2 * kAcc);

    // Window coordinates (dynamic_window wrappers, src/dynamic_window.f90:80-86).
    int nx_wc = 0, x_i = 0, x_f = 0;
    psdm_dynamic_window(NumRec, nxSou, nxRec, dd, nx, dd_space, &nx_wc, &x_i, &x_f);
    if (nx_wc != nx_w)
        return nfail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, nx_wc);
    const int zs = g.dn + nySou - 1, xs = g.dn + (nxSou - x_i + 1) - 1;
    if (zs < 0 || zs >= g.nyt || xs < 0 || xs >= g.nxt)
        return nfail(PSDM_ERR_ARG, "source at padded (z=%d, x=%d) lies outside the %dx%d grid", zs, xs, g.nyt, g.nxt);
    for (int r = 0; r < NumRec; ++r) {
        const int zr = g.dn + nyRec[r] - 1, xr = g.dn + (nxRec[r] - x_i + 1) - 1;
        if (zr < 0 || zr >= g.nyt || xr < 0 || xr >= g.nxt)
            return nfail(PSDM_ERR_ARG, "receiver %d at padded (z=%d, x=%d) lies outside the %dx%d grid", r, zr, xr,
                         g.nyt, g.nxt);
    }
    // The reference adds the source on the interior only
    // (src/solver_ac_forward_ram.f90:443-444).
    const bool src_interior = zs >= g.dn && zs < g.dn + ny && xs >= g.dn && xs < g.dn + nx_w;

    int dev = 0, num_sms = 0;
    NA_CUDA(cudaGetDevice(&dev));
    NA_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    unsigned char* base = nullptr;
    {
        const int rc = scratch_address(dev, &base);
        if (rc) return rc;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    const size_t n = g.cells();
    Carve cv{base, 0};
    float* p[2] = {cv.take<float>(n), cv.take<float>(n)};
    float* c2 = cv.take<float>(n);
    float* phx[2] = {cv.take<float>(n), cv.take<float>(n)};
    float* chx = cv.take<float>(n);
    float* phz[2] = {cv.take<float>(n), cv.take<float>(n)};
    float* chz = cv.take<float>(n);
    float* side[2] = {cv.take<float>(g.nxt), cv.take<float>(g.nxt)};
    float* fA = cv.take<float>(g.dn);
    float* fB = cv.take<float>(g.dn);
    int* row_slot = cv.take<int>(g.ldz);
    int* inj_cols = cv.take<int>(g.nxt);
    int* rec_xy = cv.take<int>(2 * (size_t)NumRec);
    int* rec_cell = cv.take<int>(NumRec);
    int* counters = cv.take<int>(2);
    int* err = cv.take<int>(1);
    if (cv.off > kScratchBytes) return nfail(PSDM_ERR_ARG, "scratch layout exceeds its capacity");

    // The scratch holds whatever the previous call left.  Everything a step
    // reads before it writes is reset here: both wavefield levels, the C-PML
    // memory variables and their corner copies, the free-surface histories,
    // the tile counters and the error word (zero), and the injection map
    // (-1 = nothing).  c2, fA/fB, rec_xy and rec_cell are overwritten whole.
    // The output traces are cleared too, as psdm_model_shot does.
    for (float* b : {p[0], p[1], phx[0], phx[1], chx, phz[0], phz[1], chz})
        NA_CUDA(cudaMemsetAsync(b, 0, n * sizeof(float), st));
    NA_CUDA(cudaMemsetAsync(side[0], 0, g.nxt * sizeof(float), st));
    NA_CUDA(cudaMemsetAsync(side[1], 0, g.nxt * sizeof(float), st));
    NA_CUDA(cudaMemsetAsync(row_slot, 0xff, g.ldz * sizeof(int), st));
    NA_CUDA(cudaMemsetAsync(inj_cols, 0xff, g.nxt * sizeof(int), st));
    NA_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(int), st));
    NA_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    NA_CUDA(cudaMemsetAsync(d_Data_synth, 0, (size_t)NumRec * nt * sizeof(float), st));

    // C-PML profiles and receiver coordinates.  The copies come from host
    // memory that is not page-locked, so they are staged before
    // cudaMemcpyAsync returns and the stack arrays may go out of scope.
    float hA[kMaxDn], hB[kMaxDn];
    pml_profiles_f32(kAcc, g.dPML, dt, dd, g.dn, hA, hB);
    NA_CUDA(cudaMemcpyAsync(fA, hA, g.dn * sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CUDA(cudaMemcpyAsync(fB, hB, g.dn * sizeof(float), cudaMemcpyHostToDevice, st));
    NA_CUDA(cudaMemcpyAsync(rec_xy, nxRec, NumRec * sizeof(int), cudaMemcpyHostToDevice, st));
    NA_CUDA(cudaMemcpyAsync(rec_xy + NumRec, nyRec, NumRec * sizeof(int), cudaMemcpyHostToDevice, st));
    noalloc_geometry_kernel<<<(NumRec + 255) / 256, 256, 0, st>>>(row_slot, inj_cols, zs + g.zoff, xs,
                                                                  src_interior ? 1 : 0, rec_xy, rec_cell, NumRec,
                                                                  g.dn, x_i, g.ldz, g.zoff);
    NA_CUDA(cudaGetLastError());
    {
        const int rc = launch_pad_c2(d_Vp_w, ny, nx_w, g.dn, g.nyt, g.nxt, g.ldz, g.zoff, dt, dd,
                                     prm->strategy == 2 ? 0 : 1, c2, st);
        if (rc) return nfail(PSDM_ERR_CUDA, "pad_c2 launch: %s", cudaGetErrorString((cudaError_t)rc));
    }

    // Step arguments of a forward pass with receivers and no snapshots.
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.c2 = c2;
    a.chix = chx;
    a.chiz = chz;
    a.fA = fA;
    a.fB = fB;
    psdm_fd_coef(1, kAcc, a.cf1);
    psdm_fd_coef(2, kAcc, a.cf2);
    a.nyt = g.nyt;
    a.nxt = g.nxt;
    a.ldz = g.ldz;
    a.ny = g.ny;
    a.nx = g.nx;
    a.dn = g.dn;
    a.zoff = g.zoff;
    a.ldf = g.ldf;
    a.fs = prm->fs != 0;
    a.disk = prm->strategy == 2;
    a.dt = dt;
    a.ss = 1.f;
    a.field_w = 1.f;
    a.row_slot = row_slot;
    a.inj_cols = inj_cols;
    a.inj_trace = d_Data_source;
    a.inj_ld = 0;
    a.rec_cell = rec_cell;
    a.rec_out = d_Data_synth;
    a.nrec = NumRec;
    a.rec_ld = nt;
    a.tile_counter = counters;
    a.num_sms = num_sms;
    a.err = err;
    for (int i = 0; i < g.ldz; ++i) t_row_slot[i] = -1;
    if (src_interior) t_row_slot[zs + g.zoff] = 0;
    plan_tiles(&a, t_row_slot, false, true);

    // k = 2..nt (src/solver_ac_forward_ram.f90:344-577): source sample
    // S(k-1), receivers Rec(k-2) gathered from level k-1.
    for (int k = 2; k <= nt; ++k) {
        const int c = (k - 2) & 1;
        a.counter_sel = c;
        a.p = p[c];
        a.pm = p[c ^ 1];
        a.phix_in = phx[c];
        a.phix_out = phx[c ^ 1];
        a.phiz_in = phz[c];
        a.phiz_out = phz[c ^ 1];
        a.side_p = side[c];
        a.side_pm = side[c ^ 1];
        a.inj_t = k - 2;
        a.rec_t = k >= 3 ? k - 3 : -1;
        const int rc = launch_step(0, a, st);
        if (rc) return nfail(PSDM_ERR_CUDA, "forward step %d: %s", k, cudaGetErrorString((cudaError_t)rc));
    }
    {
        const int rc = launch_rec_final(rec_cell, p[(nt - 1) & 1], d_Data_synth, NumRec, nt, nt, st);
        if (rc) return nfail(PSDM_ERR_CUDA, "receiver gather: %s", cudaGetErrorString((cudaError_t)rc));
    }
    int herr = 0;
    NA_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    NA_CUDA(cudaStreamSynchronize(st));
    if (herr) return nfail(PSDM_ERR_CUDA, "%s", step_error_message(herr));
    return PSDM_OK;
}
