// RTM engine: device buffers, time loops and the C ABI (include/psdm_rtm.h).
//
// Host orchestration of one shot follows src/calculate_PSDM_RTM.f90:395-466
// and the solver wrappers of src/dynamic_window.f90:54-183.  Each time step
// is one fused kernel launch (rtm_step.cu); the snapshots of the forward
// pass stay in HBM for the backward pass.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/psdm_rtm.h"
#include "rtm_internal.h"

using namespace psdm;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                           \
    do {                                                                                         \
        cudaError_t e_ = (expr);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(e_ == cudaErrorMemoryAllocation ? PSDM_ERR_NOMEM : PSDM_ERR_CUDA,        \
                        "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__);    \
    } while (0)

#define TRY(expr)                  \
    do {                           \
        int r_ = (expr);           \
        if (r_ != PSDM_OK) return r_; \
    } while (0)

}  // namespace

struct psdm_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    struct Buf {
        void* ptr = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buf> bufs;

    // Grow-only named device buffer.
    int get(const char* name, size_t bytes, void** out) {
        Buf& b = bufs[name];
        if (b.bytes < bytes) {
            if (b.ptr) CUDA_TRY(cudaFree(b.ptr));
            b.ptr = nullptr;
            b.bytes = 0;
            CUDA_TRY(cudaMalloc(&b.ptr, std::max<size_t>(bytes, 256)));
            b.bytes = std::max<size_t>(bytes, 256);
        }
        *out = b.ptr;
        return PSDM_OK;
    }
    template <class T>
    int get(const char* name, size_t count, T** out) {
        return get(name, count * sizeof(T), reinterpret_cast<void**>(out));
    }
    int64_t total() const {
        int64_t s = 0;
        for (auto& kv : bufs) s += (int64_t)kv.second.bytes;
        return s;
    }
    int trim() {
        for (auto& kv : bufs)
            if (kv.second.ptr) CUDA_TRY(cudaFree(kv.second.ptr));
        bufs.clear();
        return PSDM_OK;
    }
};

namespace {

// Device state of one shot on the padded grid.
struct Shot {
    Grid g;
    float dt = 0.f, dd = 0.f;
    int fs = 0, disk = 0;
    float* p[2] = {nullptr, nullptr};
    float* c2 = nullptr;
    float* phx[2] = {nullptr, nullptr};
    float* chx = nullptr;
    float* phz[2] = {nullptr, nullptr};
    float* chz = nullptr;
    float* side[2] = {nullptr, nullptr};
    float* fA = nullptr;
    float* fB = nullptr;
    float cf1[4], cf2[4];
};

// Injection map (sources or adjoint sources at receivers), last write wins
// as in `source(nys(j),nxs(j)) = ...` (solver_ac_backward_ram.f90:333-336).
struct InjMap {
    std::vector<int> row_slot;
    std::vector<int> cols;
    int nslots = 0;
};

int check_params(const psdm_params* prm) {
    if (!prm) return fail(PSDM_ERR_ARG, "params is NULL");
    // The profile divides by the PML width (dPML-1)*d (solver_PML_coeffs.f90:13).
    if (prm->dPML < 2) return fail(PSDM_ERR_ARG, "dPML must be >= 2 (got %d)", prm->dPML);
    if (prm->strategy != 1 && prm->strategy != 2)
        return fail(PSDM_ERR_ARG, "strategy must be 1 (RAM) or 2 (disk) (got %d)", prm->strategy);
    return PSDM_OK;
}

int build_grid(const psdm_params* prm, int ny, int nx, Grid* g) {
    if (ny < 1 || nx < 1) return fail(PSDM_ERR_ARG, "grid must be at least 1x1 (ny=%d nx=%d)", ny, nx);
    g->ny = ny;
    g->nx = nx;
    g->dPML = prm->dPML;
    g->dn = prm->dPML + 2 * kAcc;
    g->nyt = g->dn + ny + g->dn;
    g->nxt = nx + 2 * g->dn;
    g->ldz = (g->nyt + 31) / 32 * 32;
    return PSDM_OK;
}

int setup_shot(psdm_engine* e, const psdm_params* prm, int ny, int nx, float dd, float dt, const float* h_vp,
               Shot* s) {
    TRY(build_grid(prm, ny, nx, &s->g));
    const Grid& g = s->g;
    // The RAM solvers' padding loops read ctmp(1, j) for j <= dn
    // (solver_ac_forward_ram.f90:288-293): a window narrower than dn would
    // read outside the model there.
    if (prm->strategy == 1 && nx < g.dn)
        return fail(PSDM_ERR_ARG, "RAM ordering needs nx_w >= dPML+6 (nx_w=%d, dPML=%d)", nx, prm->dPML);
    s->dt = dt;
    s->dd = dd;
    s->fs = prm->fs != 0;
    s->disk = prm->strategy == 2;
    const size_t n = g.cells();
    TRY(e->get("p0", n, &s->p[0]));
    TRY(e->get("p1", n, &s->p[1]));
    TRY(e->get("c2", n, &s->c2));
    TRY(e->get("phx0", n, &s->phx[0]));
    TRY(e->get("phx1", n, &s->phx[1]));
    TRY(e->get("chx", n, &s->chx));
    TRY(e->get("phz0", n, &s->phz[0]));
    TRY(e->get("phz1", n, &s->phz[1]));
    TRY(e->get("chz", n, &s->chz));
    TRY(e->get("side0", (size_t)g.nxt, &s->side[0]));
    TRY(e->get("side1", (size_t)g.nxt, &s->side[1]));
    TRY(e->get("fA", (size_t)g.dn, &s->fA));
    TRY(e->get("fB", (size_t)g.dn, &s->fB));
    float* d_vp = nullptr;
    TRY(e->get("vp", (size_t)ny * nx, &d_vp));

    std::vector<float> fA(g.dn), fB(g.dn);
    pml_profiles_f32(kAcc, g.dPML, dt, dd, g.dn, fA.data(), fB.data());
    psdm_fd_coef(1, kAcc, s->cf1);
    psdm_fd_coef(2, kAcc, s->cf2);

    cudaStream_t st = e->stream;
    CUDA_TRY(cudaMemcpyAsync(s->fA, fA.data(), g.dn * sizeof(float), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(s->fB, fB.data(), g.dn * sizeof(float), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(d_vp, h_vp, (size_t)ny * nx * sizeof(float), cudaMemcpyHostToDevice, st));
    for (float* b : {s->p[0], s->p[1], s->phx[0], s->phx[1], s->chx, s->phz[0], s->phz[1], s->chz})
        CUDA_TRY(cudaMemsetAsync(b, 0, n * sizeof(float), st));
    CUDA_TRY(cudaMemsetAsync(s->side[0], 0, g.nxt * sizeof(float), st));
    CUDA_TRY(cudaMemsetAsync(s->side[1], 0, g.nxt * sizeof(float), st));
    int rc = launch_pad_c2(d_vp, ny, nx, g.dn, g.nyt, g.nxt, g.ldz, dt, dd, s->disk ? 0 : 1, s->c2, st);
    if (rc) return fail(PSDM_ERR_CUDA, "pad_c2 launch: %s", cudaGetErrorString((cudaError_t)rc));
    return PSDM_OK;
}

// zs/xs: padded 0-based coordinates.  Points outside the padded grid are an
// error (the reference would index outside its arrays); points in the PML are
// kept out of the map because the reference adds `source` only on the
// interior (solver_ac_forward_ram.f90:443-444).
int build_inj(const Grid& g, int n, const int* zs, const int* xs, InjMap* m) {
    m->row_slot.assign(g.nyt, -1);
    m->cols.clear();
    m->nslots = 0;
    for (int j = 0; j < n; ++j) {
        const int z = zs[j], x = xs[j];
        if (z < 0 || z >= g.nyt || x < 0 || x >= g.nxt)
            return fail(PSDM_ERR_ARG, "injection point %d at padded (z=%d, x=%d) lies outside the %dx%d grid", j, z,
                        x, g.nyt, g.nxt);
        if (z < g.dn || z >= g.dn + g.ny || x < g.dn || x >= g.dn + g.nx) continue;
        if (m->row_slot[z] < 0) {
            m->row_slot[z] = m->nslots++;
            m->cols.resize((size_t)m->nslots * g.nxt, -1);
        }
        m->cols[(size_t)m->row_slot[z] * g.nxt + x] = j;
    }
    return PSDM_OK;
}

int upload_inj(psdm_engine* e, const Grid& g, const InjMap& m, int** d_row, int** d_cols) {
    TRY(e->get("inj_row", (size_t)g.nyt, d_row));
    TRY(e->get("inj_cols", std::max<size_t>(m.cols.size(), 1), d_cols));
    CUDA_TRY(cudaMemcpyAsync(*d_row, m.row_slot.data(), g.nyt * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    if (!m.cols.empty())
        CUDA_TRY(cudaMemcpyAsync(*d_cols, m.cols.data(), m.cols.size() * sizeof(int), cudaMemcpyHostToDevice,
                                 e->stream));
    return PSDM_OK;
}

StepArgs base_args(const Shot& s) {
    StepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.c2 = s.c2;
    a.chix = s.chx;
    a.chiz = s.chz;
    a.fA = s.fA;
    a.fB = s.fB;
    for (int i = 0; i < 4; ++i) { a.cf1[i] = s.cf1[i]; a.cf2[i] = s.cf2[i]; }
    a.nyt = s.g.nyt; a.nxt = s.g.nxt; a.ldz = s.g.ldz; a.ny = s.g.ny; a.nx = s.g.nx; a.dn = s.g.dn;
    a.fs = s.fs;
    a.disk = s.disk;
    a.dt = s.dt;
    a.rec_t = -1;
    a.ss = 1.f;
    a.field_w = 1.f;
    return a;
}

// Rotate ping-pong pointers for step number `it` (0 for k = 2).
void set_buffers(const Shot& s, int it, StepArgs* a) {
    const int c = it & 1;
    a->p = s.p[c];
    a->pm = s.p[c ^ 1];
    a->phix_in = s.phx[c];
    a->phix_out = s.phx[c ^ 1];
    a->phiz_in = s.phz[c];
    a->phiz_out = s.phz[c ^ 1];
    a->side_p = s.side[c];
    a->side_pm = s.side[c ^ 1];
}

// Forward pass over k = 2..nt (solver_ac_forward_ram.f90:344-577).
//   d_S: source trace (nt); d_fields: snapshot slots (nslots of ny*nx) or null;
//   d_rec: receiver traces (NumRec, nt) or null.
int run_forward(psdm_engine* e, Shot& s, int nt, int store_snap, const float* d_S, int zs, int xs,
                float* d_fields, int nslots, int nrec, const int* h_rec_cell, float* d_rec) {
    const Grid& g = s.g;
    InjMap inj;
    TRY(build_inj(g, 1, &zs, &xs, &inj));
    int *d_row = nullptr, *d_cols = nullptr;
    TRY(upload_inj(e, g, inj, &d_row, &d_cols));
    int* d_rec_cell = nullptr;
    if (d_rec && nrec > 0) {
        TRY(e->get("rec_cell", (size_t)nrec, &d_rec_cell));
        CUDA_TRY(cudaMemcpyAsync(d_rec_cell, h_rec_cell, nrec * sizeof(int), cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaMemsetAsync(d_rec, 0, (size_t)nrec * nt * sizeof(float), e->stream));
    }
    StepArgs a = base_args(s);
    a.row_slot = d_row;
    a.inj_cols = d_cols;
    a.inj_trace = d_S;
    a.inj_ld = 0;
    a.rec_cell = d_rec_cell;
    a.rec_out = d_rec;
    a.nrec = d_rec ? nrec : 0;
    a.rec_ld = nt;
    const size_t fstride = (size_t)g.ny * g.nx;
    for (int k = 2; k <= nt; ++k) {
        const int it = k - 2;
        set_buffers(s, it, &a);
        a.inj_t = k - 2;                        // S(k-1)
        a.rec_t = (d_rec && k >= 3) ? k - 3 : -1;  // Rec(k-2) from p = level k-1
        a.field = nullptr;
        if (d_fields && (k - 1) % store_snap == 0) {
            const int snap = (k - 1) / store_snap;  // 1-based slot
            if (snap > nslots) return fail(PSDM_ERR_ARG, "snapshot slot %d exceeds nt_snap=%d", snap, nslots);
            a.field = d_fields + (size_t)(snap - 1) * fstride;
        }
        int rc = launch_step(0, a, e->stream);
        if (rc) return fail(PSDM_ERR_CUDA, "forward step %d: %s", k, cudaGetErrorString((cudaError_t)rc));
    }
    if (d_rec && nrec > 0 && nt >= 2) {
        const float* pfin = s.p[(nt - 1) & 1];  // p3 of the last step
        int rc = launch_rec_final(d_rec_cell, pfin, d_rec, nrec, nt, nt, e->stream);
        if (rc) return fail(PSDM_ERR_CUDA, "receiver gather: %s", cudaGetErrorString((cudaError_t)rc));
    }
    return PSDM_OK;
}

// Backward pass over k = 2..nt (solver_ac_backward_ram.f90:329-545).
//   d_back: adjoint traces (nt, NumRec); snapshots: slot `snap` (1-based) is
//   d_fields + (snap - slot_lo) * ny*nx when slot_lo <= snap <= slot_hi, and
//   zero otherwise; h_w[snap - 1] is the taper weight of slot `snap`
//   (size nt_snap, may be null for all-ones).
int run_backward(psdm_engine* e, Shot& s, int nt, int store_snap, int nt_snap, const float* d_back, int nrec,
                 const int* zr, const int* xr, const float* d_fields, int slot_lo, int slot_hi,
                 const float* h_w, float* d_image) {
    const Grid& g = s.g;
    InjMap inj;
    TRY(build_inj(g, nrec, zr, xr, &inj));
    int *d_row = nullptr, *d_cols = nullptr;
    TRY(upload_inj(e, g, inj, &d_row, &d_cols));
    StepArgs a = base_args(s);
    a.row_slot = d_row;
    a.inj_cols = d_cols;
    a.inj_trace = d_back;
    a.inj_ld = nt;
    a.image = d_image;
    a.ss = float(store_snap);
    const size_t fstride = (size_t)g.ny * g.nx;
    int snap = nt_snap;
    for (int k = 2; k <= nt; ++k) {
        const int it = k - 2;
        set_buffers(s, it, &a);
        a.inj_t = k - 2;  // Sadj(k-1)
        a.field = nullptr;
        if ((k - 1) % store_snap == 0) {
            snap = snap - 1;
            if (d_fields && snap >= slot_lo && snap <= slot_hi && snap >= 1) {
                a.field = const_cast<float*>(d_fields) + (size_t)(snap - slot_lo) * fstride;
                a.field_w = h_w ? h_w[snap - 1] : 1.f;
                if (a.field_w == 0.f) a.field = nullptr;  // zero-padded slot: no contribution
            }
        }
        int rc = launch_step(1, a, e->stream);
        if (rc) return fail(PSDM_ERR_CUDA, "backward step %d: %s", k, cudaGetErrorString((cudaError_t)rc));
    }
    return PSDM_OK;
}

int check_engine(psdm_engine* e) {
    if (!e) return fail(PSDM_ERR_STATE, "engine is NULL");
    CUDA_TRY(cudaSetDevice(e->device));
    return PSDM_OK;
}

int sync(psdm_engine* e) {
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return PSDM_OK;
}

// Window coordinates of a shot (dynamic_window wrappers,
// src/dynamic_window.f90:80-86): x_i from the model-coordinate geometry.
struct WinGeom {
    int x_i = 1, nx_w_calc = 0;
    int zs = 0, xs = 0;               // padded 0-based source
    std::vector<int> zr, xr;          // padded 0-based receivers
    std::vector<int> rec_cell;        // xr*ldz + zr
};

int window_geometry(const Grid& g, int NumRec, int nxSou, int nySou, const int* nxRec, const int* nyRec, float dd,
                    int nx_model, float dd_space, WinGeom* w) {
    int nx_w = 0, x_i = 0, x_f = 0;
    psdm_dynamic_window(NumRec, nxSou, nxRec, dd, nx_model, dd_space, &nx_w, &x_i, &x_f);
    w->x_i = x_i;
    w->nx_w_calc = nx_w;
    w->zs = g.dn + nySou - 1;
    w->xs = g.dn + (nxSou - x_i + 1) - 1;
    w->zr.resize(NumRec);
    w->xr.resize(NumRec);
    w->rec_cell.resize(NumRec);
    for (int r = 0; r < NumRec; ++r) {
        w->zr[r] = g.dn + nyRec[r] - 1;
        w->xr[r] = g.dn + (nxRec[r] - x_i + 1) - 1;
        if (w->zr[r] < 0 || w->zr[r] >= g.nyt || w->xr[r] < 0 || w->xr[r] >= g.nxt)
            return fail(PSDM_ERR_ARG, "receiver %d at padded (z=%d, x=%d) lies outside the %dx%d grid", r, w->zr[r],
                        w->xr[r], g.nyt, g.nxt);
        w->rec_cell[r] = w->xr[r] * g.ldz + w->zr[r];
    }
    return PSDM_OK;
}

}  // namespace

extern "C" {

const char* psdm_last_error(void) { return g_last_error.c_str(); }

int psdm_engine_create(int32_t device, psdm_engine** out) {
    if (!out) return fail(PSDM_ERR_ARG, "out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t err = cudaGetDeviceCount(&n);
    if (err != cudaSuccess || n <= 0)
        return fail(PSDM_ERR_CUDA, "no CUDA device available (%s); the engine has no CPU fallback",
                    err != cudaSuccess ? cudaGetErrorString(err) : "0 devices");
    if (device < 0 || device >= n) return fail(PSDM_ERR_ARG, "device %d out of range (%d devices)", device, n);
    CUDA_TRY(cudaSetDevice(device));
    psdm_engine* e = new psdm_engine();
    e->device = device;
    err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        delete e;
        return fail(PSDM_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(err));
    }
    *out = e;
    return PSDM_OK;
}

int psdm_engine_destroy(psdm_engine* e) {
    if (!e) return PSDM_OK;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    int rc = e->trim();
    cudaStreamDestroy(e->stream);
    delete e;
    return rc;
}

int64_t psdm_engine_device_bytes(const psdm_engine* e) { return e ? e->total() : 0; }

int psdm_engine_trim(psdm_engine* e) {
    TRY(check_engine(e));
    TRY(sync(e));
    return e->trim();
}

int psdm_dynamic_window_solver_forward_ram(psdm_engine* e, const psdm_params* prm, int32_t NumRec,
                                           const int32_t* nxSou, const int32_t* nySou, const int32_t* nxRec,
                                           const int32_t* nyRec, const float* Data_source, float dd, float dt,
                                           int32_t ny, int32_t nx, int32_t nx_w, const float* Vp_w, float dd_space,
                                           int32_t store_snap, int32_t nt_snap, int32_t nt, float* Fields,
                                           float* Data_synth) {
    TRY(check_engine(e));
    TRY(check_params(prm));
    if (prm->precision != PSDM_PREC_FP32) return fail(PSDM_ERR_ARG, "the *_ram entry points are FP32 only");
    if (NumRec < 0 || !nxSou || !nySou || !Data_source || !Vp_w || (NumRec > 0 && (!nxRec || !nyRec)))
        return fail(PSDM_ERR_ARG, "null argument");
    if (nt < 2 || store_snap < 1 || nt_snap < 0) return fail(PSDM_ERR_ARG, "need nt >= 2, store_snap >= 1");
    Shot s;
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, Vp_w, &s));
    WinGeom w;
    TRY(window_geometry(s.g, NumRec, nxSou[0], nySou[0], nxRec, nyRec, dd, nx, dd_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    float *d_S = nullptr, *d_F = nullptr, *d_rec = nullptr;
    TRY(e->get("S", (size_t)nt, &d_S));
    CUDA_TRY(cudaMemcpyAsync(d_S, Data_source, nt * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    const int nsnap = (nt - 1) / store_snap;
    if (Fields && nsnap > nt_snap) return fail(PSDM_ERR_ARG, "nt_snap=%d < %d snapshots", nt_snap, nsnap);
    const size_t fstride = (size_t)ny * nx_w;
    if (Fields && nsnap > 0) TRY(e->get("fields", fstride * nsnap, &d_F));
    if (Data_synth && NumRec > 0) TRY(e->get("rec", (size_t)NumRec * nt, &d_rec));
    TRY(run_forward(e, s, nt, store_snap, d_S, w.zs, w.xs, d_F, nsnap, NumRec, w.rec_cell.data(), d_rec));
    if (d_F)
        CUDA_TRY(cudaMemcpyAsync(Fields, d_F, fstride * nsnap * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    if (d_rec)
        CUDA_TRY(cudaMemcpyAsync(Data_synth, d_rec, (size_t)NumRec * nt * sizeof(float), cudaMemcpyDeviceToHost,
                                 e->stream));
    return sync(e);
}

int psdm_dynamic_window_solver_backward_ram(psdm_engine* e, const psdm_params* prm, int32_t NumRec,
                                            const int32_t* nxSou, const int32_t* nySou, const int32_t* nxRec,
                                            const int32_t* nyRec, const float* AdjSource, float dd, float dt,
                                            int32_t ny, int32_t nx, int32_t nx_w, const float* Vp_w,
                                            float dd_space, int32_t store_snap, int32_t nt_snap, int32_t nt,
                                            const float* Fields, float* PSDM_thread) {
    TRY(check_engine(e));
    TRY(check_params(prm));
    if (prm->precision != PSDM_PREC_FP32) return fail(PSDM_ERR_ARG, "the *_ram entry points are FP32 only");
    if (NumRec < 0 || !nxSou || !nySou || !Vp_w || !PSDM_thread || (NumRec > 0 && (!nxRec || !nyRec || !AdjSource)))
        return fail(PSDM_ERR_ARG, "null argument");
    if (nt < 2 || store_snap < 1) return fail(PSDM_ERR_ARG, "need nt >= 2, store_snap >= 1");
    Shot s;
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, Vp_w, &s));
    WinGeom w;
    TRY(window_geometry(s.g, NumRec, nxSou[0], nySou[0], nxRec, nyRec, dd, nx, dd_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    // Slots read: nt_snap - m for m = 1..(nt-1)/store_snap, clipped to [1, nt_snap].
    const int nimg = (nt - 1) / store_snap;
    const int lo = std::max(1, nt_snap - nimg), hi = nt_snap - 1;
    if (nt_snap - nimg < 1 && nimg > 0 && Fields)
        return fail(PSDM_ERR_ARG, "imaging would read snapshot slot %d < 1 (nt_snap=%d)", nt_snap - nimg, nt_snap);
    const size_t fstride = (size_t)ny * nx_w;
    float *d_back = nullptr, *d_F = nullptr, *d_img = nullptr;
    if (NumRec > 0) {
        TRY(e->get("back", (size_t)NumRec * nt, &d_back));
        CUDA_TRY(cudaMemcpyAsync(d_back, AdjSource, (size_t)NumRec * nt * sizeof(float), cudaMemcpyHostToDevice,
                                 e->stream));
    }
    if (Fields && hi >= lo) {
        TRY(e->get("fields", fstride * (hi - lo + 1), &d_F));
        CUDA_TRY(cudaMemcpyAsync(d_F, Fields + (size_t)(lo - 1) * fstride, fstride * (hi - lo + 1) * sizeof(float),
                                 cudaMemcpyHostToDevice, e->stream));
    }
    TRY(e->get("image", fstride, &d_img));
    CUDA_TRY(cudaMemcpyAsync(d_img, PSDM_thread, fstride * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    TRY(run_backward(e, s, nt, store_snap, nt_snap, d_back, NumRec, w.zr.data(), w.xr.data(), d_F, lo, hi, nullptr,
                     d_img));
    CUDA_TRY(cudaMemcpyAsync(PSDM_thread, d_img, fstride * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    return sync(e);
}

int psdm_rtm_shot(psdm_engine* e, const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
                  const int32_t* nxRec, const int32_t* nyRec, const float* Data_source, const float* Data_target,
                  float dd, float dt, int32_t ny, int32_t nx, int32_t nx_w, const float* Vp_w, float added_space,
                  int32_t store_snap, int32_t nt_snap, int32_t nt_prop2, int32_t nt_taper, int32_t taper_option,
                  int32_t N_taper, int32_t N_zeros, float* PSDM_w) {
    TRY(check_engine(e));
    TRY(check_params(prm));
    if (prm->precision != PSDM_PREC_FP32) return fail(PSDM_ERR_ARG, "mixed precision is not built yet");
    if (NumRec < 1 || !nxRec || !nyRec || !Data_source || !Data_target || !Vp_w || !PSDM_w)
        return fail(PSDM_ERR_ARG, "null argument or NumRec < 1");
    if (nt_prop2 < 2 || nt_taper < 2 || store_snap < 1 || nt_taper < nt_prop2)
        return fail(PSDM_ERR_ARG, "need 2 <= nt_prop2 <= nt_taper and store_snap >= 1");
    if (taper_option != 0 && N_taper < 1) return fail(PSDM_ERR_ARG, "N_taper must be >= 1");
    Shot s;
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, Vp_w, &s));
    WinGeom w;
    TRY(window_geometry(s.g, NumRec, nxSou, nySou, nxRec, nyRec, dd, nx, added_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    const size_t fstride = (size_t)ny * nx_w;
    const int nsnap = (nt_prop2 - 1) / store_snap;  // slots written by the forward pass
    float *d_S = nullptr, *d_F = nullptr, *d_back = nullptr, *d_img = nullptr;
    TRY(e->get("S", (size_t)nt_prop2, &d_S));
    CUDA_TRY(cudaMemcpyAsync(d_S, Data_source, nt_prop2 * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    if (nsnap > 0) TRY(e->get("fields", fstride * nsnap, &d_F));
    TRY(run_forward(e, s, nt_prop2, store_snap, d_S, w.zs, w.xs, d_F, nsnap, 0, nullptr, nullptr));

    // Taper of the snapshot series (calculate_PSDM_RTM.f90:421-427): a weight
    // per slot, applied when the slot is read.
    std::vector<float> wts(std::max(nt_taper, 1), 1.f);
    if (taper_option != 0) {
        const int i0 = std::max(1, nt_prop2 - N_taper + 1);
        for (int n = 0; n < N_taper; ++n)
            if (i0 + n <= nt_prop2) wts[i0 + n - 1] = taper_weight(n, N_taper);
        if (N_zeros > 0)
            for (int i = nt_prop2; i < nt_taper; ++i) wts[i] = 0.f;
    }
    // BackSource(:,j) = Data_target(nt_taper:1:-1, j) (:448-450).
    std::vector<float> back((size_t)NumRec * nt_taper);
    for (int r = 0; r < NumRec; ++r)
        for (int t = 0; t < nt_taper; ++t)
            back[(size_t)r * nt_taper + t] = Data_target[(size_t)r * nt_taper + (nt_taper - 1 - t)];
    TRY(e->get("back", back.size(), &d_back));
    CUDA_TRY(cudaMemcpyAsync(d_back, back.data(), back.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    TRY(e->get("image", fstride, &d_img));
    CUDA_TRY(cudaMemsetAsync(d_img, 0, fstride * sizeof(float), e->stream));
    // Second propagator call: nt_snap = nt = nt_taper (:456-458).
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, Vp_w, &s));
    TRY(run_backward(e, s, nt_taper, store_snap, nt_taper, d_back, NumRec, w.zr.data(), w.xr.data(), d_F, 1, nsnap,
                     wts.data(), d_img));
    CUDA_TRY(cudaMemcpyAsync(PSDM_w, d_img, fstride * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    return sync(e);
}

int psdm_model_shot(psdm_engine* e, const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
                    const int32_t* nxRec, const int32_t* nyRec, const float* Data_source, float dd, float dt,
                    int32_t ny, int32_t nx, int32_t nx_w, const float* Vp_w, float dd_space, int32_t nt,
                    float* Data_synth) {
    TRY(check_engine(e));
    TRY(check_params(prm));
    if (NumRec < 1 || !nxRec || !nyRec || !Data_source || !Vp_w || !Data_synth)
        return fail(PSDM_ERR_ARG, "null argument or NumRec < 1");
    if (nt < 2) return fail(PSDM_ERR_ARG, "need nt >= 2");
    Shot s;
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, Vp_w, &s));
    WinGeom w;
    TRY(window_geometry(s.g, NumRec, nxSou, nySou, nxRec, nyRec, dd, nx, dd_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    float *d_S = nullptr, *d_rec = nullptr;
    TRY(e->get("S", (size_t)nt, &d_S));
    CUDA_TRY(cudaMemcpyAsync(d_S, Data_source, nt * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    TRY(e->get("rec", (size_t)NumRec * nt, &d_rec));
    TRY(run_forward(e, s, nt, 1, d_S, w.zs, w.xs, nullptr, 0, NumRec, w.rec_cell.data(), d_rec));
    CUDA_TRY(cudaMemcpyAsync(Data_synth, d_rec, (size_t)NumRec * nt * sizeof(float), cudaMemcpyDeviceToHost,
                             e->stream));
    return sync(e);
}

}  // extern "C"
