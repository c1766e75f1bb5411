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
#include <array>
#include <complex>
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

#define TRY(expr)                     \
    do {                              \
        int r_ = (expr);              \
        if (r_ != PSDM_OK) return r_; \
    } while (0)

}  // namespace

void psdm::set_last_error(const char* msg) { g_last_error = msg; }

struct psdm_engine {
    int device = 0;
    int num_sms = 148;
    // Kernels that give up waiting for their copies set this word (host
    // memory mapped into the device); checked after each synchronisation.
    volatile int* h_err = nullptr;
    int* d_err = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;  // own_stream or the caller's
    struct Buf {
        void* ptr = nullptr;
        size_t bytes = 0;
    };
    std::map<std::string, Buf> bufs;
    // statistics
    int64_t launches = 0;
    int64_t fwd_steps = 0, bwd_steps = 0;
    bool profiling = false;
    std::vector<cudaEvent_t> events;  // triples (start, forward done, backward done)
    size_t events_used = 0;
    // Captured step loops, one per pass kind (forward / backward), replayed
    // while every launch argument is unchanged.
    struct GraphCache {
        std::vector<StepArgs> args;
        cudaGraphExec_t exec = nullptr;
    } graphs[3];
    bool use_graphs = true;
    // Time steps per launch: 1 (default, the faster form on the B200) = one
    // launch per step, 2 = pair launches (rtm_pair.cu).  Captured pair loops,
    // one per pass kind.
    int steps_per_launch = 1;
    struct PairGraphCache {
        std::vector<PairArgs> args;
        cudaGraphExec_t exec = nullptr;
    } pgraphs[3];
    // Passes of one shot as one cooperative launch each where the pass allows
    // it: 1 = pass_kernel (tiles re-read every step), 2 = res_kernel (regions
    // resident in shared memory); the neighbour, receiver and work lists of
    // the last plan of each pass kind stay on the device while the plan (key)
    // is unchanged.
    int use_pass = 0;
    std::vector<int> pass_key[3];  // by pass kind (mode)
    std::vector<int> res_key[2];   // resident form, by pass kind
    int res_nreg[2] = {0, 0}, res_sw[2] = {0, 0};
    cudaEvent_t pass_staged[3] = {nullptr, nullptr, nullptr};  // copies out of the staging buffers done
    int batch_slots = 0;  // slots used by the last batched call
    int ckpt_interval = 0;  // > 0: shots keep checkpoints every K steps instead of all snapshots
    std::map<int, cudaGraphExec_t> bgraphs;  // batched launches: an executable graph per run length
    bool recon = false;     // FP32 shots reconstruct the source wavefield from a saved band
    std::map<std::pair<int, int>, std::array<int, 2>> fft_plans;  // (length, batch) -> cuFFT plans
    // dt -> (fast division exact, 1/dt, lo, hi); the check costs ~50 ms
    std::map<float, std::pair<int, std::vector<float>>> div_cache;

    // Grow-only named device buffer.
    int get(const char* name, size_t bytes, void** out) {
        Buf& b = bufs[name];
        if (b.bytes < bytes) {
            if (b.ptr) {
                CUDA_TRY(cudaStreamSynchronize(stream));
                drop_graphs();  // captured launches may reference this buffer
                CUDA_TRY(cudaFree(b.ptr));
            }
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
    // Grow-only named page-locked host buffer (staging of batched shots).
    std::map<std::string, Buf> pinned;
    int get_pinned(const char* name, size_t bytes, void** out) {
        Buf& b = pinned[name];
        if (b.bytes < bytes) {
            if (b.ptr) {
                CUDA_TRY(cudaStreamSynchronize(stream));
                CUDA_TRY(cudaFreeHost(b.ptr));
            }
            b.ptr = nullptr;
            b.bytes = 0;
            CUDA_TRY(cudaMallocHost(&b.ptr, std::max<size_t>(bytes, 256)));
            b.bytes = std::max<size_t>(bytes, 256);
        }
        *out = b.ptr;
        return PSDM_OK;
    }
    int64_t total() const {
        int64_t s = 0;
        for (auto& kv : bufs) s += (int64_t)kv.second.bytes;
        return s;
    }
    int trim() {
        drop_graphs();
        for (auto& k : pass_key) k.clear();
        for (auto& k : res_key) k.clear();
        for (auto& kv : fft_plans) destroy_fft_plans(kv.second.data());
        fft_plans.clear();
        for (auto& kv : bufs)
            if (kv.second.ptr) CUDA_TRY(cudaFree(kv.second.ptr));
        bufs.clear();
        for (auto& kv : pinned)
            if (kv.second.ptr) CUDA_TRY(cudaFreeHost(kv.second.ptr));
        pinned.clear();
        return PSDM_OK;
    }
    void drop_graphs() {
        for (auto& kv : bgraphs)
            if (kv.second) cudaGraphExecDestroy(kv.second);
        bgraphs.clear();
        for (auto& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
            g.args.clear();
        }
        for (auto& g : pgraphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
            g.args.clear();
        }
    }
    // Profiling marks: 0 = shot start, 1 = forward done, 2 = backward done.
    int record(int which) {
        if (!profiling) return PSDM_OK;
        if (which == 0 && events_used + 3 > events.size())
            for (int i = 0; i < 3; ++i) {
                cudaEvent_t ev;
                CUDA_TRY(cudaEventCreate(&ev));
                events.push_back(ev);
            }
        const size_t idx = (which == 0) ? events_used : events_used - 3 + which;
        CUDA_TRY(cudaEventRecord(events[idx], stream));
        if (which == 0) events_used += 3;
        return PSDM_OK;
    }
};

namespace {

// Device state of one shot on the padded grid.
struct Shot {
    Grid g;
    float dt = 0.f, dd = 0.f;
    int fs = 0, disk = 0;
    // p[0], p[1]: the two levels of one launch per step (p1 overwritten in
    // place); p[2] and p[3] for launches of two steps, whose wavefield
    // rotates through all four.
    float* p[4] = {nullptr, nullptr, nullptr, nullptr};
    float* c2 = nullptr;
    float* phx[2] = {nullptr, nullptr};
    float* chx = nullptr;
    float* chx2 = nullptr;  // second chi buffers (launches of two steps)
    float* phz[2] = {nullptr, nullptr};
    float* chz = nullptr;
    float* chz2 = nullptr;
    float* side[4] = {nullptr, nullptr, nullptr, nullptr};
    float* fA = nullptr;
    float* fB = nullptr;
    float cf1[4], cf2[4];
    float inv_dt = 0.f, div_lo = 0.f, div_hi = 0.f, div_tiny = 0.f;
    int fast_div = 0;
    int* counters = nullptr;  // two tile counters, alternating per step
    int num_sms = 0;
    int* err = nullptr;       // device view of the engine's error word
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
    *g = make_grid(prm->dPML, ny, nx);
    return PSDM_OK;
}

// Zero the wavefield, memory variables and free-surface histories.
int reset_state(psdm_engine* e, Shot* s) {
    const size_t n = s->g.cells();
    for (float* b : {s->p[0], s->p[1], s->p[2], s->p[3], s->phx[0], s->phx[1], s->chx, s->chx2, s->phz[0], s->phz[1],
                     s->chz, s->chz2})
        CUDA_TRY(cudaMemsetAsync(b, 0, n * sizeof(float), e->stream));
    for (float* b : s->side) CUDA_TRY(cudaMemsetAsync(b, 0, s->g.nxt * sizeof(float), e->stream));
    CUDA_TRY(cudaMemsetAsync(s->counters, 0, 2 * sizeof(int), e->stream));
    return PSDM_OK;
}

// Allocate and initialise the state of a shot from a window model already in
// device memory (d_vp, (ny, nx) column-major).
int setup_shot(psdm_engine* e, const psdm_params* prm, int ny, int nx, float dd, float dt, const float* d_vp,
               Shot* s, const std::string& tag = "") {
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
    for (int i = 0; i < 4; ++i) TRY(e->get(("p" + std::to_string(i) + tag).c_str(), n, &s->p[i]));
    TRY(e->get(("c2" + tag).c_str(), n, &s->c2));
    TRY(e->get(("phx0" + tag).c_str(), n, &s->phx[0]));
    TRY(e->get(("phx1" + tag).c_str(), n, &s->phx[1]));
    TRY(e->get(("chx" + tag).c_str(), n, &s->chx));
    TRY(e->get(("chx2" + tag).c_str(), n, &s->chx2));
    TRY(e->get(("phz0" + tag).c_str(), n, &s->phz[0]));
    TRY(e->get(("phz1" + tag).c_str(), n, &s->phz[1]));
    TRY(e->get(("chz" + tag).c_str(), n, &s->chz));
    TRY(e->get(("chz2" + tag).c_str(), n, &s->chz2));
    for (int i = 0; i < 4; ++i)
        TRY(e->get(("side" + std::to_string(i) + tag).c_str(), (size_t)g.nxt, &s->side[i]));
    TRY(e->get(("fA" + tag).c_str(), (size_t)g.dn, &s->fA));
    TRY(e->get(("fB" + tag).c_str(), (size_t)g.dn, &s->fB));
    TRY(e->get(("tile_counters" + tag).c_str(), 2, &s->counters));
    s->num_sms = e->num_sms;
    s->err = e->d_err;

    std::vector<float> fA(g.dn), fB(g.dn);
    if (prm->precision == PSDM_PREC_FP32) {  // the reference's single-precision set-up
        pml_profiles_f32(kAcc, g.dPML, dt, dd, g.dn, fA.data(), fB.data());
        psdm_fd_coef(1, kAcc, s->cf1);
        psdm_fd_coef(2, kAcc, s->cf2);
    } else {  // mixed precision: FD coefficients and C-PML profiles in double, rounded once
        std::vector<double> a64(g.dn), b64(g.dn);
        pml_profiles_f64(kAcc, g.dPML, (double)dt, (double)dd, g.dn, a64.data(), b64.data());
        for (int i = 0; i < g.dn; ++i) {
            fA[i] = (float)a64[i];
            fB[i] = (float)b64[i];
        }
        double c1[4], c2[4];
        fd_coef_f64(1, c1);
        fd_coef_f64(2, c2);
        for (int k = 0; k < 4; ++k) {
            s->cf1[k] = (float)c1[k];
            s->cf2[k] = (float)c2[k];
        }
    }
    auto it = e->div_cache.find(dt);
    if (it == e->div_cache.end()) {
        float r = 0.f, lo = 0.f, hi = 0.f, tiny = 0.f;
        const int ok = fast_div_exact(dt, &r, &lo, &hi, &tiny) ? 1 : 0;
        it = e->div_cache.emplace(dt, std::make_pair(ok, std::vector<float>{r, lo, hi, tiny})).first;
    }
    s->fast_div = it->second.first;
    s->inv_dt = it->second.second[0];
    s->div_lo = it->second.second[1];
    s->div_hi = it->second.second[2];
    s->div_tiny = it->second.second[3];

    CUDA_TRY(cudaMemcpyAsync(s->fA, fA.data(), g.dn * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(s->fB, fB.data(), g.dn * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    TRY(reset_state(e, s));
    int rc = launch_pad_c2(d_vp, ny, nx, g.dn, g.nyt, g.nxt, g.ldz, g.zoff, dt, dd, s->disk ? 0 : 1, s->c2,
                           e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "pad_c2 launch: %s", cudaGetErrorString((cudaError_t)rc));
    e->launches += 1;
    return PSDM_OK;
}

// Same, uploading the window model from host memory first.
int setup_shot_host(psdm_engine* e, const psdm_params* prm, int ny, int nx, float dd, float dt, const float* h_vp,
                    Shot* s) {
    float* d_vp = nullptr;
    TRY(e->get("vp", (size_t)ny * nx, &d_vp));
    CUDA_TRY(cudaMemcpyAsync(d_vp, h_vp, (size_t)ny * nx * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    return setup_shot(e, prm, ny, nx, dd, dt, d_vp, s);
}

// zs/xs: padded 0-based coordinates.  Points outside the padded grid are an
// error (the reference would index outside its arrays); points in the PML are
// kept out of the map because the reference adds `source` only on the
// interior (solver_ac_forward_ram.f90:443-444).
int build_inj(const Grid& g, int n, const int* zs, const int* xs, InjMap* m) {
    m->row_slot.assign(g.ldz, -1);
    m->cols.clear();
    m->nslots = 0;
    for (int j = 0; j < n; ++j) {
        const int z = zs[j], x = xs[j];
        if (z < 0 || z >= g.nyt || x < 0 || x >= g.nxt)
            return fail(PSDM_ERR_ARG, "injection point %d at padded (z=%d, x=%d) lies outside the %dx%d grid", j, z,
                        x, g.nyt, g.nxt);
        if (z < g.dn || z >= g.dn + g.ny || x < g.dn || x >= g.dn + g.nx) continue;
        const int zd = z + g.zoff;
        if (m->row_slot[zd] < 0) {
            m->row_slot[zd] = m->nslots++;
            m->cols.resize((size_t)m->nslots * g.nxt, -1);
        }
        m->cols[(size_t)m->row_slot[zd] * g.nxt + x] = j;
    }
    return PSDM_OK;
}

// Pageable-host sources are staged by cudaMemcpyAsync before it returns, so
// the vectors may be released right after.
int upload_inj(psdm_engine* e, const Grid& g, const InjMap& m, const char* tag, int** d_row, int** d_cols) {
    const std::string rn = std::string("inj_row_") + tag, cn = std::string("inj_cols_") + tag;
    TRY(e->get(rn.c_str(), (size_t)g.ldz, d_row));
    TRY(e->get(cn.c_str(), std::max<size_t>(m.cols.size(), 1), d_cols));
    CUDA_TRY(cudaMemcpyAsync(*d_row, m.row_slot.data(), g.ldz * sizeof(int), cudaMemcpyHostToDevice, e->stream));
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
    a.zoff = s.g.zoff; a.ldf = s.g.ldf;
    a.fs = s.fs;
    a.tile_counter = s.counters;
    a.num_sms = s.num_sms;
    a.err = s.err;
    a.fs = s.fs;
    a.disk = s.disk;
    a.dt = s.dt;
    a.inv_dt = s.inv_dt;
    a.div_lo = s.div_lo;
    a.div_hi = s.div_hi;
    a.div_tiny = s.div_tiny;
    a.fast_div = s.fast_div;
    a.rec_t = -1;
    a.ss = 1.f;
    a.field_w = 1.f;
    return a;
}

// Rotate ping-pong pointers for step number `it` (0 for k = 2).
void set_buffers(const Shot& s, int it, StepArgs* a) {
    const int c = it & 1;
    a->counter_sel = c;
    a->p = s.p[c];
    a->pm = s.p[c ^ 1];
    a->phix_in = s.phx[c];
    a->phix_out = s.phx[c ^ 1];
    a->phiz_in = s.phz[c];
    a->phiz_out = s.phz[c ^ 1];
    a->side_p = s.side[c];
    a->side_pm = s.side[c ^ 1];
}

// The steps of a pass as the pass kernel's input: the arguments of the first
// two steps as parity bases, and the values that change from step to step.
// False when steps differ in anything else, or when a step reduces over the
// whole grid (the mixed form's per-snapshot maximum and its conversion), which
// the pass kernel's tile-by-tile progress cannot order.
bool pass_form(const std::vector<StepArgs>& args, StepArgs base[2], std::vector<PassVar>* var) {
    const size_t n = args.size();
    base[0] = args[0];
    base[1] = n > 1 ? args[1] : args[0];
    var->assign(n, PassVar{});
    for (size_t i = 0; i < n; ++i) {
        const StepArgs& a = args[i];
        if (a.q_src != nullptr || a.field_amax != nullptr) return false;
        if (a.counter_sel != (int)(i & 1)) return false;
        PassVar& v = (*var)[i];
        v.field = a.field;
        v.field16 = a.field16;
        v.field_iscale = a.field_iscale;
        v.field_w = a.field_w;
        v.inj_t = a.inj_t;
        v.rec_t = a.rec_t;
        v.par = (int)(i & 1);
        const StepArgs& b = base[i & 1];
        StepArgs t = a;
        t.field = b.field;
        t.field16 = b.field16;
        t.field_iscale = b.field_iscale;
        t.field_w = b.field_w;
        t.inj_t = b.inj_t;
        t.rec_t = b.rec_t;
        if (std::memcmp(&t, &b, sizeof(StepArgs)) != 0) return false;
    }
    const StepArgs &b0 = base[0], &b1 = base[1];
    return b0.nrect == b1.nrect && b0.itx == b1.itx && b0.ixb == b1.ixb &&
           std::memcmp(b0.r_type, b1.r_type, sizeof b0.r_type) == 0 &&
           std::memcmp(b0.r_zd0, b1.r_zd0, sizeof b0.r_zd0) == 0 && std::memcmp(b0.r_x0, b1.r_x0, sizeof b0.r_x0) == 0 &&
           std::memcmp(b0.r_h, b1.r_h, sizeof b0.r_h) == 0 && std::memcmp(b0.r_w, b1.r_w, sizeof b0.r_w) == 0 &&
           std::memcmp(b0.r_tz, b1.r_tz, sizeof b0.r_tz) == 0 &&
           std::memcmp(b0.r_first, b1.r_first, sizeof b0.r_first) == 0;
}

// One cooperative launch for the whole pass.  Returns PSDM_OK when launched,
// 1 when the pass does not have the form (the caller launches per step), or
// an error code.
int launch_pass_form(psdm_engine* e, int mode, const std::vector<StepArgs>& args, int nrec, const int* h_rec_cell) {
    StepArgs base[2];
    std::vector<PassVar> var;
    if (!pass_form(args, base, &var)) return 1;
    const StepArgs& a = base[0];
    if (mode == 0 && a.nrec > 0 && (h_rec_cell == nullptr || nrec != a.nrec)) return 1;
    const int ntiles = a.r_first[a.nrect];
    const int nb = pass_blocks_per_sm(mode);
    if (nb <= 0 || ntiles <= 0) return 1;
    const int grid = std::min(ntiles, nb * e->num_sms);
    std::vector<int> key = {mode == 0 ? a.nrec : 0, a.nrect, a.itx, a.ixb, a.ldz, a.nxt};
    key.insert(key.end(), a.r_type, a.r_type + a.nrect);
    key.insert(key.end(), a.r_zd0, a.r_zd0 + a.nrect);
    key.insert(key.end(), a.r_x0, a.r_x0 + a.nrect);
    key.insert(key.end(), a.r_h, a.r_h + a.nrect);
    key.insert(key.end(), a.r_w, a.r_w + a.nrect);
    if (mode == 0 && a.nrec > 0) key.insert(key.end(), h_rec_cell, h_rec_cell + nrec);
    int *d_nf = nullptr, *d_nb = nullptr, *d_rf = nullptr, *d_ri = nullptr;
    const std::string m = std::to_string(mode);
    const bool fresh = key != e->pass_key[mode];
    std::vector<int> nf, nbv, rf, ri;
    if (fresh) {
        pass_lists(a, mode == 0 ? a.nrec : 0, h_rec_cell, &nf, &nbv, &rf, &ri);
        e->pass_key[mode].clear();
    }
    TRY(e->get(("pass_nbr_first" + m).c_str(), nf.size(), &d_nf));
    TRY(e->get(("pass_nbr" + m).c_str(), std::max<size_t>(nbv.size(), 1), &d_nb));
    TRY(e->get(("pass_rec_first" + m).c_str(), rf.size(), &d_rf));
    TRY(e->get(("pass_rec_idx" + m).c_str(), std::max<size_t>(ri.size(), 1), &d_ri));
    if (fresh) {
        CUDA_TRY(cudaMemcpyAsync(d_nf, nf.data(), nf.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
        if (!nbv.empty())
            CUDA_TRY(cudaMemcpyAsync(d_nb, nbv.data(), nbv.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaMemcpyAsync(d_rf, rf.data(), rf.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
        if (!ri.empty())
            CUDA_TRY(cudaMemcpyAsync(d_ri, ri.data(), ri.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaStreamSynchronize(e->stream));  // the host lists go out of scope
        e->pass_key[mode] = key;
    }
    StepArgs* d_base = nullptr;
    PassVar* d_var = nullptr;
    int* d_flags = nullptr;
    TRY(e->get(("pass_base" + m).c_str(), 2, &d_base));
    TRY(e->get(("pass_var" + m).c_str(), var.size(), &d_var));
    TRY(e->get("pass_flags", (size_t)ntiles + 1, &d_flags));  // + the abort word
    // Staged through page-locked buffers, one per pass kind, refilled only
    // after the previous copy out of them has completed.
    const size_t sbytes = 2 * sizeof(StepArgs) + var.size() * sizeof(PassVar);
    char* h = nullptr;
    const std::string sname = "pass_stage" + m;
    TRY(e->get_pinned(sname.c_str(), sbytes, reinterpret_cast<void**>(&h)));
    cudaEvent_t& done = e->pass_staged[mode];
    if (done == nullptr) CUDA_TRY(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    CUDA_TRY(cudaEventSynchronize(done));
    std::memcpy(h, base, 2 * sizeof(StepArgs));
    std::memcpy(h + 2 * sizeof(StepArgs), var.data(), var.size() * sizeof(PassVar));
    CUDA_TRY(cudaMemcpyAsync(d_base, h, 2 * sizeof(StepArgs), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(d_var, h + 2 * sizeof(StepArgs), var.size() * sizeof(PassVar), cudaMemcpyHostToDevice,
                             e->stream));
    CUDA_TRY(cudaEventRecord(done, e->stream));
    CUDA_TRY(cudaMemsetAsync(d_flags, 0, ((size_t)ntiles + 1) * sizeof(int), e->stream));
    PassParams pp{};
    pp.base = d_base;
    pp.var = d_var;
    pp.nsteps = (int)var.size();
    pp.ntiles = ntiles;
    pp.nbr_first = d_nf;
    pp.nbr = d_nb;
    pp.rec_first = d_rf;
    pp.rec_idx = d_ri;
    pp.flags = d_flags;
    pp.abort = d_flags + ntiles;
    pp.err = a.err;
    const int rc = launch_pass(mode, pp, grid, e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "pass launch: %s", cudaGetErrorString((cudaError_t)rc));
    return PSDM_OK;
}

// One resident launch (res_kernel) for the whole pass: forward and plain
// backward passes of one shot whose grid fits the device's regions.  Returns
// PSDM_OK when launched, 1 when the pass does not have the form, or an error.
int launch_resident_form(psdm_engine* e, int mode, const std::vector<StepArgs>& args, int nrec,
                         const int* h_rec_cell) {
    if (mode != 0 && mode != 1) return 1;
    StepArgs base[2];
    std::vector<PassVar> var;
    if (!pass_form(args, base, &var)) return 1;
    const StepArgs& a = base[0];
    if (a.field16 != nullptr) return 1;
    if (mode == 0 && a.nrec > 0 && (h_rec_cell == nullptr || nrec != a.nrec)) return 1;
    const int msw = resident_max_sw();
    if (msw < kResMinSide + 6) return 1;
    std::vector<int> key = {mode == 0 ? a.nrec : 0, a.nrect, a.ldz, a.nxt, a.nyt, a.dn, a.zoff, a.fs, a.ny, a.nx};
    key.insert(key.end(), a.r_type, a.r_type + a.nrect);
    key.insert(key.end(), a.r_zd0, a.r_zd0 + a.nrect);
    key.insert(key.end(), a.r_h, a.r_h + a.nrect);
    if (mode == 0 && a.nrec > 0) key.insert(key.end(), h_rec_cell, h_rec_cell + nrec);
    const std::string m = std::to_string(mode);
    ResRegion* d_reg = nullptr;
    int *d_nbr = nullptr, *d_rec = nullptr, *d_wf = nullptr, *d_items = nullptr;
    int& nreg = e->res_nreg[mode];
    int& sw = e->res_sw[mode];
    if (key != e->res_key[mode]) {
        e->res_key[mode].clear();
        ResPlan plan;
        int nb = resident_blocks_per_sm(mode, msw);
        if (nb <= 0) return 1;
        if (!plan_resident(a, nb * e->num_sms, msw, mode == 0 ? a.nrec : 0, h_rec_cell, &plan)) return 1;
        if (resident_blocks_per_sm(mode, plan.sw) * e->num_sms < (int)plan.reg.size()) return 1;
        TRY(e->get(("res_reg" + m).c_str(), plan.reg.size(), &d_reg));
        TRY(e->get(("res_nbr" + m).c_str(), std::max<size_t>(plan.nbr.size(), 1), &d_nbr));
        TRY(e->get(("res_rec" + m).c_str(), std::max<size_t>(plan.rec.size(), 1), &d_rec));
        TRY(e->get(("res_wf" + m).c_str(), plan.warp_first.size(), &d_wf));
        TRY(e->get(("res_items" + m).c_str(), std::max<size_t>(plan.items.size(), 2), &d_items));
        CUDA_TRY(cudaMemcpyAsync(d_reg, plan.reg.data(), plan.reg.size() * sizeof(ResRegion), cudaMemcpyHostToDevice,
                                 e->stream));
        if (!plan.nbr.empty())
            CUDA_TRY(cudaMemcpyAsync(d_nbr, plan.nbr.data(), plan.nbr.size() * sizeof(int), cudaMemcpyHostToDevice,
                                     e->stream));
        if (!plan.rec.empty())
            CUDA_TRY(cudaMemcpyAsync(d_rec, plan.rec.data(), plan.rec.size() * sizeof(int), cudaMemcpyHostToDevice,
                                     e->stream));
        CUDA_TRY(cudaMemcpyAsync(d_wf, plan.warp_first.data(), plan.warp_first.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, e->stream));
        if (!plan.items.empty())
            CUDA_TRY(cudaMemcpyAsync(d_items, plan.items.data(), plan.items.size() * sizeof(int),
                                     cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaStreamSynchronize(e->stream));  // the host lists go out of scope
        nreg = (int)plan.reg.size();
        sw = plan.sw;
        e->res_key[mode] = key;
    } else {
        TRY(e->get(("res_reg" + m).c_str(), (size_t)nreg, &d_reg));
        TRY(e->get(("res_nbr" + m).c_str(), 1, &d_nbr));
        TRY(e->get(("res_rec" + m).c_str(), 1, &d_rec));
        TRY(e->get(("res_wf" + m).c_str(), 1, &d_wf));
        TRY(e->get(("res_items" + m).c_str(), 2, &d_items));
    }
    StepArgs* d_base = nullptr;
    PassVar* d_var = nullptr;
    int* d_flags = nullptr;
    TRY(e->get(("pass_base" + m).c_str(), 2, &d_base));
    TRY(e->get(("pass_var" + m).c_str(), var.size(), &d_var));
    TRY(e->get("pass_flags", (size_t)nreg + 1, &d_flags));  // + the abort word
    const size_t sbytes = 2 * sizeof(StepArgs) + var.size() * sizeof(PassVar);
    char* h = nullptr;
    const std::string sname = "pass_stage" + m;
    TRY(e->get_pinned(sname.c_str(), sbytes, reinterpret_cast<void**>(&h)));
    cudaEvent_t& done = e->pass_staged[mode];
    if (done == nullptr) CUDA_TRY(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    CUDA_TRY(cudaEventSynchronize(done));
    std::memcpy(h, base, 2 * sizeof(StepArgs));
    std::memcpy(h + 2 * sizeof(StepArgs), var.data(), var.size() * sizeof(PassVar));
    CUDA_TRY(cudaMemcpyAsync(d_base, h, 2 * sizeof(StepArgs), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(d_var, h + 2 * sizeof(StepArgs), var.size() * sizeof(PassVar), cudaMemcpyHostToDevice,
                             e->stream));
    CUDA_TRY(cudaEventRecord(done, e->stream));
    CUDA_TRY(cudaMemsetAsync(d_flags, 0, ((size_t)nreg + 1) * sizeof(int), e->stream));
    ResParams rp{};
    rp.base = d_base;
    rp.var = d_var;
    rp.nsteps = (int)var.size();
    rp.nreg = nreg;
    rp.sw = sw;
    rp.reg = d_reg;
    rp.nbr = d_nbr;
    rp.rec = d_rec;
    rp.warp_first = d_wf;
    rp.items = d_items;
    rp.flags = d_flags;
    rp.abort = d_flags + nreg;
    rp.err = a.err;
    const int rc = launch_resident(mode, rp, e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "resident pass launch: %s", cudaGetErrorString((cudaError_t)rc));
    return PSDM_OK;
}

// Launch the step kernels of one pass.  The launches are captured once into
// a CUDA graph and the graph is replayed while the argument list is
// identical (same buffers, geometry, step count and per-step values), which
// removes the host launch cost per time step.  Falls back to direct launches
// if the capture is not possible.
int launch_steps(psdm_engine* e, int mode, const std::vector<StepArgs>& args, int nrec = 0,
                 const int* h_rec_cell = nullptr) {
    if (args.empty()) return PSDM_OK;
    if (e->use_pass) {
        const int rc = e->use_pass == 2 ? launch_resident_form(e, mode, args, nrec, h_rec_cell)
                                        : launch_pass_form(e, mode, args, nrec, h_rec_cell);
        if (rc == PSDM_OK) {
            e->launches += 1;
            return PSDM_OK;
        }
        if (rc != 1) return rc;
    }
    e->launches += (int64_t)args.size();
    auto& gc = e->graphs[mode];
    if (e->use_graphs) {
        const bool same = gc.exec && gc.args.size() == args.size() &&
                          std::memcmp(gc.args.data(), args.data(), args.size() * sizeof(StepArgs)) == 0;
        if (!same) {
            if (gc.exec) cudaGraphExecDestroy(gc.exec);
            gc.exec = nullptr;
            gc.args.clear();
            cudaStream_t cs = e->own_stream;
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                for (const StepArgs& a : args)
                    if (launch_step(mode, a, cs) != 0) { ok = false; break; }
                ok = (cudaStreamEndCapture(cs, &graph) == cudaSuccess) && ok;
            }
            if (ok) ok = cudaGraphInstantiate(&gc.exec, graph, 0) == cudaSuccess;
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();  // clear a failed capture
            if (ok) {
                gc.args = args;
            } else {
                gc.exec = nullptr;
                e->use_graphs = false;
            }
        }
        if (gc.exec) {
            CUDA_TRY(cudaGraphLaunch(gc.exec, e->stream));
            return PSDM_OK;
        }
    }
    for (const StepArgs& a : args) {
        int rc = launch_step(mode, a, e->stream);
        if (rc) return fail(PSDM_ERR_CUDA, "step launch: %s", cudaGetErrorString((cudaError_t)rc));
    }
    return PSDM_OK;
}

// Buffers of the mixed-precision form (see below): FP32 staging of the
// snapshots (slot m in stage[m % 4]; a snapshot is converted by the launch
// after the one that stages it, and a launch of two steps may stage two),
// 16-bit snapshots with their scales, and the image's Kahan compensation.
struct MixedBufs {
    int kind = 0;  // 1 binary16, 2 bfloat16
    int ks = 1;    // snapshot interval (store_snap)
    int nsnap = 0;
    size_t fstride = 0;
    float* stage[4] = {nullptr, nullptr, nullptr, nullptr};
    unsigned int* amax = nullptr;  // nsnap
    unsigned short* snap16 = nullptr;  // nsnap * fstride
    float* iscale = nullptr;       // nsnap
    float* comp = nullptr;         // fstride
};

// ---- two steps per launch -------------------------------------------------
//
// A pass of pair launches (rtm_pair.cu) is made from the pass's one-step
// arguments: the kernels need the per-step values of one or two steps, the
// shot's buffers rotated as the levels advance, and a tile plan of their own.

bool pair_on(const psdm_engine* e) { return e->steps_per_launch == 2 && !e->use_pass; }

// Rotation of a shot's buffers through a pass of pair launches.  At the
// first step of a pass the one-step launches read p = p[0] (level n), p1 =
// p[1], phi from phx[0] / phz[0], chi from chx / chz and the free-surface
// histories side[0] (level n) and side[1]; pair launches start from the
// same state and write to the other buffers.
struct PairRot {
    float* prev;   // level n-1
    float* cur;    // level n
    float* fr[2];  // free: levels n+1, n+2
    float *phx_in, *phx_out, *phz_in, *phz_out;
    float *chx_in, *chx_out, *chz_in, *chz_out;
    float* sprev;
    float* scur;
    float* sfr[2];
};

PairRot pair_rot_start(const Shot& s) {
    return PairRot{s.p[1],   s.p[0], {s.p[2], s.p[3]}, s.phx[0],  s.phx[1],  s.phz[0], s.phz[1],
                   s.chx,    s.chx2, s.chz,            s.chz2,    s.side[1], s.side[0], {s.side[2], s.side[3]}};
}

void pair_rot_advance(PairRot& r, int nsub) {
    if (nsub == 2) {
        std::swap(r.prev, r.fr[0]);
        std::swap(r.cur, r.fr[1]);
        std::swap(r.sprev, r.sfr[0]);
        std::swap(r.scur, r.sfr[1]);
    } else {
        float* t = r.prev;
        r.prev = r.cur;
        r.cur = r.fr[0];
        r.fr[0] = t;
        t = r.sprev;
        r.sprev = r.scur;
        r.scur = r.sfr[0];
        r.sfr[0] = t;
    }
    std::swap(r.phx_in, r.phx_out);
    std::swap(r.phz_in, r.phz_out);
    std::swap(r.chx_in, r.chx_out);
    std::swap(r.chz_in, r.chz_out);
}

// Pair launches for the one-step arguments steps[first, first + count) of a
// pass of mode `mode` (step k = i - first + 2).  row_slot: the host copy of
// the pass's injection row map.  Forward passes with receivers gather them
// inside the tiles (h_rec_cell: the receivers' cells, nrec of them).  mb:
// the mixed form's buffers for a forward pass, whose snapshot conversions
// move to the launch after the one that stages the snapshot, or null.
// Out: the launches, the buffer holding the pass's last level, and the
// snapshot slots staged by the last launch (to be converted after the pass).
int make_pairs(psdm_engine* e, const Shot& s, int mode, const std::vector<StepArgs>& steps, size_t first,
               size_t count, const std::vector<int>& row_slot, int nrec, const int* h_rec_cell, const MixedBufs* mb,
               const std::string& tag, std::vector<PairArgs>* out, float** last, std::vector<int>* pending,
               float** prev_last = nullptr) {
    PairRot r = pair_rot_start(s);
    *last = r.cur;
    if (prev_last) *prev_last = r.prev;
    if (pending) pending->clear();
    if (count == 0) return PSDM_OK;
    PairArgs base;
    std::memset(&base, 0, sizeof(base));
    base.a = steps[first];
    if (!plan_pair(&base, row_slot.empty() ? nullptr : row_slot.data()))
        return fail(PSDM_ERR_ARG, "the tile plan of the two-step launches needs more than %d rectangles", kPairRects);
    const bool recs = mode == 0 && base.a.rec_out != nullptr && base.a.nrec > 0;
    if (recs) {
        std::vector<int> f, ix;
        pair_rec_lists(base, nrec, h_rec_cell, &f, &ix);
        int *d_f = nullptr, *d_i = nullptr;
        TRY(e->get(("pair_recf" + tag).c_str(), f.size(), &d_f));
        TRY(e->get(("pair_reci" + tag).c_str(), std::max<size_t>(ix.size(), 1), &d_i));
        CUDA_TRY(cudaMemcpyAsync(d_f, f.data(), f.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
        if (!ix.empty())
            CUDA_TRY(cudaMemcpyAsync(d_i, ix.data(), ix.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaStreamSynchronize(e->stream));  // the host lists go out of scope
        base.rec_first = d_f;
        base.rec_idx = d_i;
    }
    std::vector<int> pend;  // slots staged by the previous launch
    const size_t end = first + count;
    int sel = 0;
    out->reserve(out->size() + (count + 1) / 2);
    for (size_t i = first; i < end;) {
        const int ns = end - i >= 2 ? 2 : 1;
        PairArgs q = base;
        q.a = steps[i];
        q.a.counter_sel = sel;
        sel ^= 1;
        q.a.pm = r.prev;
        q.a.p = r.cur;
        q.p_out[0] = r.fr[0];
        q.p_out[1] = r.fr[1];
        q.a.phix_in = r.phx_in;
        q.a.phix_out = r.phx_out;
        q.a.phiz_in = r.phz_in;
        q.a.phiz_out = r.phz_out;
        q.chix_in = r.chx_in;
        q.a.chix = r.chx_out;
        q.chiz_in = r.chz_in;
        q.a.chiz = r.chz_out;
        q.a.side_pm = r.sprev;
        q.a.side_p = r.scur;
        q.side_out[0] = r.sfr[0];
        q.side_out[1] = r.sfr[1];
        q.nsub = ns;
        for (int j = 0; j < ns; ++j) {
            const StepArgs& t = steps[i + j];
            SubStep& u = q.sub[j];
            u.field = t.field;
            u.field16 = t.field16;
            u.field_iscale = t.field_iscale;
            u.field_amax = t.field_amax;
            u.field_w = t.field_w;
            u.inj_t = t.inj_t;
            u.rec_t = recs ? (int)(i + j - first) : -1;  // step k gives Rec(k-1)
        }
        q.a.q_src = nullptr;
        q.q_src2 = nullptr;
        if (mb) {
            for (size_t k = 0; k < pend.size() && k < 2; ++k) {
                const int m = pend[k];
                const float* src = mb->stage[m & 3];
                const unsigned int* am = mb->amax + (m - 1);
                void* dst = mb->snap16 + (size_t)(m - 1) * mb->fstride;
                float* isc = mb->iscale + (m - 1);
                if (k == 0) {
                    q.a.q_n = (int)mb->fstride;
                    q.a.q_src = src;
                    q.a.q_amax = am;
                    q.a.q_dst = dst;
                    q.a.q_iscale = isc;
                } else {
                    q.q_n2 = (int)mb->fstride;
                    q.q_src2 = src;
                    q.q_amax2 = am;
                    q.q_dst2 = dst;
                    q.q_iscale2 = isc;
                }
            }
            pend.clear();
            for (int j = 0; j < ns; ++j)
                if (steps[i + j].field_amax != nullptr) pend.push_back((int)(steps[i + j].field_amax - mb->amax) + 1);
        }
        out->push_back(q);
        pair_rot_advance(r, ns);
        i += ns;
    }
    *last = r.cur;
    if (prev_last) *prev_last = r.prev;
    if (pending) *pending = pend;
    return PSDM_OK;
}

// Launch a pass of pair launches, captured once into a CUDA graph and
// replayed while the argument list is unchanged (as launch_steps does).
int launch_pairs(psdm_engine* e, int mode, const std::vector<PairArgs>& L) {
    if (L.empty()) return PSDM_OK;
    e->launches += (int64_t)L.size();
    auto& gc = e->pgraphs[mode];
    if (e->use_graphs) {
        const bool same = gc.exec && gc.args.size() == L.size() &&
                          std::memcmp(gc.args.data(), L.data(), L.size() * sizeof(PairArgs)) == 0;
        if (!same) {
            if (gc.exec) cudaGraphExecDestroy(gc.exec);
            gc.exec = nullptr;
            gc.args.clear();
            cudaStream_t cs = e->own_stream;
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                for (const PairArgs& q : L)
                    if (launch_pair(mode, q, cs) != 0) {
                        ok = false;
                        break;
                    }
                ok = (cudaStreamEndCapture(cs, &graph) == cudaSuccess) && ok;
            }
            if (ok) ok = cudaGraphInstantiate(&gc.exec, graph, 0) == cudaSuccess;
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();  // clear a failed capture
            if (ok) {
                gc.args = L;
            } else {
                gc.exec = nullptr;
                e->use_graphs = false;
            }
        }
        if (gc.exec) {
            CUDA_TRY(cudaGraphLaunch(gc.exec, e->stream));
            return PSDM_OK;
        }
    }
    for (const PairArgs& q : L) {
        const int rc = launch_pair(mode, q, e->stream);
        if (rc) return fail(PSDM_ERR_CUDA, "pair launch: %s", cudaGetErrorString((cudaError_t)rc));
    }
    return PSDM_OK;
}

// Step arguments of a forward pass over k = 2..nt
// (solver_ac_forward_ram.f90:344-577).
//   d_S: source trace (nt); d_fields: snapshot slots (nslots of ny*nx) or null;
//   d_rec: receiver traces (NumRec, nt) or null.
//   tag: suffix of the engine buffers holding the injection map and the
//   receiver cells; the per-step arguments are appended to *steps_out.
int build_forward(psdm_engine* e, Shot& s, int nt, int store_snap, const float* d_S, int zs, int xs,
                  float* d_fields, int nslots, int nrec, const int* h_rec_cell, float* d_rec, const std::string& tag,
                  std::vector<StepArgs>* steps_out, bool batched = false, std::vector<int>* row_slot_out = nullptr) {
    const Grid& g = s.g;
    InjMap inj;
    TRY(build_inj(g, 1, &zs, &xs, &inj));
    if (row_slot_out) *row_slot_out = inj.row_slot;
    int *d_row = nullptr, *d_cols = nullptr;
    TRY(upload_inj(e, g, inj, ("src" + tag).c_str(), &d_row, &d_cols));
    int* d_rec_cell = nullptr;
    if (d_rec && nrec > 0) {
        TRY(e->get(("rec_cell" + tag).c_str(), (size_t)nrec, &d_rec_cell));
        CUDA_TRY(cudaMemcpyAsync(d_rec_cell, h_rec_cell, nrec * sizeof(int), cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaMemsetAsync(d_rec, 0, (size_t)nrec * nt * sizeof(float), e->stream));
    }
    StepArgs a = base_args(s);
    plan_tiles(&a, inj.row_slot.data(), batched, true);
    a.row_slot = d_row;
    a.inj_cols = d_cols;
    a.inj_trace = d_S;
    a.inj_ld = 0;
    a.rec_cell = d_rec_cell;
    a.rec_out = d_rec;
    a.nrec = d_rec ? nrec : 0;
    a.rec_ld = nt;
    const size_t fstride = g.field_cells();
    std::vector<StepArgs>& steps = *steps_out;
    steps.reserve(steps.size() + (nt > 1 ? nt - 1 : 0));
    for (int k = 2; k <= nt; ++k) {
        const int it = k - 2;
        set_buffers(s, it, &a);
        a.inj_t = k - 2;                           // S(k-1)
        a.rec_t = (d_rec && k >= 3) ? k - 3 : -1;  // Rec(k-2) from p = level k-1
        a.field = nullptr;
        if (d_fields && (k - 1) % store_snap == 0) {
            const int snap = (k - 1) / store_snap;  // 1-based slot
            if (snap > nslots) return fail(PSDM_ERR_ARG, "snapshot slot %d exceeds nt_snap=%d", snap, nslots);
            a.field = d_fields + (size_t)(snap - 1) * fstride;
        }
        steps.push_back(a);
    }
    return PSDM_OK;
}

// Forward pass over k = 2..nt (solver_ac_forward_ram.f90:344-577).
//   d_S: source trace (nt); d_fields: snapshot slots (nslots of ny*nx) or null;
//   d_rec: receiver traces (NumRec, nt) or null.
int run_forward(psdm_engine* e, Shot& s, int nt, int store_snap, const float* d_S, int zs, int xs,
                float* d_fields, int nslots, int nrec, const int* h_rec_cell, float* d_rec) {
    std::vector<StepArgs> steps;
    std::vector<int> row_slot;
    TRY(build_forward(e, s, nt, store_snap, d_S, zs, xs, d_fields, nslots, nrec, h_rec_cell, d_rec, "", &steps, false,
                      &row_slot));
    const int* d_rec_cell = steps.empty() ? nullptr : steps[0].rec_cell;
    const float* pfin = s.p[(nt - 1) & 1];  // p3 of the last step
    if (pair_on(e)) {
        std::vector<PairArgs> pairs;
        float* last = nullptr;
        TRY(make_pairs(e, s, 0, steps, 0, steps.size(), row_slot, nrec, h_rec_cell, nullptr, "", &pairs, &last,
                       nullptr));
        TRY(launch_pairs(e, 0, pairs));
        pfin = last;
    } else {
        TRY(launch_steps(e, 0, steps, nrec, h_rec_cell));
    }
    e->fwd_steps += nt - 1;
    if (d_rec && nrec > 0 && nt >= 2) {
        int rc = launch_rec_final(d_rec_cell, pfin, d_rec, nrec, nt, nt, e->stream);
        if (rc) return fail(PSDM_ERR_CUDA, "receiver gather: %s", cudaGetErrorString((cudaError_t)rc));
        e->launches += 1;
    }
    return PSDM_OK;
}

// Step arguments of a backward pass over k = 2..nt
// (solver_ac_backward_ram.f90:329-545); run_backward launches them.
//   d_back: adjoint traces (nt, NumRec); with reverse = 1 they are read in
//   reverse time order, which is BackSource(:,j) = Data_target(nt:1:-1, j)
//   (calculate_PSDM_RTM.f90:448-450) without materialising it.
//   Snapshots: slot `snap` (1-based) is d_fields + (snap - slot_lo) * ny*nx
//   when slot_lo <= snap <= slot_hi, and zero otherwise; h_w[snap - 1] is the
//   taper weight of slot `snap` (size >= nt_snap; null for all ones).
int build_backward(psdm_engine* e, Shot& s, int nt, int store_snap, int nt_snap, const float* d_back, int reverse,
                   int nrec, const int* zr, const int* xr, const float* d_fields, int slot_lo, int slot_hi,
                   const float* h_w, float* d_image, const std::string& tag, std::vector<StepArgs>* steps_out,
                   std::vector<int>* slot_of_step = nullptr, bool batched = false,
                   std::vector<int>* row_slot_out = nullptr) {
    const Grid& g = s.g;
    InjMap inj;
    TRY(build_inj(g, nrec, zr, xr, &inj));
    if (row_slot_out) *row_slot_out = inj.row_slot;
    int *d_row = nullptr, *d_cols = nullptr;
    TRY(upload_inj(e, g, inj, ("rec" + tag).c_str(), &d_row, &d_cols));
    StepArgs a = base_args(s);
    plan_tiles(&a, inj.row_slot.data(), batched);
    a.row_slot = d_row;
    a.inj_cols = d_cols;
    a.inj_trace = d_back;
    a.inj_ld = nt;
    a.image = d_image;
    a.ss = float(store_snap);
    const size_t fstride = g.field_cells();
    int snap = nt_snap;
    std::vector<StepArgs>& steps = *steps_out;
    steps.reserve(steps.size() + (nt > 1 ? nt - 1 : 0));
    for (int k = 2; k <= nt; ++k) {
        const int it = k - 2;
        set_buffers(s, it, &a);
        a.inj_t = reverse ? nt - k + 1 : k - 2;  // Sadj(k-1)
        a.field = nullptr;
        a.field_w = 1.f;
        int used = 0;
        if ((k - 1) % store_snap == 0) {
            snap = snap - 1;
            if (d_fields && snap >= slot_lo && snap <= slot_hi && snap >= 1) {
                a.field = const_cast<float*>(d_fields) + (size_t)(snap - slot_lo) * fstride;
                a.field_w = h_w ? h_w[snap - 1] : 1.f;
                if (a.field_w == 0.f) a.field = nullptr;  // zero-padded slot: no contribution
                if (a.field) used = snap;
            }
        }
        if (slot_of_step) slot_of_step->push_back(used);
        steps.push_back(a);
    }
    return PSDM_OK;
}

int run_backward(psdm_engine* e, Shot& s, int nt, int store_snap, int nt_snap, const float* d_back, int reverse,
                 int nrec, const int* zr, const int* xr, const float* d_fields, int slot_lo, int slot_hi,
                 const float* h_w, float* d_image) {
    std::vector<StepArgs> steps;
    std::vector<int> row_slot;
    TRY(build_backward(e, s, nt, store_snap, nt_snap, d_back, reverse, nrec, zr, xr, d_fields, slot_lo, slot_hi, h_w,
                       d_image, "", &steps, nullptr, false, &row_slot));
    if (pair_on(e)) {
        std::vector<PairArgs> pairs;
        float* last = nullptr;
        TRY(make_pairs(e, s, 1, steps, 0, steps.size(), row_slot, 0, nullptr, nullptr, "", &pairs, &last, nullptr));
        TRY(launch_pairs(e, 1, pairs));
    } else {
        TRY(launch_steps(e, 1, steps));
    }
    e->bwd_steps += nt - 1;
    return PSDM_OK;
}

int check_engine(psdm_engine* e) {
    if (!e) return fail(PSDM_ERR_STATE, "engine is NULL");
    CUDA_TRY(cudaSetDevice(e->device));
    return PSDM_OK;
}

int sync(psdm_engine* e) {
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (e->h_err && *e->h_err) {
        const int code = *e->h_err;
        *e->h_err = 0;
        return fail(PSDM_ERR_CUDA, "%s", step_error_message(code));
    }
    return PSDM_OK;
}

// Window coordinates of a shot (dynamic_window wrappers,
// src/dynamic_window.f90:80-86): x_i from the model-coordinate geometry.
struct WinGeom {
    int x_i = 1, nx_w_calc = 0;
    int zs = 0, xs = 0;         // padded 0-based source (logical rows)
    std::vector<int> zr, xr;    // padded 0-based receivers (logical rows)
    std::vector<int> rec_cell;  // xr*ldz + zr + zoff
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
        w->rec_cell[r] = w->xr[r] * g.ldz + w->zr[r] + g.zoff;
    }
    return PSDM_OK;
}

// ---- mixed-precision form ----------------------------------------------------
//
// prm->precision = PSDM_PREC_FP16 / _BF16.  Propagation is the same FP32
// step; the forward pass keeps a snapshot every store_snap steps as 16-bit
// values scaled by a power of two chosen from that snapshot's largest
// magnitude (the snapshot is written in FP32 to a staging buffer with its
// maximum, and converted by the next step's launch), and the backward pass
// images at the steps paired in time with the stored snapshots,
// k_b = nt_taper + 1 - store_snap*m for slot m, summing the image with Kahan
// compensation.  The taper weight of slot m is the weight of its time
// sample store_snap*m.  This form has no reference counterpart; for
// store_snap = 1 its pairing is the reference's.

// nslots16: 16-bit snapshot slots to allocate (all nsnap of the pass when
// negative; fewer when the slots are reused, as by checkpointed shots).
int mixed_bufs(psdm_engine* e, const Shot& s, int kind, int ks, int nt_prop2, const std::string& tag, MixedBufs* mb,
               int nslots16 = -1) {
    mb->kind = kind;
    mb->ks = ks;
    mb->nsnap = (nt_prop2 - 1) / ks;
    mb->fstride = s.g.field_cells();
    const size_t fs = mb->fstride, ns = (size_t)std::max(mb->nsnap, 1);
    const size_t n16 = nslots16 < 0 ? ns : (size_t)std::max(nslots16, 1);
    for (int i = 0; i < 4; ++i) TRY(e->get(("stage" + std::to_string(i) + tag).c_str(), fs, &mb->stage[i]));
    TRY(e->get(("amax" + tag).c_str(), ns, &mb->amax));
    TRY(e->get(("snap16" + tag).c_str(), n16 * fs, &mb->snap16));
    TRY(e->get(("iscale" + tag).c_str(), ns, &mb->iscale));
    TRY(e->get(("comp" + tag).c_str(), fs, &mb->comp));
    // The staging buffers' pad rows are converted too: keep them zero.
    for (float* b : mb->stage) CUDA_TRY(cudaMemsetAsync(b, 0, fs * sizeof(float), e->stream));
    CUDA_TRY(cudaMemsetAsync(mb->amax, 0, ns * sizeof(unsigned int), e->stream));
    CUDA_TRY(cudaMemsetAsync(mb->comp, 0, fs * sizeof(float), e->stream));
    return PSDM_OK;
}

// Forward steps (k = 2..nt) of the mixed form: snapshot slot m at the steps
// with (k-1) % ks == 0, each converted by the following step.  *pending =
// the slot taken at the last step (to be converted after the pass), or 0.
void mixed_forward_args(const MixedBufs& mb, std::vector<StepArgs>& steps, size_t first, int* pending) {
    int prev = 0;
    for (size_t i = first; i < steps.size(); ++i) {
        StepArgs& a = steps[i];
        const int k = (int)(i - first) + 2;
        a.kind16 = mb.kind;
        a.field = nullptr;
        a.field_amax = nullptr;
        a.q_src = nullptr;
        if (prev > 0) {
            a.q_src = mb.stage[prev & 3];
            a.q_amax = mb.amax + (prev - 1);
            a.q_dst = mb.snap16 + (size_t)(prev - 1) * mb.fstride;
            a.q_iscale = mb.iscale + (prev - 1);
            a.q_n = (int)mb.fstride;
            prev = 0;
        }
        if ((k - 1) % mb.ks == 0) {
            const int m = (k - 1) / mb.ks;
            if (m >= 1 && m <= mb.nsnap) {
                a.field = mb.stage[m & 3];
                a.field_amax = mb.amax + (m - 1);
                prev = m;
            }
        }
    }
    *pending = prev;
}

int mixed_quantize(psdm_engine* e, const MixedBufs& mb, int m) {
    if (m <= 0) return PSDM_OK;
    const int rc = launch_quantize(mb.stage[m & 3], mb.amax + (m - 1), mb.snap16 + (size_t)(m - 1) * mb.fstride,
                                   mb.iscale + (m - 1), (int)mb.fstride, mb.kind, e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "snapshot conversion launch: %s", cudaGetErrorString((cudaError_t)rc));
    e->launches += 1;
    return PSDM_OK;
}

// Backward steps (k = 2..nt) of the mixed form: slot m pairs with
// k = nt + 1 - ks*m; h_w = per-sample taper weights (nt entries) or null.
void mixed_backward_args(const MixedBufs& mb, int nt, const float* h_w, std::vector<StepArgs>& steps,
                         size_t first) {
    for (size_t i = first; i < steps.size(); ++i) {
        StepArgs& a = steps[i];
        const int k = (int)(i - first) + 2;
        a.kind16 = mb.kind;
        a.field = nullptr;
        a.field16 = nullptr;
        a.comp = mb.comp;
        a.ss = float(mb.ks);
        a.field_w = 1.f;
        const int r = nt + 1 - k;
        if (r % mb.ks != 0) continue;
        const int m = r / mb.ks;
        if (m < 1 || m > mb.nsnap) continue;
        const float w = h_w ? h_w[(size_t)mb.ks * m - 1] : 1.f;
        if (w == 0.f) continue;  // zero weight: no contribution
        a.field16 = mb.snap16 + (size_t)(m - 1) * mb.fstride;
        a.field_iscale = mb.iscale + (m - 1);
        a.field_w = w;
    }
}

// Per-sample taper weights of the snapshot series (calculate_PSDM_RTM.f90:421-427).
std::vector<float> taper_weights(int nt_prop2, int nt_taper, int taper_option, int N_taper, int N_zeros) {
    std::vector<float> wts(std::max(nt_taper, 1), 1.f);
    if (taper_option != 0) {
        const int i0 = std::max(1, nt_prop2 - N_taper + 1);
        for (int n = 0; n < N_taper; ++n)
            if (i0 + n <= nt_prop2) wts[i0 + n - 1] = taper_weight(n, N_taper);
        if (N_zeros > 0)
            for (int i = nt_prop2; i < nt_taper; ++i) wts[i] = 0.f;
    }
    return wts;
}

// ---- checkpointed FP32 shot ------------------------------------------------------
//
// In place of keeping every snapshot of the forward pass (the RAM strategy)
// or writing them to files (the disk strategy, solver_ac_forward_disk.f90:
// 469-517), the forward pass keeps the whole propagation state every K steps
// (p at both levels, the C-PML variables, the free-surface histories), and
// the backward pass recomputes each K-step segment of the forward pass from
// its checkpoint into a K-slot buffer just before it needs the segment's
// snapshots, visiting the segments from last to first.  The kernels and
// their arguments are those of the plain shot, so the image is the same bit
// for bit; the forward pass runs twice.  Memory: (segments - 1) states plus
// K snapshots instead of nt_prop2 snapshots.

struct StateView {
    float* a[10];
    size_t n[10];
};

StateView state_of(Shot& s) {
    const size_t n = s.g.cells(), m = (size_t)s.g.nxt;
    return StateView{{s.p[0], s.p[1], s.phx[0], s.phx[1], s.chx, s.phz[0], s.phz[1], s.chz, s.side[0], s.side[1]},
                     {n, n, n, n, n, n, n, n, m, m}};
}

size_t state_floats(const Shot& s) { return 8 * s.g.cells() + 2 * (size_t)s.g.nxt; }

int copy_state(psdm_engine* e, Shot& s, float* ck, bool save) {
    const StateView v = state_of(s);
    size_t off = 0;
    for (int i = 0; i < 10; ++i) {
        float* dst = save ? ck + off : v.a[i];
        const float* src = save ? v.a[i] : ck + off;
        CUDA_TRY(cudaMemcpyAsync(dst, src, v.n[i] * sizeof(float), cudaMemcpyDeviceToDevice, e->stream));
        off += v.n[i];
    }
    if (!save) CUDA_TRY(cudaMemsetAsync(s.counters, 0, 2 * sizeof(int), e->stream));
    return PSDM_OK;
}

int launch_direct(psdm_engine* e, int mode, const StepArgs& a) {
    const int rc = launch_step(mode, a, e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "step launch: %s", cudaGetErrorString((cudaError_t)rc));
    e->launches += 1;
    return PSDM_OK;
}

int rtm_shot_checkpointed(psdm_engine* e, const psdm_params* prm, int NumRec, int nxSou, int nySou, const int* nxRec,
                          const int* nyRec, const float* d_S, const float* d_tgt, float dd, float dt, int ny, int nx,
                          int nx_w, const float* d_vp, float added_space, int store_snap, int nt_prop2, int nt_taper,
                          const float* wts, float* d_img, int K) {
    Shot f, b;  // forward (recomputed) and backward states
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, d_vp, &f, "_ckf"));
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, d_vp, &b));
    WinGeom w;
    TRY(window_geometry(f.g, NumRec, nxSou, nySou, nxRec, nyRec, dd, nx, added_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    const size_t fstride = f.g.field_cells();
    const int nsteps = nt_prop2 - 1, nseg = (nsteps + K - 1) / K;
    const int nsnap = (nt_prop2 - 1) / store_snap;
    float *segbuf = nullptr, *ckpts = nullptr, *d_imgp = nullptr;
    TRY(e->get("ck_segment", fstride * (size_t)K, &segbuf));
    const size_t sf = state_floats(f);
    if (nseg > 1) TRY(e->get("ck_states", sf * (size_t)(nseg - 1), &ckpts));
    TRY(e->get("image_pitched", fstride, &d_imgp));
    TRY(e->record(0));
    // Forward steps: without snapshots (first pass), and with the snapshot
    // of step k in segment slot (k-2) % K (recomputation).
    std::vector<StepArgs> fwd;
    TRY(build_forward(e, f, nt_prop2, store_snap, d_S, w.zs, w.xs, nullptr, 0, 0, nullptr, nullptr, "_ckf", &fwd));
    for (int i = 0; i < nsteps; ++i) {
        if (i > 0 && i % K == 0) TRY(copy_state(e, f, ckpts + sf * (size_t)(i / K - 1), true));
        TRY(launch_direct(e, 0, fwd[i]));
    }
    e->fwd_steps += nsteps;
    TRY(e->record(1));
    // Backward steps, with each imaging step's slot remapped into the segment buffer.
    std::vector<StepArgs> bwd;
    std::vector<int> slot;
    CUDA_TRY(cudaMemsetAsync(d_imgp, 0, fstride * sizeof(float), e->stream));
    TRY(build_backward(e, b, nt_taper, store_snap, nt_taper, d_tgt, 1, NumRec, w.zr.data(), w.xr.data(), segbuf, 1,
                       nsnap, wts, d_imgp, "", &bwd, &slot));
    int cur = -1;
    for (size_t i = 0; i < bwd.size(); ++i) {
        const int m = slot[i];
        if (m > 0) {
            const int kf = store_snap * m + 1;  // forward step that took slot m
            const int j = (kf - 2) / K;
            if (j != cur) {  // recompute segment j from its checkpoint
                if (j == 0)
                    TRY(reset_state(e, &f));
                else
                    TRY(copy_state(e, f, ckpts + sf * (size_t)(j - 1), false));
                const int i1 = std::min((j + 1) * K, nsteps);
                for (int t = j * K; t < i1; ++t) {
                    StepArgs a = fwd[t];
                    const int k = t + 2;
                    if ((k - 1) % store_snap == 0 && (k - 1) / store_snap <= nsnap)
                        a.field = segbuf + (size_t)(t - j * K) * fstride;
                    TRY(launch_direct(e, 0, a));
                }
                e->fwd_steps += i1 - j * K;
                cur = j;
            }
            bwd[i].field = segbuf + (size_t)(kf - 2 - j * K) * fstride;
        }
        TRY(launch_direct(e, 1, bwd[i]));
    }
    e->bwd_steps += (int64_t)bwd.size();
    TRY(e->record(2));
    CUDA_TRY(cudaMemcpy2DAsync(d_img, (size_t)ny * sizeof(float), d_imgp, (size_t)b.g.ldf * sizeof(float),
                               (size_t)ny * sizeof(float), nx_w, cudaMemcpyDeviceToDevice, e->stream));
    return PSDM_OK;
}

// ---- boundary-saved reconstruction of the source wavefield -----------------
//
// In place of keeping the forward pass's snapshots (the RAM strategy) or
// writing them to files (the disk strategy, solver_ac_forward_disk.f90:
// 469-517), the forward pass (two steps per launch) saves every level's band
// -- the 3 C-PML cells next to the interior on each side -- and keeps its
// last two levels; the backward pass runs the source wavefield backwards in
// time on the interior, P(L) = (2 P(L+1) + c2 (...)) - P(L+2) with the band
// of level L put back, which yields each imaging step's snapshot just before
// the step needs it.  The reverse recursion repeats the forward step's
// rounding in the opposite direction, so the image equals the plain shot's
// to rounding level, not bit for bit.  Memory: the band, 4 B x (6 ny + 6 nx)
// per step, in place of ny x nx_w per step.  FP32 with store_snap 1; the
// passes use pair launches (the band is written by the pair kernels' tiles)
// whatever the engine's launch form.
int rtm_shot_reconstructed(psdm_engine* e, const psdm_params* prm, int NumRec, int nxSou, int nySou,
                           const int* nxRec, const int* nyRec, const float* d_S, const float* d_tgt, float dd,
                           float dt, int ny, int nx, int nx_w, const float* d_vp, float added_space, int nt_prop2,
                           int nt_taper, const float* wts, float* d_img) {
    Shot f, b;  // forward (its last two levels feed the reconstruction) and backward states
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, d_vp, &f, "_rcf"));
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, d_vp, &b));
    WinGeom w;
    TRY(window_geometry(f.g, NumRec, nxSou, nySou, nxRec, nyRec, dd, nx, added_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    const size_t fstride = f.g.field_cells();
    const int nsnap = nt_prop2 - 1;
    const size_t nband = (size_t)band_count(ny, nx_w);
    float *band = nullptr, *snap = nullptr, *d_imgp = nullptr;
    TRY(e->get("rc_band", nband * (size_t)(nt_prop2 + 1), &band));
    TRY(e->get("rc_snap", 2 * fstride, &snap));
    TRY(e->get("image_pitched", fstride, &d_imgp));
    CUDA_TRY(cudaMemsetAsync(band, 0, nband * (nt_prop2 + 1) * sizeof(float), e->stream));
    TRY(e->record(0));
    // forward: no snapshots, the band of every level k (written by step k)
    std::vector<StepArgs> fwd;
    std::vector<int> frow;
    TRY(build_forward(e, f, nt_prop2, 1, d_S, w.zs, w.xs, nullptr, 0, 0, nullptr, nullptr, "_rcf", &fwd, false,
                      &frow));
    std::vector<PairArgs> fp;
    float *last = nullptr, *prev = nullptr;
    TRY(make_pairs(e, f, 0, fwd, 0, fwd.size(), frow, 0, nullptr, nullptr, "_rcf", &fp, &last, nullptr, &prev));
    for (size_t q = 0, i = 0; q < fp.size(); i += fp[q].nsub, ++q)
        for (int j = 0; j < fp[q].nsub; ++j) fp[q].sub[j].band = band + nband * (size_t)(i + j + 2);
    TRY(launch_pairs(e, 0, fp));
    e->fwd_steps += nt_prop2 - 1;
    TRY(e->record(1));
    // backward: slot m is imaged at step k = nt_taper + 1 - m from a
    // snapshot the reverse step writes just before the launch
    CUDA_TRY(cudaMemsetAsync(d_imgp, 0, fstride * sizeof(float), e->stream));
    std::vector<StepArgs> bwd;
    std::vector<int> brow, slot;
    TRY(build_backward(e, b, nt_taper, 1, nt_taper, d_tgt, 1, NumRec, w.zr.data(), w.xr.data(), snap, 1, nsnap, wts,
                       d_imgp, "", &bwd, &slot, false, &brow));
    std::vector<PairArgs> bp;
    float* blast = nullptr;
    TRY(make_pairs(e, b, 1, bwd, 0, bwd.size(), brow, 0, nullptr, nullptr, "", &bp, &blast, nullptr));
    const StepArgs& fa = fwd[0];
    ReconArgs r;
    std::memset(&r, 0, sizeof(r));
    r.c2 = f.c2;
    for (int k = 0; k < 4; ++k) r.cf2[k] = f.cf2[k];
    r.nyt = f.g.nyt; r.nxt = f.g.nxt; r.ldz = f.g.ldz; r.ny = ny; r.nx = nx_w; r.dn = f.g.dn; r.zoff = f.g.zoff;
    r.ldf = f.g.ldf;
    r.fs = f.fs;
    r.row_slot = fa.row_slot;
    r.inj_cols = fa.inj_cols;
    r.inj_trace = d_S;
    r.dt = f.dt; r.inv_dt = f.inv_dt; r.div_lo = f.div_lo; r.div_hi = f.div_hi; r.div_tiny = f.div_tiny;
    r.fast_div = f.fast_div;
    float* cur = prev;  // level m = nsnap
    float* nxt = last;  // level m + 1
    int m_next = nsnap;  // the next slot the recursion produces
    for (size_t q = 0, i = 0; q < bp.size(); i += bp[q].nsub, ++q) {
        for (int j = 0; j < bp[q].nsub; ++j) {
            const int m = slot[i + j] > 0 ? slot[i + j] : 0;
            bp[q].sub[j].field = nullptr;
            if (m <= 0) continue;
            while (m_next >= m) {  // P(m_next - 1) from P(m_next), P(m_next + 1); its snapshot is slot m_next
                r.pc = cur;
                r.pn = nxt;
                r.band_L = band + nband * (size_t)(m_next - 1);
                r.snap = snap + (size_t)j * fstride;
                r.inj_t = m_next - 1;  // the source sample of forward step m_next + 1
                const int rc = launch_reconstruct(r, e->stream);
                if (rc) return fail(PSDM_ERR_CUDA, "reconstruction launch: %s", cudaGetErrorString((cudaError_t)rc));
                e->launches += 2;
                std::swap(cur, nxt);  // now cur = level m_next - 1, nxt = level m_next
                --m_next;
            }
            bp[q].sub[j].field = snap + (size_t)j * fstride;
        }
        const int rc = launch_pair(1, bp[q], e->stream);
        if (rc) return fail(PSDM_ERR_CUDA, "pair launch: %s", cudaGetErrorString((cudaError_t)rc));
        e->launches += 1;
    }
    e->bwd_steps += (int64_t)bwd.size();
    TRY(e->record(2));
    CUDA_TRY(cudaMemcpy2DAsync(d_img, (size_t)ny * sizeof(float), d_imgp, (size_t)b.g.ldf * sizeof(float),
                               (size_t)ny * sizeof(float), nx_w, cudaMemcpyDeviceToDevice, e->stream));
    return PSDM_OK;
}

// One shot of RTM with every array in device memory
// (calculate_PSDM_RTM.f90:395-466).  Asynchronous on e->stream.
int rtm_shot_mixed_ckpt(psdm_engine* e, const psdm_params* prm, int NumRec, int nxSou, int nySou, const int* nxRec,
                        const int* nyRec, const float* d_S, const float* d_tgt, float dd, float dt, int ny, int nx,
                        int nx_w, const float* d_vp, float added_space, int store_snap, int nt_prop2, int nt_taper,
                        int taper_option, int N_taper, int N_zeros, float* d_img);

int rtm_shot_core(psdm_engine* e, const psdm_params* prm, int NumRec, int nxSou, int nySou, const int* nxRec,
                  const int* nyRec, const float* d_S, const float* d_tgt, float dd, float dt, int ny, int nx,
                  int nx_w, const float* d_vp, float added_space, int store_snap, int nt_snap, int nt_prop2,
                  int nt_taper, int taper_option, int N_taper, int N_zeros, float* d_img) {
    TRY(check_params(prm));
    if (prm->precision != PSDM_PREC_FP32 && prm->precision != PSDM_PREC_FP16 && prm->precision != PSDM_PREC_BF16)
        return fail(PSDM_ERR_ARG, "unknown precision %d", prm->precision);
    if (NumRec < 1 || !nxRec || !nyRec || !d_S || !d_tgt || !d_vp || !d_img)
        return fail(PSDM_ERR_ARG, "null argument or NumRec < 1");
    if (nt_prop2 < 2 || nt_taper < 2 || store_snap < 1 || nt_taper < nt_prop2)
        return fail(PSDM_ERR_ARG, "need 2 <= nt_prop2 <= nt_taper and store_snap >= 1");
    if (taper_option != 0 && N_taper < 1) return fail(PSDM_ERR_ARG, "N_taper must be >= 1");
    const int nsnap = (nt_prop2 - 1) / store_snap;  // slots written by the forward pass
    if (nsnap > nt_snap) return fail(PSDM_ERR_ARG, "nt_snap=%d < %d snapshots", nt_snap, nsnap);
    if (prm->precision != PSDM_PREC_FP32 && e->ckpt_interval > 0)
        return rtm_shot_mixed_ckpt(e, prm, NumRec, nxSou, nySou, nxRec, nyRec, d_S, d_tgt, dd, dt, ny, nx, nx_w, d_vp,
                                   added_space, store_snap, nt_prop2, nt_taper, taper_option, N_taper, N_zeros, d_img);
    Shot s;
    TRY(setup_shot(e, prm, ny, nx_w, dd, dt, d_vp, &s));
    WinGeom w;
    TRY(window_geometry(s.g, NumRec, nxSou, nySou, nxRec, nyRec, dd, nx, added_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    const size_t fstride = s.g.field_cells();
    float *d_F = nullptr, *d_imgp = nullptr;
    TRY(e->get("image_pitched", fstride, &d_imgp));
    if (prm->precision != PSDM_PREC_FP32) {
        MixedBufs mb;
        TRY(mixed_bufs(e, s, prm->precision, store_snap, nt_prop2, "", &mb));
        TRY(e->record(0));
        std::vector<StepArgs> fw;
        std::vector<int> row_slot;
        TRY(build_forward(e, s, nt_prop2, store_snap, d_S, w.zs, w.xs, nullptr, 0, 0, nullptr, nullptr, "", &fw,
                          false, &row_slot));
        int pending = 0;
        mixed_forward_args(mb, fw, 0, &pending);
        if (pair_on(e)) {
            std::vector<PairArgs> pairs;
            std::vector<int> pend;
            float* last = nullptr;
            TRY(make_pairs(e, s, 0, fw, 0, fw.size(), row_slot, 0, nullptr, &mb, "", &pairs, &last, &pend));
            TRY(launch_pairs(e, 0, pairs));
            for (int m : pend) TRY(mixed_quantize(e, mb, m));
        } else {
            TRY(launch_steps(e, 0, fw));
            TRY(mixed_quantize(e, mb, pending));
        }
        e->fwd_steps += nt_prop2 - 1;
        TRY(e->record(1));
        const std::vector<float> wts = taper_weights(nt_prop2, nt_taper, taper_option, N_taper, N_zeros);
        CUDA_TRY(cudaMemsetAsync(d_imgp, 0, fstride * sizeof(float), e->stream));
        TRY(reset_state(e, &s));
        std::vector<StepArgs> bw;
        std::vector<int> brow;
        TRY(build_backward(e, s, nt_taper, store_snap, nt_taper, d_tgt, 1, NumRec, w.zr.data(), w.xr.data(), nullptr,
                           1, 0, nullptr, d_imgp, "", &bw, nullptr, false, &brow));
        mixed_backward_args(mb, nt_taper, wts.data(), bw, 0);
        if (pair_on(e)) {
            std::vector<PairArgs> pairs;
            float* last = nullptr;
            TRY(make_pairs(e, s, 2, bw, 0, bw.size(), brow, 0, nullptr, nullptr, "", &pairs, &last, nullptr));
            TRY(launch_pairs(e, 2, pairs));
        } else {
            TRY(launch_steps(e, 2, bw));
        }
        e->bwd_steps += nt_taper - 1;
        TRY(e->record(2));
        CUDA_TRY(cudaMemcpy2DAsync(d_img, (size_t)ny * sizeof(float), d_imgp, (size_t)s.g.ldf * sizeof(float),
                                   (size_t)ny * sizeof(float), nx_w, cudaMemcpyDeviceToDevice, e->stream));
        return PSDM_OK;
    }
    if (e->recon) {
        if (store_snap != 1) return fail(PSDM_ERR_ARG, "reconstruction of the source wavefield needs store_snap 1");
        const std::vector<float> wts = taper_weights(nt_prop2, nt_taper, taper_option, N_taper, N_zeros);
        return rtm_shot_reconstructed(e, prm, NumRec, nxSou, nySou, nxRec, nyRec, d_S, d_tgt, dd, dt, ny, nx, nx_w,
                                      d_vp, added_space, nt_prop2, nt_taper, wts.data(), d_img);
    }
    if (e->ckpt_interval > 0) {
        const std::vector<float> wts = taper_weights(nt_prop2, nt_taper, taper_option, N_taper, N_zeros);
        return rtm_shot_checkpointed(e, prm, NumRec, nxSou, nySou, nxRec, nyRec, d_S, d_tgt, dd, dt, ny, nx, nx_w,
                                     d_vp, added_space, store_snap, nt_prop2, nt_taper, wts.data(), d_img,
                                     e->ckpt_interval);
    }
    if (nsnap > 0) TRY(e->get("fields", fstride * nsnap, &d_F));
    TRY(e->record(0));
    TRY(run_forward(e, s, nt_prop2, store_snap, d_S, w.zs, w.xs, d_F, nsnap, 0, nullptr, nullptr));
    TRY(e->record(1));

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
    CUDA_TRY(cudaMemsetAsync(d_imgp, 0, fstride * sizeof(float), e->stream));
    // Second propagator call: nt_snap = nt = nt_taper (:456-458); same model.
    TRY(reset_state(e, &s));
    TRY(run_backward(e, s, nt_taper, store_snap, nt_taper, d_tgt, 1, NumRec, w.zr.data(), w.xr.data(), d_F, 1,
                     nsnap, wts.data(), d_imgp));
    TRY(e->record(2));
    // Pitched interior image -> caller's (ny, nx_w) image.
    CUDA_TRY(cudaMemcpy2DAsync(d_img, (size_t)ny * sizeof(float), d_imgp, (size_t)s.g.ldf * sizeof(float),
                               (size_t)ny * sizeof(float), nx_w, cudaMemcpyDeviceToDevice, e->stream));
    return PSDM_OK;
}

// ---- batched shots ----------------------------------------------------------
//
// Several shots ("slots") advance together, one batched launch per time step
// (batch_step_kernel): each launch takes one step of every active slot, in
// whichever pass that slot is.  A slot runs its shot's forward pass, then
// its backward pass with the imaging condition, then takes the next shot of
// the list, so shots of different window widths and record lengths mix
// freely.  Every slot owns its wavefield, C-PML state, snapshots and image;
// the per-step arguments of a shot's two passes are built on the host once,
// staged through page-locked memory and read by the kernel from HBM.

// One entry of a slot's program: a step launch (batched with the other
// slots' next launches) or a state operation between two of its launches.
enum SlotOpKind { OP_LAUNCH, OP_SAVE, OP_RESTORE, OP_RESET, OP_RESET_F, OP_QUANT };
struct SlotOp {
    int kind = OP_LAUNCH;
    int mode = 0;   // OP_LAUNCH: 0 forward, 1 backward, 2 mixed backward
    int arg = 0;    // OP_LAUNCH: index of its arguments; OP_SAVE / OP_RESTORE: checkpoint; OP_QUANT: snapshot m
    int tiles = 0;  // OP_LAUNCH: tiles of the launch
    unsigned short* dst = nullptr;  // OP_QUANT: where the 16-bit snapshot goes
};

struct BatchSlot {
    int shot = -1;       // shot index, -1 = idle
    int nfwd = 0, nbwd = 0;
    int tiles[2] = {0, 0};
    std::string tag;
    Shot s;
    StepArgs* d_args = nullptr;  // nfwd forward steps, then nbwd backward steps
    // Pair launches (two steps each): nfwd forward launches, then nbwd
    // backward launches; steps of each pass.
    bool pairs = false;
    PairArgs* d_pargs = nullptr;
    int fwd_steps = 0, bwd_steps = 0;
    std::vector<int> pend;         // mixed form, pair launches: slots staged by the last forward launch
    float* d_imgp = nullptr;     // pitched window image
    float* d_out = nullptr;      // device variant: caller's image
    float* h_out = nullptr;      // host variant: caller's image, pending copy-out
    int out_ny = 0, out_nx = 0;
    cudaEvent_t staged = nullptr;  // the slot's page-locked staging is free again
    int bwd_mode = 1;              // 1 plain backward, 2 mixed-precision backward
    MixedBufs mb;                  // mixed form: the slot's 16-bit snapshots
    int pending = 0;               // mixed form: slot taken at the last forward step
    std::vector<SlotOp> ops;       // the shot's program
    size_t pc = 0;                 // next entry of ops
    Shot f;                        // checkpointed shots: the recomputed forward state
    float* ckpts = nullptr;        // checkpointed shots: states saved every K forward steps
};

struct BatchJob {
    const psdm_params* prm;
    const psdm_shot* shots;
    int nshots;
    const float* d_S;
    float dd, dt, added_space;
    int ny, nx, store_snap, taper_option, N_taper, N_zeros;
    bool host_io;
};

int check_batch_shot(const BatchJob& j, int i) {
    const psdm_shot& sh = j.shots[i];
    if (sh.NumRec < 1 || !sh.nxRec || !sh.nyRec || !sh.Vp_w || !sh.Data_target || !sh.PSDM_w)
        return fail(PSDM_ERR_ARG, "shot %d: null argument or NumRec < 1", i);
    if (sh.nt_prop2 < 2 || sh.nt_taper < sh.nt_prop2)
        return fail(PSDM_ERR_ARG, "shot %d: need 2 <= nt_prop2 <= nt_taper", i);
    return PSDM_OK;
}

// Start shot `i` in slot `sl`: inputs, state, window, per-step arguments.
// The program of a slot's shot with every snapshot kept (FP32 slots or the
// mixed form's 16-bit slots): its forward launches, the conversion of the
// last staged snapshots, a fresh wavefield, its backward launches.
int batch_program_plain(psdm_engine* e, const BatchJob& j, BatchSlot& sl, int i, const WinGeom& w,
                        const float* d_tgt) {
    const psdm_shot& sh = j.shots[i];
    const std::string& tag = sl.tag;
    const int nt_prop2 = sh.nt_prop2, nt_taper = sh.nt_taper;
    const int nsnap = (nt_prop2 - 1) / j.store_snap;
    const size_t fstride = sl.s.g.field_cells();
    const bool mixed = j.prm->precision != PSDM_PREC_FP32;
    float* d_F = nullptr;
    if (mixed)
        TRY(mixed_bufs(e, sl.s, j.prm->precision, j.store_snap, nt_prop2, tag, &sl.mb));
    else if (nsnap > 0)
        TRY(e->get(("fields" + tag).c_str(), fstride * nsnap, &d_F));
    TRY(e->get(("imgp" + tag).c_str(), fstride, &sl.d_imgp));
    const std::vector<float> wts = taper_weights(nt_prop2, nt_taper, j.taper_option, j.N_taper, j.N_zeros);
    std::vector<StepArgs> steps;
    std::vector<int> frow, brow;
    TRY(build_forward(e, sl.s, nt_prop2, j.store_snap, j.d_S, w.zs, w.xs, d_F, nsnap, 0, nullptr, nullptr, tag,
                      &steps, true, &frow));
    sl.nfwd = (int)steps.size();
    sl.pending = 0;
    if (mixed) mixed_forward_args(sl.mb, steps, 0, &sl.pending);
    TRY(build_backward(e, sl.s, nt_taper, j.store_snap, nt_taper, d_tgt, 1, sh.NumRec, w.zr.data(), w.xr.data(),
                       d_F, 1, nsnap, wts.data(), sl.d_imgp, tag, &steps, nullptr, true, &brow));
    if (mixed) mixed_backward_args(sl.mb, nt_taper, wts.data(), steps, (size_t)sl.nfwd);
    sl.bwd_mode = mixed ? 2 : 1;
    sl.nbwd = (int)steps.size() - sl.nfwd;
    sl.fwd_steps = sl.nfwd;
    sl.bwd_steps = sl.nbwd;
    sl.pairs = pair_on(e);
    if (sl.pairs) {
        std::vector<PairArgs> pl;
        float* last = nullptr;
        TRY(make_pairs(e, sl.s, 0, steps, 0, (size_t)sl.nfwd, frow, 0, nullptr, mixed ? &sl.mb : nullptr, tag, &pl,
                       &last, &sl.pend));
        const int nf = (int)pl.size();
        TRY(make_pairs(e, sl.s, sl.bwd_mode, steps, (size_t)sl.nfwd, (size_t)sl.nbwd, brow, 0, nullptr, nullptr, tag,
                       &pl, &last, nullptr));
        sl.nfwd = nf;
        sl.nbwd = (int)pl.size() - nf;
        sl.tiles[0] = sl.nfwd > 0 ? pl[0].r_first[pl[0].nrect] : 0;
        sl.tiles[1] = sl.nbwd > 0 ? pl[nf].r_first[pl[nf].nrect] : 0;
        const size_t abytes = pl.size() * sizeof(PairArgs);
        PairArgs* h_args = nullptr;
        TRY(e->get_pinned(("hargs" + tag).c_str(), abytes, (void**)&h_args));
        std::memcpy(h_args, pl.data(), abytes);
        TRY(e->get(("pargs" + tag).c_str(), abytes, (void**)&sl.d_pargs));
        CUDA_TRY(cudaMemcpyAsync(sl.d_pargs, h_args, abytes, cudaMemcpyHostToDevice, e->stream));
    } else {
        sl.tiles[0] = sl.nfwd > 0 ? steps[0].r_first[steps[0].nrect] : 0;
        sl.tiles[1] = sl.nbwd > 0 ? steps[sl.nfwd].r_first[steps[sl.nfwd].nrect] : 0;
        const size_t abytes = steps.size() * sizeof(StepArgs);
        StepArgs* h_args = nullptr;
        TRY(e->get_pinned(("hargs" + tag).c_str(), abytes, (void**)&h_args));
        std::memcpy(h_args, steps.data(), abytes);
        TRY(e->get(("args" + tag).c_str(), abytes, (void**)&sl.d_args));
        CUDA_TRY(cudaMemcpyAsync(sl.d_args, h_args, abytes, cudaMemcpyHostToDevice, e->stream));
    }
    sl.ops.clear();
    for (int q = 0; q < sl.nfwd; ++q) sl.ops.push_back(SlotOp{OP_LAUNCH, 0, q, sl.tiles[0], nullptr});
    if (mixed) {
        std::vector<int> ms = sl.pairs ? sl.pend : std::vector<int>{sl.pending};
        for (int m : ms)
            if (m > 0) sl.ops.push_back(SlotOp{OP_QUANT, 0, m, 0, sl.mb.snap16 + (size_t)(m - 1) * fstride});
    }
    sl.ops.push_back(SlotOp{OP_RESET, 0, 0, 0, nullptr});  // second propagator call: fresh wavefield
    for (int q = 0; q < sl.nbwd; ++q)
        sl.ops.push_back(SlotOp{OP_LAUNCH, sl.bwd_mode, sl.nfwd + q, sl.tiles[1], nullptr});
    return PSDM_OK;
}

// The program of a checkpointed slot's shot (FP32 or mixed precision): a
// forward pass on the slot's second state `f` without snapshots, saving
// the state every K steps; then the backward pass, before whose first
// imaging step of each segment of K forward steps (last segment first) the
// segment is recomputed from its checkpoint with its snapshots, into K
// FP32 slots or K/ks + 2 reused 16-bit slots.  The recomputed snapshots are
// those of the uncheckpointed pass bit for bit, so is the image.
int batch_program_ckpt(psdm_engine* e, const BatchJob& j, BatchSlot& sl, int i, const WinGeom& w, const float* d_vp,
                       const float* d_tgt, int K) {
    const psdm_shot& sh = j.shots[i];
    const std::string& tag = sl.tag;
    const int nt_prop2 = sh.nt_prop2, nt_taper = sh.nt_taper, ks = j.store_snap;
    const int nsnap = (nt_prop2 - 1) / ks;
    const size_t fstride = sl.s.g.field_cells();
    const bool mixed = j.prm->precision != PSDM_PREC_FP32;
    const int nsteps = nt_prop2 - 1, nseg = (nsteps + K - 1) / K;
    TRY(setup_shot(e, j.prm, j.ny, sh.nx_w, j.dd, j.dt, d_vp, &sl.f, tag + "_ckf"));
    const size_t sf = state_floats(sl.f);
    sl.ckpts = nullptr;
    if (nseg > 1) TRY(e->get(("ck_states" + tag).c_str(), sf * (size_t)(nseg - 1), &sl.ckpts));
    TRY(e->get(("imgp" + tag).c_str(), fstride, &sl.d_imgp));
    const int S = K / ks + 2;  // 16-bit slots of one segment, reused segment after segment
    float* segbuf = nullptr;
    if (mixed)
        TRY(mixed_bufs(e, sl.s, j.prm->precision, ks, nt_prop2, tag, &sl.mb, S));
    else
        TRY(e->get(("ck_segment" + tag).c_str(), fstride * (size_t)K, &segbuf));
    const std::vector<float> wts = taper_weights(nt_prop2, nt_taper, j.taper_option, j.N_taper, j.N_zeros);
    // Arguments: [0, nsteps) the first forward pass, [nsteps, 2 nsteps) the
    // recomputation of each step, then the backward steps.
    std::vector<StepArgs> steps;
    TRY(build_forward(e, sl.f, nt_prop2, ks, j.d_S, w.zs, w.xs, nullptr, 0, 0, nullptr, nullptr, tag + "_ckf", &steps,
                      true));
    for (int t = 0; t < nsteps; ++t) steps.push_back(steps[t]);
    std::vector<int> seg_pending(nseg, 0);  // mixed: the snapshot staged by a segment's last step
    for (int jj = 0; jj < nseg; ++jj) {
        int prev = 0;
        for (int t = jj * K; t < std::min((jj + 1) * K, nsteps); ++t) {
            StepArgs& a = steps[(size_t)nsteps + t];
            const int k = t + 2;
            const bool snap = (k - 1) % ks == 0 && (k - 1) / ks >= 1 && (k - 1) / ks <= nsnap;
            if (!mixed) {
                if (snap) a.field = segbuf + (size_t)(t % K) * fstride;
                continue;
            }
            a.kind16 = sl.mb.kind;
            a.field = nullptr;
            a.field_amax = nullptr;
            a.q_src = nullptr;
            if (prev > 0) {  // convert the snapshot staged by the previous step
                a.q_src = sl.mb.stage[prev & 3];
                a.q_amax = sl.mb.amax + (prev - 1);
                a.q_dst = sl.mb.snap16 + (size_t)((prev - 1) % S) * fstride;
                a.q_iscale = sl.mb.iscale + (prev - 1);
                a.q_n = (int)fstride;
                prev = 0;
            }
            if (snap) {
                const int m = (k - 1) / ks;
                a.field = sl.mb.stage[m & 3];
                a.field_amax = sl.mb.amax + (m - 1);
                prev = m;
            }
        }
        seg_pending[jj] = prev;
    }
    const size_t b0 = steps.size();
    std::vector<int> slot;
    TRY(build_backward(e, sl.s, nt_taper, ks, nt_taper, d_tgt, 1, sh.NumRec, w.zr.data(), w.xr.data(),
                       mixed ? nullptr : segbuf, 1, nsnap, wts.data(), sl.d_imgp, tag, &steps, &slot, true));
    const int nbwd = (int)(steps.size() - b0);
    if (mixed) {
        mixed_backward_args(sl.mb, nt_taper, wts.data(), steps, b0);
        for (int q = 0; q < nbwd; ++q) {  // the slot each step images, in the segment's 16-bit slots
            StepArgs& a = steps[b0 + q];
            slot[q] = 0;
            if (a.field16 == nullptr) continue;
            const int m = (int)(a.field_iscale - sl.mb.iscale) + 1;
            slot[q] = m;
            a.field16 = sl.mb.snap16 + (size_t)((m - 1) % S) * fstride;
        }
    } else {
        for (int q = 0; q < nbwd; ++q)
            if (slot[q] > 0) steps[b0 + q].field = segbuf + (size_t)((ks * slot[q] - 1) % K) * fstride;
    }
    const int ftiles = nsteps > 0 ? steps[0].r_first[steps[0].nrect] : 0;
    const int btiles = nbwd > 0 ? steps[b0].r_first[steps[b0].nrect] : 0;
    sl.pairs = false;
    sl.bwd_mode = mixed ? 2 : 1;
    sl.ops.clear();
    for (int t = 0; t < nsteps; ++t) {
        if (t > 0 && t % K == 0) sl.ops.push_back(SlotOp{OP_SAVE, 0, t / K - 1, 0, nullptr});
        sl.ops.push_back(SlotOp{OP_LAUNCH, 0, t, ftiles, nullptr});
    }
    int cur = -1, recomputed = 0;
    for (int q = 0; q < nbwd; ++q) {
        const int m = slot[q];
        if (m > 0) {
            const int jj = (ks * m - 1) / K;  // segment of forward step t = ks*m - 1
            if (jj != cur) {
                sl.ops.push_back(jj == 0 ? SlotOp{OP_RESET_F, 0, 0, 0, nullptr}
                                         : SlotOp{OP_RESTORE, 0, jj - 1, 0, nullptr});
                const int t1 = std::min((jj + 1) * K, nsteps);
                for (int t = jj * K; t < t1; ++t) sl.ops.push_back(SlotOp{OP_LAUNCH, 0, nsteps + t, ftiles, nullptr});
                recomputed += t1 - jj * K;
                const int pm = seg_pending[jj];
                if (mixed && pm > 0)
                    sl.ops.push_back(SlotOp{OP_QUANT, 0, pm, 0, sl.mb.snap16 + (size_t)((pm - 1) % S) * fstride});
                cur = jj;
            }
        }
        sl.ops.push_back(SlotOp{OP_LAUNCH, sl.bwd_mode, (int)b0 + q, btiles, nullptr});
    }
    sl.nfwd = nsteps;
    sl.nbwd = nbwd;
    sl.fwd_steps = nsteps + recomputed;
    sl.bwd_steps = nbwd;
    const size_t abytes = steps.size() * sizeof(StepArgs);
    StepArgs* h_args = nullptr;
    TRY(e->get_pinned(("hargs" + tag).c_str(), abytes, (void**)&h_args));
    std::memcpy(h_args, steps.data(), abytes);
    TRY(e->get(("args" + tag).c_str(), abytes, (void**)&sl.d_args));
    CUDA_TRY(cudaMemcpyAsync(sl.d_args, h_args, abytes, cudaMemcpyHostToDevice, e->stream));
    return PSDM_OK;
}

int batch_start(psdm_engine* e, const BatchJob& j, BatchSlot& sl, int i) {
    const psdm_shot& sh = j.shots[i];
    const int ny = j.ny, nx_w = sh.nx_w;
    const std::string& tag = sl.tag;
    const float* d_vp = sh.Vp_w;
    const float* d_tgt = sh.Data_target;
    const size_t nvp = (size_t)ny * nx_w, ntgt = (size_t)sh.NumRec * sh.nt_taper;
    // The slot's page-locked staging is reused only once its previous
    // copies have completed.
    CUDA_TRY(cudaEventSynchronize(sl.staged));
    if (j.host_io) {
        float *h_vp = nullptr, *h_tgt = nullptr, *dv = nullptr, *dtg = nullptr;
        TRY(e->get_pinned(("hvp" + tag).c_str(), nvp * sizeof(float), (void**)&h_vp));
        TRY(e->get_pinned(("htgt" + tag).c_str(), ntgt * sizeof(float), (void**)&h_tgt));
        std::memcpy(h_vp, sh.Vp_w, nvp * sizeof(float));
        std::memcpy(h_tgt, sh.Data_target, ntgt * sizeof(float));
        TRY(e->get(("vp" + tag).c_str(), nvp, &dv));
        TRY(e->get(("tgt" + tag).c_str(), ntgt, &dtg));
        CUDA_TRY(cudaMemcpyAsync(dv, h_vp, nvp * sizeof(float), cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaMemcpyAsync(dtg, h_tgt, ntgt * sizeof(float), cudaMemcpyHostToDevice, e->stream));
        d_vp = dv;
        d_tgt = dtg;
    }
    TRY(setup_shot(e, j.prm, ny, nx_w, j.dd, j.dt, d_vp, &sl.s, tag));
    WinGeom w;
    TRY(window_geometry(sl.s.g, sh.NumRec, sh.nxSou, sh.nySou, sh.nxRec, sh.nyRec, j.dd, j.nx, j.added_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "shot %d: nx_w=%d does not match the window of its geometry (%d)", i, nx_w,
                    w.nx_w_calc);
    if (e->ckpt_interval > 0)
        TRY(batch_program_ckpt(e, j, sl, i, w, d_vp, d_tgt, e->ckpt_interval));
    else
        TRY(batch_program_plain(e, j, sl, i, w, d_tgt));
    const size_t fstride = sl.s.g.field_cells();
    CUDA_TRY(cudaEventRecord(sl.staged, e->stream));
    CUDA_TRY(cudaMemsetAsync(sl.d_imgp, 0, fstride * sizeof(float), e->stream));
    sl.shot = i;
    sl.pc = 0;
    sl.out_ny = ny;
    sl.out_nx = nx_w;
    sl.d_out = j.host_io ? nullptr : sh.PSDM_w;
    sl.h_out = nullptr;
    return PSDM_OK;
}

// Host variant: copy a finished image out of the slot's page-locked buffer.
int batch_flush(psdm_engine* e, BatchSlot& sl) {
    if (!sl.h_out) return PSDM_OK;
    CUDA_TRY(cudaEventSynchronize(sl.staged));
    void* h_img = nullptr;
    const size_t bytes = (size_t)sl.out_ny * sl.out_nx * sizeof(float);
    TRY(e->get_pinned(("himg" + sl.tag).c_str(), bytes, &h_img));
    std::memcpy(sl.h_out, h_img, bytes);
    sl.h_out = nullptr;
    return PSDM_OK;
}

// The slot's shot is done: hand its image to the caller.
int batch_finish(psdm_engine* e, const BatchJob& j, BatchSlot& sl) {
    const size_t ld = (size_t)sl.s.g.ldf * sizeof(float), row = (size_t)sl.out_ny * sizeof(float);
    if (j.host_io) {
        // D2H into page-locked memory; batch_flush copies it out once done.
        float* h_img = nullptr;
        CUDA_TRY(cudaEventSynchronize(sl.staged));
        TRY(e->get_pinned(("himg" + sl.tag).c_str(), row * sl.out_nx, (void**)&h_img));
        CUDA_TRY(cudaMemcpy2DAsync(h_img, row, sl.d_imgp, ld, row, sl.out_nx, cudaMemcpyDeviceToHost, e->stream));
        CUDA_TRY(cudaEventRecord(sl.staged, e->stream));
        sl.h_out = j.shots[sl.shot].PSDM_w;
    } else {
        CUDA_TRY(cudaMemcpy2DAsync(sl.d_out, row, sl.d_imgp, ld, row, sl.out_nx, cudaMemcpyDeviceToDevice,
                                   e->stream));
    }
    return PSDM_OK;
}

int run_batch(psdm_engine* e, const BatchJob& j, int max_slots) {
    if (j.nshots <= 0) return PSDM_OK;
    for (int i = 0; i < j.nshots; ++i) TRY(check_batch_shot(j, i));
    // Slots: as many as asked for, at most kMaxSlots, and as many as fit in
    // the free device memory with every slot sized for the largest shot.
    size_t per_slot = 0;
    for (int i = 0; i < j.nshots; ++i) {
        Grid g;
        TRY(build_grid(j.prm, j.ny, j.shots[i].nx_w, &g));
        const size_t nsnap = (size_t)(j.shots[i].nt_prop2 - 1) / j.store_snap;
        const size_t steps = (size_t)j.shots[i].nt_prop2 + j.shots[i].nt_taper;
        const bool mixed = j.prm->precision != PSDM_PREC_FP32;
        const int K = e->ckpt_interval;
        size_t b;
        if (K > 0) {  // two states, the checkpoints, one segment's snapshots
            const size_t nsteps = (size_t)j.shots[i].nt_prop2 - 1, nseg = (nsteps + K - 1) / K;
            const size_t seg = mixed ? ((size_t)(K / j.store_snap + 2) * 2 + 6 * 4) * g.field_cells()
                                     : ((size_t)K + 1) * g.field_cells() * sizeof(float);
            b = 2 * 13 * g.cells() * sizeof(float) + (nseg - 1) * (8 * g.cells() + 2 * (size_t)g.nxt) * sizeof(float) +
                seg + (nsteps + steps) * sizeof(PairArgs);
        } else {
            const size_t snap_bytes = mixed ? (nsnap * 2 + 6 * 4) * g.field_cells()  // 16-bit slots, 4 stages, comp, image
                                            : (nsnap + 1) * g.field_cells() * sizeof(float);
            b = 13 * g.cells() * sizeof(float) + snap_bytes + steps * sizeof(PairArgs);
        }
        if (j.host_io) b += ((size_t)j.ny * j.shots[i].nx_w + (size_t)j.shots[i].NumRec * j.shots[i].nt_taper) *
                            sizeof(float);
        per_slot = std::max(per_slot, b);
    }
    const size_t reserve = (size_t)1 << 30;
    auto slots_that_fit = [&](int* fit, size_t* free_b) -> int {
        size_t total_b = 0;
        CUDA_TRY(cudaMemGetInfo(free_b, &total_b));
        *fit = *free_b > reserve ? (int)std::min<size_t>((*free_b - reserve) / std::max<size_t>(per_slot, 1),
                                                         (size_t)kMaxSlots)
                                 : 0;
        return PSDM_OK;
    };
    int nslots = std::min(std::min(max_slots > 0 ? max_slots : kMaxSlots, kMaxSlots), j.nshots);
    int fit = 0;
    size_t free_b = 0;
    TRY(slots_that_fit(&fit, &free_b));
    if (fit < nslots && e->total() > 0) {
        // The engine's cached buffers (earlier shots or batches) may hold the
        // memory: release them and count again.
        CUDA_TRY(cudaStreamSynchronize(e->stream));
        TRY(e->trim());
        TRY(slots_that_fit(&fit, &free_b));
    }
    nslots = std::min(nslots, fit);
    if (nslots < 1)
        return fail(PSDM_ERR_NOMEM, "one batch slot needs %.1f GB of device memory, %.1f GB are free",
                    per_slot / 1e9, free_b / 1e9);
    e->batch_slots = nslots;
    int* counters = nullptr;
    TRY(e->get("batch_counters", 2, &counters));
    CUDA_TRY(cudaMemsetAsync(counters, 0, 2 * sizeof(int), e->stream));
    std::vector<BatchSlot> slots(nslots);
    int rc = PSDM_OK;
    for (int k = 0; k < nslots; ++k) {
        slots[k].tag = "_b" + std::to_string(k);
        if (cudaEventCreateWithFlags(&slots[k].staged, cudaEventDisableTiming) != cudaSuccess) {
            rc = fail(PSDM_ERR_CUDA, "cudaEventCreate failed");
            break;
        }
    }
    int next = 0;
    for (int k = 0; rc == PSDM_OK && k < nslots && next < j.nshots; ++k) rc = batch_start(e, j, slots[k], next++);
    // Run a slot's program up to its next launch; a finished shot hands over
    // its image and the slot takes the next shot.
    auto advance = [&](BatchSlot& sl) -> int {
        for (;;) {
            if (sl.shot < 0) return PSDM_OK;
            if (sl.pc >= sl.ops.size()) {
                e->fwd_steps += sl.fwd_steps;
                e->bwd_steps += sl.bwd_steps;
                TRY(batch_finish(e, j, sl));
                sl.shot = -1;
                if (next < j.nshots) {
                    TRY(batch_flush(e, sl));
                    TRY(batch_start(e, j, sl, next++));
                }
                continue;
            }
            const SlotOp& op = sl.ops[sl.pc];
            if (op.kind == OP_LAUNCH) return PSDM_OK;
            switch (op.kind) {
                case OP_SAVE:
                    TRY(copy_state(e, sl.f, sl.ckpts + state_floats(sl.f) * (size_t)op.arg, true));
                    break;
                case OP_RESTORE:
                    TRY(copy_state(e, sl.f, sl.ckpts + state_floats(sl.f) * (size_t)op.arg, false));
                    break;
                case OP_RESET: TRY(reset_state(e, &sl.s)); break;
                case OP_RESET_F: TRY(reset_state(e, &sl.f)); break;
                default: {  // OP_QUANT
                    const int m = op.arg;
                    const int qr = launch_quantize(sl.mb.stage[m & 3], sl.mb.amax + (m - 1), op.dst,
                                                   sl.mb.iscale + (m - 1), (int)sl.mb.fstride, sl.mb.kind, e->stream);
                    if (qr) return fail(PSDM_ERR_CUDA, "snapshot conversion launch: %s",
                                        cudaGetErrorString((cudaError_t)qr));
                    e->launches += 1;
                }
            }
            ++sl.pc;
        }
    };
    // The time loop is captured in CUDA graphs: the launches between two host
    // operations of any slot are queued and replayed as graphs of up to
    // kBatchRun launches (an executable graph per run length, updated in
    // place with the run's parameters).
    struct Queued {
        bool pairs;
        BatchParams bp;
        PairBatchParams pb;
    };
    constexpr int kBatchRun = 64;
    std::vector<Queued> queued;
    auto launch_one = [&](const Queued& q, cudaStream_t st) {
        return q.pairs ? launch_pair_batch(q.pb, e->num_sms, st) : launch_batch_step(q.bp, e->num_sms, st);
    };
    auto flush = [&]() -> int {
        if (queued.empty()) return PSDM_OK;
        bool done = false;
        if (e->use_graphs && queued.size() >= 8) {
            cudaStream_t cs = e->own_stream;
            cudaGraph_t graph = nullptr;
            bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                for (const Queued& q : queued)
                    if (launch_one(q, cs) != 0) {
                        ok = false;
                        break;
                    }
                ok = (cudaStreamEndCapture(cs, &graph) == cudaSuccess) && ok;
            }
            cudaGraphExec_t& ex = e->bgraphs[(int)queued.size()];
            if (ok && ex) {
                cudaGraphExecUpdateResultInfo info;
                if (cudaGraphExecUpdate(ex, graph, &info) != cudaSuccess) {
                    cudaGraphExecDestroy(ex);
                    ex = nullptr;
                }
            }
            if (ok && !ex) ok = cudaGraphInstantiate(&ex, graph, 0) == cudaSuccess;
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();  // clear a failed capture or update
            if (ok) {
                CUDA_TRY(cudaGraphLaunch(ex, e->stream));
                done = true;
            } else {
                if (ex) cudaGraphExecDestroy(ex);
                e->bgraphs.erase((int)queued.size());
                e->use_graphs = false;
            }
        }
        if (!done)
            for (const Queued& q : queued) {
                const int lr = launch_one(q, e->stream);
                if (lr) return fail(PSDM_ERR_CUDA, "batched step launch: %s", cudaGetErrorString((cudaError_t)lr));
            }
        queued.clear();
        return PSDM_OK;
    };
    int sel = 0;
    while (rc == PSDM_OK) {
        bool host_op = false;  // a slot is due for a state operation, or done
        for (BatchSlot& sl : slots)
            host_op = host_op || (sl.shot >= 0 && (sl.pc >= sl.ops.size() || sl.ops[sl.pc].kind != OP_LAUNCH));
        if (host_op) rc = flush();
        for (BatchSlot& sl : slots)
            if (rc == PSDM_OK) rc = advance(sl);
        if (rc != PSDM_OK) break;
        BatchParams bp;
        PairBatchParams pb;
        std::memset(&bp, 0, sizeof(bp));
        std::memset(&pb, 0, sizeof(pb));
        int n = 0;
        bool pairs = false;
        for (BatchSlot& sl : slots) {
            if (sl.shot < 0) continue;
            const SlotOp& op = sl.ops[sl.pc];
            pairs = sl.pairs;  // the same for every slot of a call
            bp.mode[n] = pb.mode[n] = op.mode;
            if (sl.pairs)
                pb.args[n] = sl.d_pargs + op.arg;
            else
                bp.args[n] = sl.d_args + op.arg;
            bp.first[n + 1] = pb.first[n + 1] = bp.first[n] + op.tiles;
            ++n;
        }
        if (n == 0) break;
        bp.nslots = pb.nslots = n;
        bp.counter = pb.counter = counters;
        bp.counter_sel = pb.counter_sel = sel;
        sel ^= 1;
        queued.push_back(Queued{pairs, bp, pb});
        if ((int)queued.size() == kBatchRun) rc = flush();
        e->launches += 1;
        for (BatchSlot& sl : slots)
            if (sl.shot >= 0) ++sl.pc;
    }
    if (rc == PSDM_OK) rc = flush();
    for (BatchSlot& sl : slots) {
        if (rc == PSDM_OK) rc = batch_flush(e, sl);
        if (sl.staged) {
            cudaEventSynchronize(sl.staged);
            cudaEventDestroy(sl.staged);
        }
    }
    return rc;
}

// One mixed-precision shot with checkpoints: the batched engine's
// checkpointed program in one slot.
int rtm_shot_mixed_ckpt(psdm_engine* e, const psdm_params* prm, int NumRec, int nxSou, int nySou, const int* nxRec,
                        const int* nyRec, const float* d_S, const float* d_tgt, float dd, float dt, int ny, int nx,
                        int nx_w, const float* d_vp, float added_space, int store_snap, int nt_prop2, int nt_taper,
                        int taper_option, int N_taper, int N_zeros, float* d_img) {
    psdm_shot sh{NumRec, nxSou, nySou, nxRec, nyRec, nx_w, nt_prop2, nt_taper, d_vp, d_tgt, d_img};
    BatchJob j{prm, &sh, 1, d_S, dd, dt, added_space, ny, nx, store_snap, taper_option, N_taper, N_zeros, false};
    const int slots = e->batch_slots;
    const int rc = run_batch(e, j, 1);
    e->batch_slots = slots;
    return rc;
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
    {
        int rc = prepare_step_kernels();
        if (rc == 0) rc = prepare_pair_kernels();
        if (rc) return fail(PSDM_ERR_CUDA, "preparing the step kernels: %s", cudaGetErrorString((cudaError_t)rc));
    }
    psdm_engine* e = new psdm_engine();
    e->device = device;
    cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device);
    err = cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
        delete e;
        return fail(PSDM_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(err));
    }
    e->stream = e->own_stream;
    void* h = nullptr;
    err = cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped);
    if (err == cudaSuccess) err = cudaHostGetDevicePointer((void**)&e->d_err, h, 0);
    if (err != cudaSuccess) {
        cudaStreamDestroy(e->own_stream);
        delete e;
        return fail(PSDM_ERR_CUDA, "mapped error word: %s", cudaGetErrorString(err));
    }
    e->h_err = (volatile int*)h;
    *e->h_err = 0;
    *out = e;
    return PSDM_OK;
}

int psdm_engine_destroy(psdm_engine* e) {
    if (!e) return PSDM_OK;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    int rc = e->trim();
    for (cudaEvent_t ev : e->events) cudaEventDestroy(ev);
    for (cudaEvent_t ev : e->pass_staged)
        if (ev) cudaEventDestroy(ev);
    if (e->h_err) cudaFreeHost((void*)e->h_err);
    cudaStreamDestroy(e->own_stream);
    delete e;
    return rc;
}

int psdm_engine_set_stream(psdm_engine* e, void* stream) {
    TRY(check_engine(e));
    TRY(sync(e));
    e->stream = stream ? (cudaStream_t)stream : e->own_stream;
    return PSDM_OK;
}

int psdm_engine_set_profiling(psdm_engine* e, int32_t on) {
    TRY(check_engine(e));
    TRY(sync(e));
    e->profiling = on != 0;
    e->events_used = 0;
    return PSDM_OK;
}

int psdm_engine_stats(psdm_engine* e, psdm_stats* out) {
    TRY(check_engine(e));
    if (!out) return fail(PSDM_ERR_ARG, "out is NULL");
    TRY(sync(e));
    std::memset(out, 0, sizeof(*out));
    out->launches = e->launches;
    out->fwd_steps = e->fwd_steps;
    out->bwd_steps = e->bwd_steps;
    double f = 0.0, b = 0.0;
    for (size_t i = 0; i + 3 <= e->events_used; i += 3) {
        float t1 = 0.f, t2 = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&t1, e->events[i], e->events[i + 1]));
        CUDA_TRY(cudaEventElapsedTime(&t2, e->events[i + 1], e->events[i + 2]));
        f += t1;
        b += t2;
        out->shots += 1;
    }
    out->fwd_ms = f;
    out->bwd_ms = b;
    return PSDM_OK;
}

int psdm_engine_reset_stats(psdm_engine* e) {
    TRY(check_engine(e));
    TRY(sync(e));
    e->launches = e->fwd_steps = e->bwd_steps = 0;
    e->events_used = 0;
    return PSDM_OK;
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
    TRY(setup_shot_host(e, prm, ny, nx_w, dd, dt, Vp_w, &s));
    WinGeom w;
    TRY(window_geometry(s.g, NumRec, nxSou[0], nySou[0], nxRec, nyRec, dd, nx, dd_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    float *d_S = nullptr, *d_F = nullptr, *d_rec = nullptr;
    TRY(e->get("S", (size_t)nt, &d_S));
    CUDA_TRY(cudaMemcpyAsync(d_S, Data_source, nt * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    const int nsnap = (nt - 1) / store_snap;
    if (Fields && nsnap > nt_snap) return fail(PSDM_ERR_ARG, "nt_snap=%d < %d snapshots", nt_snap, nsnap);
    if (Fields && nsnap > 0) TRY(e->get("fields", s.g.field_cells() * nsnap, &d_F));
    if (Data_synth && NumRec > 0) TRY(e->get("rec", (size_t)NumRec * nt, &d_rec));
    TRY(run_forward(e, s, nt, store_snap, d_S, w.zs, w.xs, d_F, nsnap, NumRec, w.rec_cell.data(), d_rec));
    if (d_F)  // pitched columns (ldf) -> dense Fields(ny, nx_w, slot)
        CUDA_TRY(cudaMemcpy2DAsync(Fields, (size_t)ny * sizeof(float), d_F, (size_t)s.g.ldf * sizeof(float),
                                   (size_t)ny * sizeof(float), (size_t)nx_w * nsnap, cudaMemcpyDeviceToHost,
                                   e->stream));
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
    TRY(setup_shot_host(e, prm, ny, nx_w, dd, dt, Vp_w, &s));
    WinGeom w;
    TRY(window_geometry(s.g, NumRec, nxSou[0], nySou[0], nxRec, nyRec, dd, nx, dd_space, &w));
    if (w.nx_w_calc != nx_w)
        return fail(PSDM_ERR_ARG, "nx_w=%d does not match the window of this geometry (%d)", nx_w, w.nx_w_calc);
    // Slots read: nt_snap - m for m = 1..(nt-1)/store_snap.
    const int nimg = (nt - 1) / store_snap;
    const int lo = nt_snap - nimg, hi = nt_snap - 1;
    if (lo < 1 && nimg > 0 && Fields)
        return fail(PSDM_ERR_ARG, "imaging would read snapshot slot %d < 1 (nt_snap=%d)", lo, nt_snap);
    const size_t hstride = (size_t)ny * nx_w;  // dense host slot
    const size_t ld = (size_t)s.g.ldf * sizeof(float), wb = (size_t)ny * sizeof(float);
    float *d_back = nullptr, *d_F = nullptr, *d_img = nullptr;
    if (NumRec > 0) {
        TRY(e->get("back", (size_t)NumRec * nt, &d_back));
        CUDA_TRY(cudaMemcpyAsync(d_back, AdjSource, (size_t)NumRec * nt * sizeof(float), cudaMemcpyHostToDevice,
                                 e->stream));
    }
    if (Fields && hi >= lo) {
        TRY(e->get("fields", s.g.field_cells() * (hi - lo + 1), &d_F));
        CUDA_TRY(cudaMemcpy2DAsync(d_F, ld, Fields + (size_t)(lo - 1) * hstride, wb, wb, (size_t)nx_w * (hi - lo + 1),
                                   cudaMemcpyHostToDevice, e->stream));
    }
    TRY(e->get("image_pitched", s.g.field_cells(), &d_img));
    CUDA_TRY(cudaMemcpy2DAsync(d_img, ld, PSDM_thread, wb, wb, nx_w, cudaMemcpyHostToDevice, e->stream));
    TRY(run_backward(e, s, nt, store_snap, nt_snap, d_back, 0, NumRec, w.zr.data(), w.xr.data(), d_F, lo, hi,
                     nullptr, d_img));
    CUDA_TRY(cudaMemcpy2DAsync(PSDM_thread, wb, d_img, ld, wb, nx_w, cudaMemcpyDeviceToHost, e->stream));
    return sync(e);
}

int psdm_rtm_shot(psdm_engine* e, const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
                  const int32_t* nxRec, const int32_t* nyRec, const float* Data_source, const float* Data_target,
                  float dd, float dt, int32_t ny, int32_t nx, int32_t nx_w, const float* Vp_w, float added_space,
                  int32_t store_snap, int32_t nt_snap, int32_t nt_prop2, int32_t nt_taper, int32_t taper_option,
                  int32_t N_taper, int32_t N_zeros, float* PSDM_w) {
    TRY(check_engine(e));
    if (!Data_source || !Data_target || !Vp_w || !PSDM_w || NumRec < 1 || nt_prop2 < 1 || nt_taper < 1 || ny < 1 ||
        nx_w < 1)
        return fail(PSDM_ERR_ARG, "null argument or empty size");
    const size_t fstride = (size_t)ny * nx_w;
    float *d_vp = nullptr, *d_S = nullptr, *d_tgt = nullptr, *d_img = nullptr;
    TRY(e->get("vp", fstride, &d_vp));
    TRY(e->get("S", (size_t)nt_prop2, &d_S));
    TRY(e->get("tgt", (size_t)NumRec * nt_taper, &d_tgt));
    TRY(e->get("image", fstride, &d_img));
    CUDA_TRY(cudaMemcpyAsync(d_vp, Vp_w, fstride * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(d_S, Data_source, nt_prop2 * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(d_tgt, Data_target, (size_t)NumRec * nt_taper * sizeof(float), cudaMemcpyHostToDevice,
                             e->stream));
    TRY(rtm_shot_core(e, prm, NumRec, nxSou, nySou, nxRec, nyRec, d_S, d_tgt, dd, dt, ny, nx, nx_w, d_vp, added_space,
                      store_snap, nt_snap, nt_prop2, nt_taper, taper_option, N_taper, N_zeros, d_img));
    CUDA_TRY(cudaMemcpyAsync(PSDM_w, d_img, fstride * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    return sync(e);
}

int psdm_rtm_shot_device(psdm_engine* e, const psdm_params* prm, int32_t NumRec, int32_t nxSou, int32_t nySou,
                         const int32_t* nxRec, const int32_t* nyRec, const float* d_Data_source,
                         const float* d_Data_target, float dd, float dt, int32_t ny, int32_t nx, int32_t nx_w,
                         const float* d_Vp_w, float added_space, int32_t store_snap, int32_t nt_snap,
                         int32_t nt_prop2, int32_t nt_taper, int32_t taper_option, int32_t N_taper, int32_t N_zeros,
                         float* d_PSDM_w) {
    TRY(check_engine(e));
    if (!d_Data_source || !d_Data_target || NumRec < 1 || nt_prop2 < 1 || nt_taper < 1)
        return fail(PSDM_ERR_ARG, "null argument or empty size");
    // The traces are copied into engine buffers so that the captured step
    // loops (whose arguments include the trace pointers) can be replayed.
    float *d_S = nullptr, *d_tgt = nullptr;
    TRY(e->get("S", (size_t)nt_prop2, &d_S));
    TRY(e->get("tgt", (size_t)NumRec * nt_taper, &d_tgt));
    CUDA_TRY(cudaMemcpyAsync(d_S, d_Data_source, nt_prop2 * sizeof(float), cudaMemcpyDeviceToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(d_tgt, d_Data_target, (size_t)NumRec * nt_taper * sizeof(float),
                             cudaMemcpyDeviceToDevice, e->stream));
    return rtm_shot_core(e, prm, NumRec, nxSou, nySou, nxRec, nyRec, d_S, d_tgt, dd, dt, ny, nx, nx_w, d_Vp_w,
                         added_space, store_snap, nt_snap, nt_prop2, nt_taper, taper_option, N_taper, N_zeros,
                         d_PSDM_w);
}

int psdm_rtm_batch(psdm_engine* e, const psdm_params* prm, int32_t nshots, const psdm_shot* shots,
                   const float* Data_source, float dd, float dt, int32_t ny, int32_t nx, float added_space,
                   int32_t store_snap, int32_t taper_option, int32_t N_taper, int32_t N_zeros, int32_t max_slots) {
    TRY(check_engine(e));
    TRY(check_params(prm));
    if (prm->precision != PSDM_PREC_FP32 && prm->precision != PSDM_PREC_FP16 && prm->precision != PSDM_PREC_BF16)
        return fail(PSDM_ERR_ARG, "unknown precision %d", prm->precision);
    if (nshots < 0 || (nshots > 0 && (!shots || !Data_source))) return fail(PSDM_ERR_ARG, "null argument");
    if (store_snap < 1) return fail(PSDM_ERR_ARG, "store_snap must be >= 1");
    if (taper_option != 0 && N_taper < 1) return fail(PSDM_ERR_ARG, "N_taper must be >= 1");
    int ntmax = 0;
    for (int i = 0; i < nshots; ++i) ntmax = std::max(ntmax, shots[i].nt_prop2);
    float* d_S = nullptr;
    TRY(e->get("S", (size_t)std::max(ntmax, 1), &d_S));
    CUDA_TRY(cudaMemcpyAsync(d_S, Data_source, (size_t)ntmax * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    BatchJob j{prm, shots, nshots, d_S, dd, dt, added_space, ny, nx, store_snap, taper_option, N_taper, N_zeros, true};
    TRY(run_batch(e, j, max_slots));
    return sync(e);
}

int psdm_rtm_batch_device(psdm_engine* e, const psdm_params* prm, int32_t nshots, const psdm_shot* shots,
                          const float* d_Data_source, float dd, float dt, int32_t ny, int32_t nx, float added_space,
                          int32_t store_snap, int32_t taper_option, int32_t N_taper, int32_t N_zeros,
                          int32_t max_slots) {
    TRY(check_engine(e));
    TRY(check_params(prm));
    if (prm->precision != PSDM_PREC_FP32 && prm->precision != PSDM_PREC_FP16 && prm->precision != PSDM_PREC_BF16)
        return fail(PSDM_ERR_ARG, "unknown precision %d", prm->precision);
    if (nshots < 0 || (nshots > 0 && (!shots || !d_Data_source))) return fail(PSDM_ERR_ARG, "null argument");
    if (store_snap < 1) return fail(PSDM_ERR_ARG, "store_snap must be >= 1");
    if (taper_option != 0 && N_taper < 1) return fail(PSDM_ERR_ARG, "N_taper must be >= 1");
    BatchJob j{prm, shots, nshots, d_Data_source, dd, dt, added_space, ny, nx, store_snap, taper_option, N_taper,
               N_zeros, false};
    TRY(run_batch(e, j, max_slots));
    return sync(e);
}

int32_t psdm_engine_batch_slots(const psdm_engine* e) { return e ? e->batch_slots : 0; }

int psdm_plan_memory(const psdm_params* prm, int32_t ny, int32_t nx_w, int32_t nt_prop2, int32_t nt_taper,
                     int32_t store_snap, int32_t NumRec, int64_t budget_bytes, int32_t max_slots, psdm_plan* out) {
    if (!prm || !out) return fail(PSDM_ERR_ARG, "null argument");
    TRY(check_params(prm));
    if (ny < 1 || nx_w < 1 || nt_prop2 < 2 || nt_taper < nt_prop2 || store_snap < 1 || NumRec < 0 ||
        budget_bytes < 0)
        return fail(PSDM_ERR_ARG, "need a non-empty window, 2 <= nt_prop2 <= nt_taper, store_snap >= 1");
    std::memset(out, 0, sizeof(*out));
    out->steps_per_launch = 1;
    out->budget_bytes = budget_bytes;
    const Grid g = make_grid(prm->dPML, ny, nx_w);
    const double cells = (double)g.cells(), field = (double)g.field_cells();
    const int nsnap = (nt_prop2 - 1) / store_snap;
    const double reserve = (double)(int64_t(1) << 30);
    const double avail = (double)budget_bytes - reserve;
    // One shot in flight: 13 grids (four wavefield levels, c2, phi and chi
    // at two levels each), the pitched image, the launch arguments of both
    // passes and the model window and traces.
    const double base = 13.0 * cells * 4 + field * 4 + (double)(nt_prop2 + nt_taper) / 2 * sizeof(PairArgs) +
                        ((double)ny * nx_w + (double)NumRec * nt_taper + nt_prop2) * 4;
    const int mslots = std::min(max_slots > 0 ? (int)max_slots : kMaxSlots, kMaxSlots);
    const bool mixed = prm->precision != PSDM_PREC_FP32;
    auto slots_of = [&](double per) { return (int)std::min<double>(avail > 0 ? std::floor(avail / per) : 0.0, mslots); };
    // All snapshots: 16-bit slots with four FP32 staging buffers and the
    // Kahan compensation, or FP32 slots.
    const double all = mixed ? base + (double)nsnap * field * 2 + 5.0 * field * 4 : base + (double)nsnap * field * 4;
    if (all <= avail) {
        out->bytes_per_slot = (int64_t)all;
        out->slots = slots_of(all);
        out->fits = 1;
        return PSDM_OK;
    }
    // Checkpoints every K steps: the state (8 grids and two history rows) at
    // each segment start but the first, one segment's snapshots (K FP32
    // slots, or K/ks + 2 16-bit slots with the staging buffers), and the
    // recomputing state's own grids; the memory is smallest near
    // K = sqrt(steps * state / snapshot).  The recomputation costs one more
    // forward pass whatever K is.
    const int nsteps = nt_prop2 - 1;
    const double state = (8.0 * cells + 2.0 * g.nxt) * 4;
    auto mem = [&](int K) {
        const int nseg = (nsteps + K - 1) / K;
        const double seg = mixed ? (double)(K / store_snap + 2) * field * 2 + 5.0 * field * 4 : (double)K * field * 4;
        return base + 13.0 * cells * 4 + seg + (double)(nseg - 1) * state;
    };
    int best = 1;
    for (int K = 1; K <= nsteps; ++K)
        if (mem(K) < mem(best)) best = K;
    best = std::max(best, std::min(16, nsteps));  // at most one state copy per 16 steps
    out->bytes_per_slot = (int64_t)mem(best);
    if (mem(best) > avail)
        return fail(PSDM_ERR_NOMEM, "one %s shot needs %.2f GB even with checkpoints every %d steps, the budget "
                    "leaves %.2f GB", mixed ? "mixed-precision" : "FP32", mem(best) / 1e9, best, avail / 1e9);
    out->checkpoint_interval = best;
    out->slots = slots_of(mem(best));
    out->fits = 1;
    return PSDM_OK;
}

int psdm_engine_autotune(psdm_engine* e, const psdm_params* prm, int32_t ny, int32_t nx_w, int32_t nt_prop2,
                         int32_t nt_taper, int32_t store_snap, int32_t NumRec, int64_t budget_bytes,
                         int32_t max_slots, int32_t probe, psdm_plan* out) {
    TRY(check_engine(e));
    TRY(sync(e));
    if (budget_bytes == 0) {
        size_t fr = 0, tot = 0;
        CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        budget_bytes = (int64_t)fr + e->total();
    }
    TRY(psdm_plan_memory(prm, ny, nx_w, nt_prop2, nt_taper, store_snap, NumRec, budget_bytes, max_slots, out));
    if (probe) {
        // A 40-step forward pass of the window (2000 m/s, no snapshots) in
        // each launch form, timed on the engine's stream after a warm-up.
        psdm_params p1 = *prm;
        p1.precision = PSDM_PREC_FP32;
        const int nt = 41;
        std::vector<float> vp((size_t)ny * nx_w, 2000.0f);
        float* d_vp = nullptr;
        float* d_S = nullptr;
        TRY(e->get("probe_vp", vp.size(), &d_vp));
        TRY(e->get("probe_S", (size_t)nt, &d_S));
        CUDA_TRY(cudaMemcpyAsync(d_vp, vp.data(), vp.size() * sizeof(float), cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaMemsetAsync(d_S, 0, nt * sizeof(float), e->stream));
        const int spl0 = e->steps_per_launch;
        cudaEvent_t t0 = nullptr, t1 = nullptr;
        CUDA_TRY(cudaEventCreate(&t0));
        CUDA_TRY(cudaEventCreate(&t1));
        int rc = PSDM_OK;
        for (int spl = 1; spl <= 2 && rc == PSDM_OK; ++spl) {
            e->steps_per_launch = spl;
            Shot s;
            rc = setup_shot(e, &p1, ny, nx_w, 10.f, 1e-3f, d_vp, &s, "_probe");
            const int zs = s.g.dn + std::min(2, ny) - 1, xs = s.g.dn + nx_w / 2;
            float ms = 0.f;
            for (int rep = 0; rep < 2 && rc == PSDM_OK; ++rep) {
                if (rep == 1 && cudaEventRecord(t0, e->stream) != cudaSuccess) rc = PSDM_ERR_CUDA;
                if (rc == PSDM_OK) rc = run_forward(e, s, nt, 1, d_S, zs, xs, nullptr, 0, 0, nullptr, nullptr);
                if (rc == PSDM_OK && rep == 1 && cudaEventRecord(t1, e->stream) != cudaSuccess) rc = PSDM_ERR_CUDA;
            }
            if (rc == PSDM_OK && cudaEventSynchronize(t1) == cudaSuccess && cudaEventElapsedTime(&ms, t0, t1) ==
                                                                                 cudaSuccess)
                out->probe_us[spl - 1] = ms * 1e3f / (nt - 1);
        }
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        e->steps_per_launch = spl0;
        TRY(rc);
        TRY(sync(e));
        out->steps_per_launch = (out->probe_us[0] > 0.f && out->probe_us[0] < out->probe_us[1]) ? 1 : 2;
    }
    e->steps_per_launch = out->steps_per_launch;
    e->ckpt_interval = out->checkpoint_interval;
    return PSDM_OK;
}

int psdm_engine_set_pass_launch(psdm_engine* e, int32_t on) {
    TRY(check_engine(e));
    if (on < 0 || on > 2) return fail(PSDM_ERR_ARG, "pass launch form must be 0, 1 or 2 (got %d)", on);
    e->use_pass = on;
    return PSDM_OK;
}

int psdm_engine_set_steps_per_launch(psdm_engine* e, int32_t steps) {
    TRY(check_engine(e));
    if (steps != 1 && steps != 2) return fail(PSDM_ERR_ARG, "steps per launch must be 1 or 2 (got %d)", steps);
    TRY(sync(e));
    e->steps_per_launch = steps;
    return PSDM_OK;
}

int psdm_engine_set_reconstruction(psdm_engine* e, int32_t on) {
    TRY(check_engine(e));
    TRY(sync(e));
    e->recon = on != 0;
    return PSDM_OK;
}

int psdm_engine_set_checkpointing(psdm_engine* e, int32_t interval) {
    TRY(check_engine(e));
    if (interval < 0) return fail(PSDM_ERR_ARG, "checkpoint interval must be >= 0");
    TRY(sync(e));
    e->ckpt_interval = interval;
    return PSDM_OK;
}

int psdm_condition_traces_device(psdm_engine* e, const psdm_conditioning* c, int32_t NumRec,
                                 const float* d_Field_Data, int32_t nt_data, float dt_data, float dt_prop,
                                 const int32_t* nt_cut, const int32_t* nt_sf, const int32_t* lens,
                                 float* d_Data_target) {
    TRY(check_engine(e));
    if (!c || !d_Field_Data || !nt_cut || !nt_sf || !lens || !d_Data_target || NumRec < 0)
        return fail(PSDM_ERR_ARG, "null argument");
    const int nt_prop2 = lens[0], nt_taper = lens[1], N_taper = lens[2], N_zeros = lens[3];
    if (nt_data < 1 || nt_prop2 < 0 || nt_taper < nt_prop2 || N_taper < 1 || N_zeros < 0)
        return fail(PSDM_ERR_ARG, "inconsistent trace lengths");
    if (dt_data != dt_prop && (dt_data <= 0.f || dt_prop <= 0.f)) return fail(PSDM_ERR_ARG, "time steps must be > 0");
    if (NumRec == 0) return PSDM_OK;
    int *d_cut = nullptr, *d_sf = nullptr;
    float* d_w = nullptr;
    TRY(e->get("cond_cut", (size_t)NumRec, &d_cut));
    TRY(e->get("cond_sf", (size_t)NumRec, &d_sf));
    TRY(e->get("cond_w", (size_t)N_taper, &d_w));
    std::vector<float> w(N_taper);
    for (int n = 0; n < N_taper; ++n) w[n] = taper_weight(n, N_taper);
    CUDA_TRY(cudaMemcpyAsync(d_cut, nt_cut, NumRec * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(d_sf, nt_sf, NumRec * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(d_w, w.data(), N_taper * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    CondArgs a;
    a.field = d_Field_Data;
    a.out = d_Data_target;
    a.nt_cut = d_cut;
    a.nt_sf = d_sf;
    a.w = d_w;
    a.nrec = NumRec;
    a.nt_data = nt_data;
    a.nt_prop2 = nt_prop2;
    a.nt_taper = nt_taper;
    a.N_taper = N_taper;
    a.N_zeros = N_zeros;
    a.cut_multiple = c->cut_multiple;
    a.cut_sf = c->cut_sf;
    a.taper_option = c->taper_option;
    a.resample = dt_data != dt_prop ? 1 : 0;
    a.dt_data = dt_data;
    a.dt_prop = dt_prop;
    const int rc = launch_condition(a, e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "conditioning launch: %s", cudaGetErrorString((cudaError_t)rc));
    e->launches += 1;
    return PSDM_OK;
}

int psdm_condition_traces(psdm_engine* e, const psdm_conditioning* c, int32_t NumRec, const float* Field_Data,
                          int32_t nt_data, float dt_data, float dt_prop, const int32_t* nt_cut, const int32_t* nt_sf,
                          const int32_t* lens, float* Data_target) {
    TRY(check_engine(e));
    if (!Field_Data || !Data_target || !lens || NumRec < 0) return fail(PSDM_ERR_ARG, "null argument");
    if (NumRec == 0) return PSDM_OK;
    const size_t nin = (size_t)NumRec * nt_data, nout = (size_t)NumRec * lens[1];
    float *d_in = nullptr, *d_out = nullptr;
    TRY(e->get("cond_in", nin, &d_in));
    TRY(e->get("cond_out", std::max<size_t>(nout, 1), &d_out));
    CUDA_TRY(cudaMemcpyAsync(d_in, Field_Data, nin * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    TRY(psdm_condition_traces_device(e, c, NumRec, d_in, nt_data, dt_data, dt_prop, nt_cut, nt_sf, lens, d_out));
    CUDA_TRY(cudaMemcpyAsync(Data_target, d_out, nout * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    return sync(e);
}

int psdm_freq_filter_device(psdm_engine* e, float* d_traces, int32_t nt, float dt, int32_t Num, int32_t typef,
                            float f1, float f2) {
    TRY(check_engine(e));
    if (!d_traces || nt < 1 || Num < 0 || !(dt > 0.f)) return fail(PSDM_ERR_ARG, "null argument or empty trace");
    if (typef < 1 || typef > 3) return fail(PSDM_ERR_ARG, "typef must be 1 (low-pass), 2 (high-pass) or 3 (band-pass)");
    if (Num == 0) return PSDM_OK;
    const int ts = 24 * nt;  // zero_pad = 24 (auxiliar.f90:511-512)
    std::vector<std::complex<float>> H(ts);
    butterworth_response(ts, 1.f / dt, typef, f1, f2, H.data());
    float *d_H = nullptr, *d_x = nullptr;
    int* d_keep = nullptr;
    TRY(e->get("filt_H", (size_t)(ts / 2 + 1) * 2, &d_H));
    TRY(e->get("filt_x", filter_work_floats(ts, Num), &d_x));
    TRY(e->get("filt_keep", (size_t)Num, &d_keep));
    CUDA_TRY(cudaMemcpyAsync(d_H, H.data(), (size_t)(ts / 2 + 1) * sizeof(std::complex<float>),
                             cudaMemcpyHostToDevice, e->stream));
    auto key = std::make_pair(ts, (int)Num);
    auto it = e->fft_plans.find(key);
    if (it == e->fft_plans.end()) {
        std::array<int, 2> plans{};
        if (make_fft_plans(ts, Num, plans.data()))
            return fail(PSDM_ERR_CUDA, "cuFFT plans of length %d x %d failed", ts, Num);
        it = e->fft_plans.emplace(key, plans).first;
    }
    const int rc = filter_traces(d_traces, nt, Num, d_H, d_x, d_keep, ts, it->second.data(), e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "frequency filter failed (step %d)", rc);
    e->launches += 5;
    return PSDM_OK;
}

int psdm_freq_filter(psdm_engine* e, float* traces, int32_t nt, float dt, int32_t Num, int32_t typef, float f1,
                     float f2) {
    TRY(check_engine(e));
    if (!traces || nt < 1 || Num < 0) return fail(PSDM_ERR_ARG, "null argument or empty trace");
    if (Num == 0) return PSDM_OK;
    float* d = nullptr;
    TRY(e->get("filt_traces", (size_t)nt * Num, &d));
    CUDA_TRY(cudaMemcpyAsync(d, traces, (size_t)nt * Num * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    TRY(psdm_freq_filter_device(e, d, nt, dt, Num, typef, f1, f2));
    CUDA_TRY(cudaMemcpyAsync(traces, d, (size_t)nt * Num * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
    return sync(e);
}

int psdm_engine_check_wait_timeout(psdm_engine* e) {
    TRY(check_engine(e));
    TRY(sync(e));
    const int rc = launch_wait_timeout_probe(e->d_err, e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "probe launch: %s", cudaGetErrorString((cudaError_t)rc));
    return sync(e);
}

int psdm_engine_dt_quotients(psdm_engine* e, float dt, const float* x, int32_t n, float* q) {
    TRY(check_engine(e));
    if (!x || !q || n <= 0 || n % 4) return fail(PSDM_ERR_ARG, "null argument, or n not a positive multiple of 4");
    TRY(sync(e));
    auto it = e->div_cache.find(dt);
    if (it == e->div_cache.end()) {
        float r = 0.f, lo = 0.f, hi = 0.f, tiny = 0.f;
        const int ok = fast_div_exact(dt, &r, &lo, &hi, &tiny) ? 1 : 0;
        it = e->div_cache.emplace(dt, std::make_pair(ok, std::vector<float>{r, lo, hi, tiny})).first;
    }
    const std::vector<float>& c = it->second.second;
    float *d_x = nullptr, *d_q = nullptr;
    TRY(e->get("dq_x", (size_t)n, &d_x));
    TRY(e->get("dq_q", (size_t)2 * n, &d_q));
    CUDA_TRY(cudaMemcpyAsync(d_x, x, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, e->stream));
    const int rc = launch_dt_quotients(dt, c[0], c[1], c[2], it->second.first, d_x, d_q, n, e->stream);
    if (rc) return fail(PSDM_ERR_CUDA, "quotient launch: %s", cudaGetErrorString((cudaError_t)rc));
    CUDA_TRY(cudaMemcpyAsync(q, d_q, (size_t)2 * n * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
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
    TRY(setup_shot_host(e, prm, ny, nx_w, dd, dt, Vp_w, &s));
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
