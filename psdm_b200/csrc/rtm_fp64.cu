// FP64 build of the time step: the error reference of the FP32 and mixed-
// precision forms on the GPU (no counterpart in the reference, whose solvers
// are FP32 throughout).
//
// The per-cell update is the one-step kernels' generic cell (rtm_device.cuh,
// cell_generic) evaluated in double precision in the same order: the 2nd
// and 1st derivative sums of src/solver_space_derivs_clean.f90 with the
// reference's edge rule, the C-PML recursions of
// src/solver_PML_matrices.f90:1-111 with factor f(max(kx, kz)) in corners,
// the strip and interior updates of src/solver_ac_forward_ram.f90:402-444,
// the free surface with the RAM solvers' strip-private histories
// (:449-473) or the disk solvers' order, the snapshot (p3 - p1) * 0.5 / dt
// (:476-488) and the imaging condition of
// src/solver_ac_backward_ram.f90:455-470.  Snapshots are taken every
// store_snap steps and imaged at the paired backward steps, the pairing of
// the engine's mixed-precision form (the reference's pairing for store_snap
// 1).  Set-up in double: FD coefficients as rationals, C-PML profiles from
// the closed form, c2 = c^2 dt^2 / d^2 from the FP32 model.
//
// One thread per cell, operands straight from HBM, one launch per step: the
// build exists for accuracy, not speed.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/psdm_rtm.h"
#include "rtm_internal.h"

namespace psdm {
namespace {

struct Step64 {
    const double* p;    // level n
    double* pm;         // level n-1 in, n+1 out (in place)
    const double* c2;
    const double* phix_in;
    double* phix_out;
    double* chix;
    const double* phiz_in;
    double* phiz_out;
    double* chiz;
    const double* side_p;  // free-surface histories (RAM order): level n
    double* side_pm;       // level n-1 in, n+1 out
    const double* fA;
    const double* fB;
    double cf1[4], cf2[4];
    int nyt, nxt, ldz, ny, nx, dn, zoff, ldf, fs, disk;
    const int* row_slot;   // injection map (as StepArgs)
    const int* inj_cols;
    const double* inj_trace;
    int inj_ld, inj_t;
    double* field;         // forward: snapshot written; backward: snapshot read; null = none
    double dt;
    double* image;
    double field_w, ss;
};

__device__ __forceinline__ int clampi64(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

#define D2D(AT, c)                                                                               \
    __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dadd_rn(AT(0), AT(0)), (c)[0]),                   \
                                  __dmul_rn(__dadd_rn(AT(1), AT(-1)), (c)[1])),                 \
                        __dmul_rn(__dadd_rn(AT(2), AT(-2)), (c)[2])),                           \
              __dmul_rn(__dadd_rn(AT(3), AT(-3)), (c)[3]))
#define D1D(AT, c)                                                                               \
    __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(AT(1), AT(-1)), (c)[1]),                            \
                        __dmul_rn(__dsub_rn(AT(2), AT(-2)), (c)[2])),                           \
              __dmul_rn(__dsub_rn(AT(3), AT(-3)), (c)[3]))

template <int MODE>
__global__ void step64_kernel(const Step64 a) {
    const int zd = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    const int z = zd - a.zoff;
    const int dn = a.dn;
    if (z < 0 || z >= a.nyt || x >= a.nxt) return;
    if (a.fs && z < dn) return;  // above a free surface: never updated
    const int kz = (z < dn) ? (dn - z) : (z >= dn + a.ny ? z - (dn + a.ny) + 1 : 0);
    const int kx = (x < dn) ? (dn - x) : (x >= dn + a.nx ? x - (dn + a.nx) + 1 : 0);
    const bool fsrow = a.fs && z == dn;
    const int cx = clampi64(x, 3, a.nxt - 4);
    const int czd = clampi64(z, 3, a.nyt - 4) + a.zoff;
    const double* colc = a.p + (size_t)cx * a.ldz + zd;
    const double* colz = a.p + (size_t)x * a.ldz + czd;
#define AX(k) colc[(ptrdiff_t)(k) * a.ldz]
#define AZ(k) colz[(k)]
    const double d2x = D2D(AX, a.cf2);
    const double d2y = D2D(AZ, a.cf2);
    const size_t g = (size_t)x * a.ldz + zd;
    const double pc = a.p[g];
    const double pmo = a.pm[g];
    const double c2v = a.c2[g];
    double pp = pc, ppm = pmo;
    if (fsrow && kx > 0 && !a.disk) { pp = a.side_p[x]; ppm = a.side_pm[x]; }
    const double base = __dadd_rn(-ppm, __dmul_rn(2.0, pp));
    double main_term, propz = 0.0;
    if (kx > 0 || kz > 0) {
        const int f = (kx > 0 && kz > 0) ? max(kx, kz) : (kx > 0 ? kx : kz);
        const double A = a.fA[f - 1], B = a.fB[f - 1];
        double propx = 0.0;
        if (kx > 0) {
            const double d1 = D1D(AX, a.cf1);
            const int sb = (x < dn) ? 0 : dn + a.nx;
            const int ci = clampi64(x - sb, 3, dn - 4) + sb;
            const double* ph = a.phix_in + (size_t)ci * a.ldz + zd;
#define PX(k) ph[(ptrdiff_t)(k) * a.ldz]
            const double dph = D1D(PX, a.cf1);
#undef PX
            const double phn = __dadd_rn(__dmul_rn(A, a.phix_in[g]), __dmul_rn(B, d1));
            const double chn = __dadd_rn(__dmul_rn(A, a.chix[g]), __dmul_rn(B, __dadd_rn(d2x, dph)));
            a.phix_out[g] = phn;
            a.chix[g] = chn;
            propx = __dadd_rn(dph, chn);
        }
        if (kz > 0) {
            const double d1 = D1D(AZ, a.cf1);
            const int sb = (z < dn) ? 0 : dn + a.ny;
            const int cj = clampi64(z - sb, 3, dn - 4) + sb + a.zoff;
            const double* ph = a.phiz_in + (size_t)x * a.ldz + cj;
#define PZ(k) ph[(k)]
            const double dph = D1D(PZ, a.cf1);
#undef PZ
            const double phn = __dadd_rn(__dmul_rn(A, a.phiz_in[g]), __dmul_rn(B, d1));
            const double chn = __dadd_rn(__dmul_rn(A, a.chiz[g]), __dmul_rn(B, __dadd_rn(d2y, dph)));
            a.phiz_out[g] = phn;
            a.chiz[g] = chn;
            propz = __dadd_rn(dph, chn);
        }
        main_term = (kx > 0) ? propx : propz;
    } else {
        double src = 0.0;
        if (a.row_slot != nullptr) {
            const int rs = a.row_slot[zd];
            if (rs >= 0) {
                const int j = a.inj_cols[rs * a.nxt + x];
                if (j >= 0) src = a.inj_trace[(size_t)j * a.inj_ld + a.inj_t];
            }
        }
        main_term = src;
    }
#undef AX
#undef AZ
    double p3 = __dadd_rn(base, __dmul_rn(c2v, __dadd_rn(__dadd_rn(d2x, d2y), main_term)));
    if (kx > 0 && kz > 0) p3 = __dadd_rn(p3, __dmul_rn(c2v, propz));
    double out = p3;
    if (fsrow) {
        if (kx > 0) {
            if (!a.disk) { a.side_pm[x] = p3; out = 0.0; }
        } else {
            out = 0.0;
        }
    }
    a.pm[g] = out;
    if (kx == 0 && kz == 0 && a.field != nullptr) {
        const size_t fi = (size_t)(x - dn) * a.ldf + (z - dn);
        if (MODE == 0) {
            a.field[fi] = __ddiv_rn(__dmul_rn(__dsub_rn(out, pmo), 0.5), a.dt);
        } else {
            double F = a.field[fi];
            if (a.field_w != 1.0) F = __dmul_rn(F, a.field_w);
            double inc = __dmul_rn(__dmul_rn(0.5, __dsub_rn(out, pmo)), F);
            if (a.ss != 1.0) inc = __dmul_rn(inc, a.ss);
            a.image[fi] = __dadd_rn(a.image[fi], inc);
        }
    }
}

// Padded c2 = ((c*c)*(dt*dt))/(dd*dd) in double from the FP32 model (edge
// replication; ram_padding: the RAM solvers' partial top and bottom strips).
__global__ void pad_c2_64_kernel(const float* vp, int ny, int nx, int dn, int nyt, int nxt, int ldz, int zoff,
                                 double dt, double dd, int ram_padding, double* c2) {
    const int zd = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    if (zd >= ldz || x >= nxt) return;
    const int z = zd - zoff;
    double v = 0.0;
    const bool strip_row = z < dn || z >= dn + ny;
    if (z >= 0 && z < nyt && !(ram_padding && strip_row && x >= 2 * dn && x < dn + nx)) {
        const int j = clampi64(z - dn, 0, ny - 1), i = clampi64(x - dn, 0, nx - 1);
        const double c = (double)vp[(size_t)i * ny + j];
        v = __ddiv_rn(__dmul_rn(__dmul_rn(c, c), __dmul_rn(dt, dt)), __dmul_rn(dd, dd));
    }
    c2[(size_t)x * ldz + zd] = v;
}

__global__ void widen_kernel(const float* in, double* out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

// Device buffers of one FP64 shot, freed on scope exit.
struct Dev64 {
    std::vector<void*> ptrs;
    ~Dev64() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t get(size_t n, T** out) {
        void* p = nullptr;
        const cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) {
            ptrs.push_back(p);
            cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T));
        }
        *out = static_cast<T*>(p);
        return e;
    }
};

}  // namespace
}  // namespace psdm

using namespace psdm;

#define F64_TRY(expr)                                                                               \
    do {                                                                                            \
        cudaError_t e_ = (expr);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            char m_[256];                                                                           \
            snprintf(m_, sizeof m_, "%s: %s", #expr, cudaGetErrorString(e_));                       \
            set_last_error(m_);                                                                     \
            return e_ == cudaErrorMemoryAllocation ? PSDM_ERR_NOMEM : PSDM_ERR_CUDA;                \
        }                                                                                           \
    } while (0)

static int f64_fail(int code, const char* msg) {
    set_last_error(msg);
    return code;
}

extern "C" int psdm_rtm_shot_fp64(int32_t device, const psdm_params* prm, int32_t NumRec, int32_t nxSou,
                                  int32_t nySou, const int32_t* nxRec, const int32_t* nyRec,
                                  const float* Data_source, const float* Data_target, float dd, float dt, int32_t ny,
                                  int32_t nx, int32_t nx_w, const float* Vp_w, float added_space, int32_t store_snap,
                                  int32_t nt_prop2, int32_t nt_taper, int32_t taper_option, int32_t N_taper,
                                  int32_t N_zeros, double* PSDM_w, double* Fields_out) {
    if (!prm || !nxRec || !nyRec || !Data_source || !Data_target || !Vp_w || !PSDM_w || NumRec < 1)
        return f64_fail(PSDM_ERR_ARG, "null argument or NumRec < 1");
    if (prm->dPML < 2 || (prm->strategy != 1 && prm->strategy != 2))
        return f64_fail(PSDM_ERR_ARG, "dPML must be >= 2 and strategy 1 or 2");
    if (nt_prop2 < 2 || nt_taper < nt_prop2 || store_snap < 1 || ny < 1 || nx_w < 1)
        return f64_fail(PSDM_ERR_ARG, "need 2 <= nt_prop2 <= nt_taper, store_snap >= 1 and a non-empty window");
    if (taper_option != 0 && N_taper < 1) return f64_fail(PSDM_ERR_ARG, "N_taper must be >= 1");
    F64_TRY(cudaSetDevice(device));
    const Grid g = make_grid(prm->dPML, ny, nx_w);
    if (prm->strategy == 1 && nx_w < g.dn) return f64_fail(PSDM_ERR_ARG, "RAM ordering needs nx_w >= dPML+6");
    int nx_wc = 0, x_i = 0, x_f = 0;
    psdm_dynamic_window(NumRec, nxSou, nxRec, dd, nx, added_space, &nx_wc, &x_i, &x_f);
    if (nx_wc != nx_w) return f64_fail(PSDM_ERR_ARG, "nx_w does not match the window of this geometry");
    // Injection maps (window coordinates shifted as the solver wrappers do,
    // src/dynamic_window.f90:80-86); points in the C-PML are not injected.
    auto build = [&](int n, const int* zs, const int* xs, std::vector<int>* rows, std::vector<int>* cols) -> bool {
        rows->assign(g.ldz, -1);
        cols->clear();
        int nslot = 0;
        for (int j = 0; j < n; ++j) {
            const int z = zs[j], x = xs[j];
            if (z < 0 || z >= g.nyt || x < 0 || x >= g.nxt) return false;
            if (z < g.dn || z >= g.dn + g.ny || x < g.dn || x >= g.dn + g.nx) continue;
            int& r = (*rows)[z + g.zoff];
            if (r < 0) {
                r = nslot++;
                cols->resize((size_t)nslot * g.nxt, -1);
            }
            (*cols)[(size_t)r * g.nxt + x] = j;
        }
        return true;
    };
    std::vector<int> zr(NumRec), xr(NumRec);
    for (int r = 0; r < NumRec; ++r) {
        zr[r] = g.dn + nyRec[r] - 1;
        xr[r] = g.dn + (nxRec[r] - x_i + 1) - 1;
    }
    const int zs0 = g.dn + nySou - 1, xs0 = g.dn + (nxSou - x_i + 1) - 1;
    std::vector<int> srow, scol, rrow, rcol;
    if (!build(1, &zs0, &xs0, &srow, &scol) || !build(NumRec, zr.data(), xr.data(), &rrow, &rcol))
        return f64_fail(PSDM_ERR_ARG, "a source or receiver lies outside the padded grid");

    const size_t n = g.cells(), fstride = g.field_cells();
    const int nsnap = (nt_prop2 - 1) / store_snap;
    Dev64 D;
    double *p0, *p1, *c2, *phx0, *phx1, *chx, *phz0, *phz1, *chz, *s0, *s1, *fA, *fB, *S, *T, *F, *img;
    float *vp32, *src32, *tgt32;
    int *d_srow, *d_scol, *d_rrow, *d_rcol;
    for (double** b : {&p0, &p1, &c2, &phx0, &phx1, &chx, &phz0, &phz1, &chz}) F64_TRY(D.get(n, b));
    F64_TRY(D.get((size_t)g.nxt, &s0));
    F64_TRY(D.get((size_t)g.nxt, &s1));
    F64_TRY(D.get((size_t)g.dn, &fA));
    F64_TRY(D.get((size_t)g.dn, &fB));
    F64_TRY(D.get((size_t)nt_prop2, &S));
    F64_TRY(D.get((size_t)NumRec * nt_taper, &T));
    F64_TRY(D.get(fstride * std::max(nsnap, 1), &F));
    F64_TRY(D.get(fstride, &img));
    F64_TRY(D.get((size_t)ny * nx_w, &vp32));
    F64_TRY(D.get((size_t)nt_prop2, &src32));
    F64_TRY(D.get((size_t)NumRec * nt_taper, &tgt32));
    F64_TRY(D.get(srow.size(), &d_srow));
    F64_TRY(D.get(std::max<size_t>(scol.size(), 1), &d_scol));
    F64_TRY(D.get(rrow.size(), &d_rrow));
    F64_TRY(D.get(std::max<size_t>(rcol.size(), 1), &d_rcol));
    F64_TRY(cudaMemcpy(vp32, Vp_w, (size_t)ny * nx_w * sizeof(float), cudaMemcpyHostToDevice));
    F64_TRY(cudaMemcpy(src32, Data_source, (size_t)nt_prop2 * sizeof(float), cudaMemcpyHostToDevice));
    // BackSource(:, j) = Data_target(nt_taper:1:-1, j) (calculate_PSDM_RTM.f90:448-450)
    std::vector<float> back((size_t)NumRec * nt_taper);
    for (int r = 0; r < NumRec; ++r)
        for (int t = 0; t < nt_taper; ++t)
            back[(size_t)r * nt_taper + t] = Data_target[(size_t)r * nt_taper + (nt_taper - 1 - t)];
    F64_TRY(cudaMemcpy(tgt32, back.data(), back.size() * sizeof(float), cudaMemcpyHostToDevice));
    widen_kernel<<<256, 256>>>(src32, S, (size_t)nt_prop2);
    widen_kernel<<<1024, 256>>>(tgt32, T, back.size());
    F64_TRY(cudaMemcpy(d_srow, srow.data(), srow.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!scol.empty()) F64_TRY(cudaMemcpy(d_scol, scol.data(), scol.size() * sizeof(int), cudaMemcpyHostToDevice));
    F64_TRY(cudaMemcpy(d_rrow, rrow.data(), rrow.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!rcol.empty()) F64_TRY(cudaMemcpy(d_rcol, rcol.data(), rcol.size() * sizeof(int), cudaMemcpyHostToDevice));
    std::vector<double> hA(g.dn), hB(g.dn);
    pml_profiles_f64(kAcc, g.dPML, (double)dt, (double)dd, g.dn, hA.data(), hB.data());
    F64_TRY(cudaMemcpy(fA, hA.data(), g.dn * sizeof(double), cudaMemcpyHostToDevice));
    F64_TRY(cudaMemcpy(fB, hB.data(), g.dn * sizeof(double), cudaMemcpyHostToDevice));
    const dim3 grid((g.ldz + 127) / 128, g.nxt);
    pad_c2_64_kernel<<<grid, 128>>>(vp32, ny, nx_w, g.dn, g.nyt, g.nxt, g.ldz, g.zoff, (double)dt, (double)dd,
                                    prm->strategy == 2 ? 0 : 1, c2);
    F64_TRY(cudaGetLastError());

    Step64 a;
    std::memset(&a, 0, sizeof a);
    a.c2 = c2;
    a.chix = chx;
    a.chiz = chz;
    a.fA = fA;
    a.fB = fB;
    fd_coef_f64(1, a.cf1);
    fd_coef_f64(2, a.cf2);
    a.nyt = g.nyt; a.nxt = g.nxt; a.ldz = g.ldz; a.ny = g.ny; a.nx = g.nx; a.dn = g.dn; a.zoff = g.zoff;
    a.ldf = g.ldf;
    a.fs = prm->fs != 0;
    a.disk = prm->strategy == 2;
    a.dt = (double)dt;
    a.image = img;
    a.field_w = 1.0;
    a.ss = 1.0;
    double* P[2] = {p0, p1};
    double* PX[2] = {phx0, phx1};
    double* PZ[2] = {phz0, phz1};
    double* SD[2] = {s0, s1};
    auto bufs = [&](int it) {
        const int c = it & 1;
        a.p = P[c];
        a.pm = P[c ^ 1];
        a.phix_in = PX[c];
        a.phix_out = PX[c ^ 1];
        a.phiz_in = PZ[c];
        a.phiz_out = PZ[c ^ 1];
        a.side_p = SD[c];
        a.side_pm = SD[c ^ 1];
    };
    // Forward pass, k = 2..nt_prop2: slot m at the steps with (k-1) % ks == 0.
    a.row_slot = d_srow;
    a.inj_cols = d_scol;
    a.inj_trace = S;
    a.inj_ld = 0;
    for (int k = 2; k <= nt_prop2; ++k) {
        bufs(k - 2);
        a.inj_t = k - 2;
        a.field = nullptr;
        if ((k - 1) % store_snap == 0 && (k - 1) / store_snap <= nsnap)
            a.field = F + (size_t)((k - 1) / store_snap - 1) * fstride;
        step64_kernel<0><<<grid, 128>>>(a);
    }
    F64_TRY(cudaGetLastError());
    if (Fields_out && nsnap > 0)
        F64_TRY(cudaMemcpy2D(Fields_out, (size_t)ny * sizeof(double), F, (size_t)g.ldf * sizeof(double),
                             (size_t)ny * sizeof(double), (size_t)nx_w * nsnap, cudaMemcpyDeviceToHost));
    // Taper weight of slot m: the weight of time sample store_snap*m
    // (calculate_PSDM_RTM.f90:421-427, filters.f90:20-48).
    std::vector<double> wts(nt_taper, 1.0);
    const double pi = 4.0 * atan(1.0);
    if (taper_option != 0) {
        const int i0 = std::max(1, nt_prop2 - N_taper + 1);
        for (int q = 0; q < N_taper; ++q)
            if (i0 + q <= nt_prop2) wts[i0 + q - 1] = 0.5 * (1.0 + cos((pi * double(q)) / double(N_taper)));
        if (N_zeros > 0)
            for (int i = nt_prop2; i < nt_taper; ++i) wts[i] = 0.0;
    }
    // Backward pass on a fresh wavefield, k = 2..nt_taper: slot m images at
    // k = nt_taper + 1 - ks*m.
    for (double* b : {p0, p1, phx0, phx1, chx, phz0, phz1, chz})
        F64_TRY(cudaMemset(b, 0, n * sizeof(double)));
    F64_TRY(cudaMemset(s0, 0, g.nxt * sizeof(double)));
    F64_TRY(cudaMemset(s1, 0, g.nxt * sizeof(double)));
    a.row_slot = d_rrow;
    a.inj_cols = d_rcol;
    a.inj_trace = T;
    a.inj_ld = nt_taper;
    a.ss = (double)store_snap;
    for (int k = 2; k <= nt_taper; ++k) {
        bufs(k - 2);
        a.inj_t = k - 2;
        a.field = nullptr;
        a.field_w = 1.0;
        const int r = nt_taper + 1 - k;
        if (r % store_snap == 0) {
            const int m = r / store_snap;
            if (m >= 1 && m <= nsnap && wts[(size_t)store_snap * m - 1] != 0.0) {
                a.field = F + (size_t)(m - 1) * fstride;
                a.field_w = wts[(size_t)store_snap * m - 1];
            }
        }
        step64_kernel<1><<<grid, 128>>>(a);
    }
    F64_TRY(cudaGetLastError());
    F64_TRY(cudaMemcpy2D(PSDM_w, (size_t)ny * sizeof(double), img, (size_t)g.ldf * sizeof(double),
                         (size_t)ny * sizeof(double), nx_w, cudaMemcpyDeviceToHost));
    F64_TRY(cudaDeviceSynchronize());
    return PSDM_OK;
}
