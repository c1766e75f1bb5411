// Fused RTM time-step kernels for sm_100a (plain FP32 engine).
//
// One launch advances the whole padded grid of one shot by one time step and
// does, per cell, everything the reference spreads over ~30 full-grid passes
// (src/solver_ac_forward_ram.f90:344-573, src/solver_ac_backward_ram.f90:329-545):
//   * 2nd-derivative stencils along x and z (space_deriv2x/2y,
//     src/solver_space_derivs_clean.f90:1-69) from a shared-memory tile of p,
//     with the reference's edge rule (centres clamped to [acc, n-1-acc]);
//   * in PML cells: the 1st-derivative stencils (space_derivx/y, :71-140),
//     the strip-local derivative of phi, and the phi/chi recursions of
//     pml_matrices_x/_y/_xycorner (src/solver_PML_matrices.f90:1-111), with
//     factor index k in strips and max(kx, kz) in corners;
//   * the interior update with source / adjoint-source injection (:443-444);
//   * the free-surface row, including the RAM solvers' strip-private
//     histories of that row (:449-473) or the disk solvers' order
//     (src/solver_ac_forward_disk.f90:506-517);
//   * forward: the snapshot (p3-p1)*0.5/dt (:476-488) and the deferred
//     receiver gather (:567-571); backward: the imaging condition
//     kernel += 0.5*(p3-p1)*Fields*store_snap (backward_ram.f90:455-470).
//
// Arithmetic is written with explicit round-to-nearest intrinsics in the
// reference's evaluation order (no FMA contraction; this file is also built
// with --fmad=false), so the engine reproduces the FP32 oracle bit for bit.
//
// Memory: p is read through a 40x38 shared tile (z-halo rounded to 16-byte
// boundaries); p1 is overwritten in place with p3; phi is ping-ponged
// because its strip stencil reads neighbours; chi is updated in place.

#include <cuda_runtime.h>

#include "rtm_internal.h"

namespace psdm {
namespace {

constexpr int TZ = 32;            // tile rows (one warp along z, contiguous)
constexpr int TX = 32;            // tile columns
constexpr int BY = 8;             // warps per block
constexpr int XPT = TX / BY;      // columns per thread
constexpr int HZ = TZ + 8;        // shared rows: 16-byte aligned halo of >= 3
constexpr int WX = TX + 6;        // shared columns: halo of 3
constexpr int NT = 32 * BY;       // threads per block

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// sum_{k=0..3} c[k] * (a(+k) + a(-k)), accumulated in the reference's order.
#define D2(AT, c)                                                                              \
    __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(__fadd_rn(AT(0), AT(0)), (c)[0]),                   \
                                  __fmul_rn(__fadd_rn(AT(1), AT(-1)), (c)[1])),                 \
                        __fmul_rn(__fadd_rn(AT(2), AT(-2)), (c)[2])),                           \
              __fmul_rn(__fadd_rn(AT(3), AT(-3)), (c)[3]))
// sum_{k=1..3} c[k] * (a(+k) - a(-k)); the k = 0 term of the reference is +0.
#define D1(AT, c)                                                                              \
    __fadd_rn(__fadd_rn(__fmul_rn(__fsub_rn(AT(1), AT(-1)), (c)[1]),                            \
                        __fmul_rn(__fsub_rn(AT(2), AT(-2)), (c)[2])),                           \
              __fmul_rn(__fsub_rn(AT(3), AT(-3)), (c)[3]))

template <int MODE>
__global__ void __launch_bounds__(NT) step_kernel(const StepArgs a) {
    __shared__ __align__(16) float ps[WX * HZ];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int z0 = blockIdx.x * TZ, x0 = blockIdx.y * TX;
    // Tile origin: centres are clamped to [3, n-4], so the last tile may need
    // columns/rows left of its own start; z origin rounded down to 4 floats.
    const int sz0 = (min(z0, a.nyt - 4) - 3) & ~3;
    const int sx0 = min(x0, a.nxt - 4) - 3;

    if (MODE == 0 && a.rec_t >= 0) {
        // Receivers of the previous step: p is that step's p3.
        const int i = (blockIdx.y * gridDim.x + blockIdx.x) * NT + tid;
        if (i < a.nrec) a.rec_out[(size_t)i * a.rec_ld + a.rec_t] = a.p[a.rec_cell[i]];
    }

    for (int q = tid; q < WX * (HZ / 4); q += NT) {
        const int col = q / (HZ / 4), r4 = q - col * (HZ / 4);
        const int gx = sx0 + col, gz = sz0 + 4 * r4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gx >= 0 && gx < a.nxt && gz >= 0 && gz < a.ldz)
            v = __ldg(reinterpret_cast<const float4*>(a.p + (size_t)gx * a.ldz + gz));
        *reinterpret_cast<float4*>(&ps[col * HZ + 4 * r4]) = v;
    }
    __syncthreads();

    const int z = z0 + tx;
    if (z >= a.nyt) return;
    // With a free surface the rows above it are never updated: p stays zero.
    if (a.fs && z < a.dn) return;

    const int dn = a.dn;
    const int zl = z - sz0;
    const int czl = clampi(z, 3, a.nyt - 4) - sz0;
    const int kz = (z < dn) ? (dn - z) : (z >= dn + a.ny ? z - (dn + a.ny) + 1 : 0);
    const bool fsrow = a.fs && z == dn;
    const int rslot = (a.row_slot != nullptr && kz == 0) ? a.row_slot[z] : -1;

#pragma unroll
    for (int r = 0; r < XPT; ++r) {
        const int x = x0 + ty * XPT + r;
        if (x >= a.nxt) break;
        const size_t g = (size_t)x * a.ldz + z;
        const int xl = x - sx0;
        const int cxl = clampi(x, 3, a.nxt - 4) - sx0;
        const float* colc = ps + cxl * HZ + zl;  // x-stencil centre
        const float* colz = ps + xl * HZ + czl;  // z-stencil centre
#define AX(k) colc[(k) * HZ]
#define AZ(k) colz[(k)]
        const float d2x = D2(AX, a.cf2);
        const float d2y = D2(AZ, a.cf2);
        const float pc = ps[xl * HZ + zl];
        const float pmo = a.pm[g];
        const float c2v = a.c2[g];
        const int kx = (x < dn) ? (dn - x) : (x >= dn + a.nx ? x - (dn + a.nx) + 1 : 0);

        float pp = pc, ppm = pmo;
        if (fsrow && kx > 0 && !a.disk) { pp = a.side_p[x]; ppm = a.side_pm[x]; }
        const float base = __fadd_rn(-ppm, __fmul_rn(2.f, pp));

        float main_term, propz = 0.f;
        if (kx > 0 || kz > 0) {
            const int f = (kx > 0 && kz > 0) ? max(kx, kz) : (kx > 0 ? kx : kz);
            const float A = __ldg(a.fA + f - 1), B = __ldg(a.fB + f - 1);
            float propx = 0.f;
            if (kx > 0) {
                const float d1 = D1(AX, a.cf1);
                const int sb = (x < dn) ? 0 : dn + a.nx;
                const int ci = clampi(x - sb, 3, dn - 4) + sb;
                const float* ph = a.phix_in + (size_t)ci * a.ldz + z;
#define PX(k) __ldg(ph + (ptrdiff_t)(k) * a.ldz)
                const float dph = D1(PX, a.cf1);
#undef PX
                const float phn = __fadd_rn(__fmul_rn(A, a.phix_in[g]), __fmul_rn(B, d1));
                const float chn = __fadd_rn(__fmul_rn(A, a.chix[g]), __fmul_rn(B, __fadd_rn(d2x, dph)));
                a.phix_out[g] = phn;
                a.chix[g] = chn;
                propx = __fadd_rn(dph, chn);
            }
            if (kz > 0) {
                const float d1 = D1(AZ, a.cf1);
                const int sb = (z < dn) ? 0 : dn + a.ny;
                const int cj = clampi(z - sb, 3, dn - 4) + sb;
                const float* ph = a.phiz_in + (size_t)x * a.ldz + cj;
#define PZ(k) __ldg(ph + (k))
                const float dph = D1(PZ, a.cf1);
#undef PZ
                const float phn = __fadd_rn(__fmul_rn(A, a.phiz_in[g]), __fmul_rn(B, d1));
                const float chn = __fadd_rn(__fmul_rn(A, a.chiz[g]), __fmul_rn(B, __fadd_rn(d2y, dph)));
                a.phiz_out[g] = phn;
                a.chiz[g] = chn;
                propz = __fadd_rn(dph, chn);
            }
            main_term = (kx > 0) ? propx : propz;
        } else {
            float src = 0.f;
            if (rslot >= 0) {
                const int j = a.inj_cols[(size_t)rslot * a.nxt + x];
                if (j >= 0) src = a.inj_trace[(size_t)j * a.inj_ld + a.inj_t];
            }
            main_term = src;
        }
#undef AX
#undef AZ
        float p3 = __fadd_rn(base, __fmul_rn(c2v, __fadd_rn(__fadd_rn(d2x, d2y), main_term)));
        if (kx > 0 && kz > 0) p3 = __fadd_rn(p3, __fmul_rn(c2v, propz));

        float out = p3;
        if (fsrow) {
            if (kx > 0) {
                if (!a.disk) { a.side_pm[x] = p3; out = 0.f; }
            } else {
                out = 0.f;
            }
        }
        a.pm[g] = out;

        if (kx == 0 && kz == 0 && a.field != nullptr) {
            const size_t fi = (size_t)(x - dn) * a.ny + (z - dn);
            if (MODE == 0) {
                a.field[fi] = __fdiv_rn(__fmul_rn(__fsub_rn(out, pmo), 0.5f), a.dt);
            } else {
                const float F = __fmul_rn(__ldg(a.field + fi), a.field_w);
                const float inc = __fmul_rn(__fmul_rn(__fmul_rn(0.5f, __fsub_rn(out, pmo)), F), a.ss);
                a.image[fi] = __fadd_rn(a.image[fi], inc);
            }
        }
    }
}

__global__ void rec_final_kernel(const int* rec_cell, const float* p, float* rec_out, int nrec, int rec_ld, int nt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrec) return;
    const float v = p[rec_cell[i]];
    rec_out[(size_t)i * rec_ld + (nt - 2)] = v;
    rec_out[(size_t)i * rec_ld + (nt - 1)] = v;
}

// Model padding and c2 = c**2*dt**2/dmodel**2 (src/solver_ac_forward_ram.f90:282-319).
// c = ctmp(clamp(z-dn), clamp(x-dn)), except in the RAM solvers' top and
// bottom strips: their loops `do j=1,dnx` (:288-302) fill only the first dn
// interior columns there, so c stays 0 for x in [2dn, dn+nx).  The disk
// solvers fill the full width (solver_ac_forward_disk.f90:294-312).
// Padding rows z >= nyt are zeroed.
__global__ void pad_c2_kernel(const float* vp, int ny, int nx, int dn, int nyt, int nxt, int ldz, float dt,
                              float dd, int ram_padding, float* c2) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    if (z >= ldz || x >= nxt) return;
    float v = 0.f;
    const bool strip_row = z < dn || z >= dn + ny;
    if (z < nyt && !(ram_padding && strip_row && x >= 2 * dn && x < dn + nx)) {
        const int j = clampi(z - dn, 0, ny - 1), i = clampi(x - dn, 0, nx - 1);
        const float c = vp[(size_t)i * ny + j];
        v = __fdiv_rn(__fmul_rn(__fmul_rn(c, c), __fmul_rn(dt, dt)), __fmul_rn(dd, dd));
    }
    c2[(size_t)x * ldz + z] = v;
}

}  // namespace

int launch_step(int mode, const StepArgs& a, void* stream) {
    const dim3 grid((a.nyt + TZ - 1) / TZ, (a.nxt + TX - 1) / TX);
    const dim3 block(32, BY);
    if (mode == 0)
        step_kernel<0><<<grid, block, 0, (cudaStream_t)stream>>>(a);
    else
        step_kernel<1><<<grid, block, 0, (cudaStream_t)stream>>>(a);
    return (int)cudaGetLastError();
}

int launch_rec_final(const int* rec_cell, const float* p, float* rec_out, int nrec, int rec_ld, int nt, void* stream) {
    if (nrec <= 0 || nt < 2) return 0;
    rec_final_kernel<<<(nrec + 255) / 256, 256, 0, (cudaStream_t)stream>>>(rec_cell, p, rec_out, nrec, rec_ld, nt);
    return (int)cudaGetLastError();
}

int launch_pad_c2(const float* vp, int ny, int nx, int dn, int nyt, int nxt, int ldz, float dt, float dd,
                  int ram_padding, float* c2, void* stream) {
    const dim3 grid((ldz + 127) / 128, nxt);
    pad_c2_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(vp, ny, nx, dn, nyt, nxt, ldz, dt, dd, ram_padding, c2);
    return (int)cudaGetLastError();
}

}  // namespace psdm
