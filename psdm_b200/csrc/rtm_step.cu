// Fused RTM time-step kernels for sm_100a (plain FP32 engine).
//
// One launch advances the whole padded grid of one shot by one time step and
// does, per cell, everything the reference spreads over ~30 full-grid passes
// (src/solver_ac_forward_ram.f90:344-573, src/solver_ac_backward_ram.f90:329-545):
//   * 2nd-derivative stencils along x and z (space_deriv2x/2y,
//     src/solver_space_derivs_clean.f90:1-69) with the reference's edge rule
//     (stencil centres clamped to [acc, n-1-acc]);
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
// Arithmetic uses explicit round-to-nearest intrinsics in the reference's
// evaluation order (no FMA contraction; the file is also built with
// --fmad=false), so the engine reproduces the FP32 oracle bit for bit.  The
// one division, (p3-p1)*0.5/dt, uses a reciprocal with an exact FMA
// correction that the host proves correctly rounded for the shot's dt.
//
// Work decomposition (one launch, two block roles, see plan_tiles):
//  * interior tiles, 128 rows x 32 columns of the interior band: p staged in
//    shared memory with a 4-row / 3-column halo; each thread owns 4
//    consecutive rows (one float4) of 8 consecutive columns and slides a
//    7-column float4 window through registers (three 16-byte shared loads
//    per 4 cells, float4 global traffic).  The free-surface row and
//    injection rows are handled inline.
//  * boundary tiles, 32 rows x 16 columns over the C-PML strips and the rows
//    outside the interior band: generic per-cell update, 4 cells a thread.
// Rows are offset by `zoff` so that the interior starts on a 16-byte
// boundary.
//
// Memory: p1 is overwritten in place with p3; phi is ping-ponged because its
// strip stencil reads neighbours; chi is updated in place.

#include <cuda_runtime.h>

#include "rtm_internal.h"

namespace psdm {
namespace {

// Interior tiles: 128 rows x 32 columns, each thread 4 rows x 8 columns.
constexpr int QZ = 32;          // float4 rows per interior tile (one warp along z)
constexpr int TZ = 4 * QZ;      // interior tile rows
constexpr int NWARP = 4;        // warps per block
constexpr int XS = 8;           // columns per thread (interior)
constexpr int TX = NWARP * XS;  // interior tile columns
constexpr int HZ = TZ + 8;      // shared rows (16-byte aligned halo of >= 3)
constexpr int HQ = HZ / 4;      // shared float4 rows
constexpr int WX = TX + 6;      // shared columns (halo of 3)
// C-PML / boundary tiles: 32 rows x 16 columns, each thread 1 row x 4 columns.
constexpr int PTZ = 32;
constexpr int PXS = 4;
constexpr int PTX = NWARP * PXS;
constexpr int PHZ = PTZ + 8;
constexpr int PHQ = PHZ / 4;
constexpr int PWX = PTX + 6;
constexpr int NT = 32 * NWARP;  // threads per block

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

// x / dt, correctly rounded (see fast_div_exact).  Inputs below div_lo are
// scaled by 2^64 first (exact), which keeps the result exact as long as the
// quotient is normal (|x| >= div_tiny); zero, subnormal quotients and huge
// inputs take the IEEE division.
__device__ __forceinline__ float div_dt(const StepArgs& a, float x) {
    const float ax = fabsf(x);
    const bool small = ax < a.div_lo;
    const float xs = small ? __fmul_rn(x, 0x1p64f) : x;
    const float q0 = __fmul_rn(xs, a.inv_dt);
    const float e = __fmaf_rn(-q0, a.dt, xs);
    float q = __fmaf_rn(e, a.inv_dt, q0);
    q = small ? __fmul_rn(q, 0x1p-64f) : q;
    if (ax == 0.f) return __fmul_rn(x, a.inv_dt);  // +-0 keeps its sign
    if (!a.fast_div || ax > a.div_hi || ax < a.div_tiny) q = __fdiv_rn(x, a.dt);
    return q;
}

__device__ __forceinline__ float comp(const float4& v, int r) {
    return r == 0 ? v.x : (r == 1 ? v.y : (r == 2 ? v.z : v.w));
}

// Stage rows [sz0, sz0+4*hq) x columns [sx0, sx0+wx) of p in shared memory
// (zero outside the array).  sz0 is a multiple of 4.
__device__ __forceinline__ void load_tile(const StepArgs& a, float* ps, int sz0, int sx0, int hq, int wx, int tid) {
    for (int q = tid; q < wx * hq; q += NT) {
        const int col = q / hq, r4 = q - col * hq;
        const int gx = sx0 + col, gz = sz0 + 4 * r4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gx >= 0 && gx < a.nxt && gz >= 0 && gz < a.ldz)
            v = __ldg(reinterpret_cast<const float4*>(a.p + gx * a.ldz + gz));
        *reinterpret_cast<float4*>(&ps[col * (4 * hq) + 4 * r4]) = v;
    }
}

// Any cell of the grid: C-PML strips and corners, free-surface row,
// injection, interior.  zd = device row (logical z = zd - zoff); the p tile
// has SH rows per column and origin (sz0, sx0).
template <int MODE, int SH>
__device__ __forceinline__ void cell_generic(const StepArgs& a, const float* __restrict__ ps, int sz0, int sx0, int zd,
                                             int x) {
    const int dn = a.dn;
    const int z = zd - a.zoff;
    if (z < 0 || z >= a.nyt || x >= a.nxt) return;
    // With a free surface the rows above it are never updated: p stays zero.
    if (a.fs && z < dn) return;
    const int kz = (z < dn) ? (dn - z) : (z >= dn + a.ny ? z - (dn + a.ny) + 1 : 0);
    const int kx = (x < dn) ? (dn - x) : (x >= dn + a.nx ? x - (dn + a.nx) + 1 : 0);
    const bool fsrow = a.fs && z == dn;
    const int zl = zd - sz0, xl = x - sx0;
    const int cxl = clampi(x, 3, a.nxt - 4) - sx0;
    const int czl = clampi(z, 3, a.nyt - 4) + a.zoff - sz0;
    const float* colc = ps + cxl * SH + zl;  // x-stencil centre
    const float* colz = ps + xl * SH + czl;  // z-stencil centre
#define AX(k) colc[(k) * SH]
#define AZ(k) colz[(k)]
    const float d2x = D2(AX, a.cf2);
    const float d2y = D2(AZ, a.cf2);
    const int g = x * a.ldz + zd;
    const float pc = ps[xl * SH + zl];
    const float pmo = a.pm[g];
    const float c2v = __ldg(a.c2 + g);

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
            const float* ph = a.phix_in + ci * a.ldz + zd;
#define PX(k) __ldg(ph + (k) * a.ldz)
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
            const int cj = clampi(z - sb, 3, dn - 4) + sb + a.zoff;
            const float* ph = a.phiz_in + x * a.ldz + cj;
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
        if (a.row_slot != nullptr) {
            const int rs = __ldg(a.row_slot + zd);
            if (rs >= 0) {
                const int j = __ldg(a.inj_cols + rs * a.nxt + x);
                if (j >= 0) src = __ldg(a.inj_trace + (size_t)j * a.inj_ld + a.inj_t);
            }
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
        const int fi = (x - dn) * a.ldf + (z - dn);
        if (MODE == 0) {
            a.field[fi] = div_dt(a, __fmul_rn(__fsub_rn(out, pmo), 0.5f));
        } else {
            float F = __ldg(a.field + fi);
            if (a.field_w != 1.f) F = __fmul_rn(F, a.field_w);
            float inc = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out, pmo)), F);
            if (a.ss != 1.f) inc = __fmul_rn(inc, a.ss);
            a.image[fi] = __fadd_rn(a.image[fi], inc);
        }
    }
}

// Interior tile (rect type 0): rows [zd0, zd0+h) are interior rows starting on a
// 16-byte boundary, columns [x0, x0+w) interior columns, so no stencil
// centre is clamped and no C-PML term applies.  The free-surface row (the
// first interior row) and injection rows are handled inline.
template <int MODE>
__device__ __forceinline__ void interior_tile(const StepArgs& a, float* ps, int r, int t) {
    const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * TZ, x0 = a.r_x0[r] + tx * TX;
    const int zend = a.r_zd0[r] + a.r_h[r], xend = a.r_x0[r] + a.r_w[r];
    const int sz0 = z0 - 4, sx0 = x0 - 3;
    load_tile(a, ps, sz0, sx0, HQ, WX, tid);
    __syncthreads();

    const int zd = z0 + 4 * lane;  // first device row of this thread's float4
    const int xb = x0 + wy * XS;   // first column of this thread
    if (zd >= zend || xb >= xend) return;
    const int ncol = min(XS, xend - xb);
    const int dn = a.dn;
    const int z = zd - a.zoff;
    const bool fsq = a.fs && z == dn;  // first row of this float4 is the free surface
    int4 rs = make_int4(-1, -1, -1, -1);
    if (a.row_slot != nullptr) rs = __ldg(reinterpret_cast<const int4*>(a.row_slot + zd));
    const bool has_inj = rs.x >= 0 || rs.y >= 0 || rs.z >= 0 || rs.w >= 0;

    const float4* __restrict__ ps4 = reinterpret_cast<const float4*>(ps);
    const int qr = (zd - sz0) >> 2;
    const float* __restrict__ c2p = a.c2;
    float* __restrict__ pmp = a.pm;
    float4 win[7];
#pragma unroll
    for (int k = 0; k < 6; ++k) win[k] = ps4[(xb - 3 + k - sx0) * HQ + qr];
    int g = xb * a.ldz + zd;
    int fi = (xb - dn) * a.ldf + (z - dn);
    const float* c2 = a.cf2;
    float4 pmv = *reinterpret_cast<const float4*>(pmp + g);
    float4 c2v = __ldg(reinterpret_cast<const float4*>(c2p + g));
#pragma unroll
    for (int c = 0; c < XS; ++c) {
        if (c >= ncol) break;
        const int col = xb + c - sx0;
        win[6] = ps4[(col + 3) * HQ + qr];
        const float4 zm = ps4[col * HQ + qr - 1];
        const float4 zp = ps4[col * HQ + qr + 1];
        // prefetch the next column's p1 and c2
        float4 pmn = pmv, c2n = c2v;
        if (c + 1 < ncol) {
            pmn = *reinterpret_cast<const float4*>(pmp + g + a.ldz);
            c2n = __ldg(reinterpret_cast<const float4*>(c2p + g + a.ldz));
        }
        float src[4] = {0.f, 0.f, 0.f, 0.f};
        if (has_inj) {
            const int x = xb + c;
            const int rsv[4] = {rs.x, rs.y, rs.z, rs.w};
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (rsv[r] >= 0) {
                    const int j = __ldg(a.inj_cols + rsv[r] * a.nxt + x);
                    if (j >= 0) src[r] = __ldg(a.inj_trace + (size_t)j * a.inj_ld + a.inj_t);
                }
        }
        const float zv[10] = {zm.y, zm.z, zm.w, win[3].x, win[3].y, win[3].z, win[3].w, zp.x, zp.y, zp.z};
        float o[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
#define WXR(k) comp(win[3 + (k)], r)
#define WZR(k) zv[3 + r + (k)]
            const float d2x = D2(WXR, c2);
            const float d2y = D2(WZR, c2);
#undef WXR
#undef WZR
            const float base = __fadd_rn(-comp(pmv, r), __fmul_rn(2.f, comp(win[3], r)));
            float lap = __fadd_rn(d2x, d2y);
            if (has_inj) lap = __fadd_rn(lap, src[r]);
            o[r] = __fadd_rn(base, __fmul_rn(comp(c2v, r), lap));
        }
        if (fsq) o[0] = 0.f;
        const float4 out = make_float4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<float4*>(pmp + g) = out;
        if (a.field != nullptr) {
            if (MODE == 0) {
                float4 s;
                s.x = div_dt(a, __fmul_rn(__fsub_rn(out.x, pmv.x), 0.5f));
                s.y = div_dt(a, __fmul_rn(__fsub_rn(out.y, pmv.y), 0.5f));
                s.z = div_dt(a, __fmul_rn(__fsub_rn(out.z, pmv.z), 0.5f));
                s.w = div_dt(a, __fmul_rn(__fsub_rn(out.w, pmv.w), 0.5f));
                *reinterpret_cast<float4*>(a.field + fi) = s;
            } else {
                float4 F = __ldg(reinterpret_cast<const float4*>(a.field + fi));
                float4 im = *reinterpret_cast<const float4*>(a.image + fi);
                if (a.field_w != 1.f) {
                    F.x = __fmul_rn(F.x, a.field_w); F.y = __fmul_rn(F.y, a.field_w);
                    F.z = __fmul_rn(F.z, a.field_w); F.w = __fmul_rn(F.w, a.field_w);
                }
                float4 inc;
                inc.x = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out.x, pmv.x)), F.x);
                inc.y = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out.y, pmv.y)), F.y);
                inc.z = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out.z, pmv.z)), F.z);
                inc.w = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out.w, pmv.w)), F.w);
                if (a.ss != 1.f) {
                    inc.x = __fmul_rn(inc.x, a.ss); inc.y = __fmul_rn(inc.y, a.ss);
                    inc.z = __fmul_rn(inc.z, a.ss); inc.w = __fmul_rn(inc.w, a.ss);
                }
                im.x = __fadd_rn(im.x, inc.x); im.y = __fadd_rn(im.y, inc.y);
                im.z = __fadd_rn(im.z, inc.z); im.w = __fadd_rn(im.w, inc.w);
                *reinterpret_cast<float4*>(a.image + fi) = im;
            }
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) win[k] = win[k + 1];
        pmv = pmn;
        c2v = c2n;
        g += a.ldz;
        fi += a.ldf;
    }
}

// C-PML x-strip over the interior band rows (rect type 1): rows are interior
// rows (kz = 0, no row clamping), columns x-PML columns.  Each thread owns 4
// rows (one float4) of 4 columns; the C-PML factor, the clamped stencil
// centre cx and the strip-local phi centre are uniform per column.
template <int MODE>
__device__ __forceinline__ void xband_tile(const StepArgs& a, float* ps, int r, int t) {
    const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * TZ, x0 = a.r_x0[r] + tx * PTX;
    const int zend = a.r_zd0[r] + a.r_h[r], xend = a.r_x0[r] + a.r_w[r];
    const int sz0 = z0 - 4;
    const int sx0 = min(x0, a.nxt - 4) - 3;
    load_tile(a, ps, sz0, sx0, HQ, PWX, tid);
    __syncthreads();
    const int zd = z0 + 4 * lane;
    if (zd >= zend) return;
    const int dn = a.dn;
    const int z = zd - a.zoff;
    const bool fsq = a.fs && z == dn;
    const float4* __restrict__ ps4 = reinterpret_cast<const float4*>(ps);
    const int qr = (zd - sz0) >> 2;
    const float* c1 = a.cf1;
    const float* c2 = a.cf2;
#pragma unroll 1
    for (int c = 0; c < PXS; ++c) {
        const int x = x0 + wy * PXS + c;
        if (x >= xend) break;
        const int kx = (x < dn) ? (dn - x) : (x - (dn + a.nx) + 1);
        const int cx = clampi(x, 3, a.nxt - 4);
        const int sb = (x < dn) ? 0 : dn + a.nx;
        const int ci = clampi(x - sb, 3, dn - 4) + sb;
        const float A = __ldg(a.fA + kx - 1), B = __ldg(a.fB + kx - 1);
        const int g = x * a.ldz + zd;
        float4 P[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) P[k] = ps4[(cx + k - 3 - sx0) * HQ + qr];
        const float4 zc = ps4[(x - sx0) * HQ + qr];
        const float4 zm = ps4[(x - sx0) * HQ + qr - 1];
        const float4 zp = ps4[(x - sx0) * HQ + qr + 1];
        float4 F[7];
#pragma unroll
        for (int k = 0; k < 7; ++k)
            if (k != 3) F[k] = __ldg(reinterpret_cast<const float4*>(a.phix_in + (ci + k - 3) * a.ldz + zd));
        F[3] = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 phc = __ldg(reinterpret_cast<const float4*>(a.phix_in + g));
        const float4 chc = *reinterpret_cast<const float4*>(a.chix + g);
        const float4 pmv = *reinterpret_cast<const float4*>(a.pm + g);
        const float4 c2v = __ldg(reinterpret_cast<const float4*>(a.c2 + g));
        const float zv[10] = {zm.y, zm.z, zm.w, zc.x, zc.y, zc.z, zc.w, zp.x, zp.y, zp.z};
        float o[4], phn[4], chn[4];
#pragma unroll
        for (int rr = 0; rr < 4; ++rr) {
#define PXR(k) comp(P[3 + (k)], rr)
#define FXR(k) comp(F[3 + (k)], rr)
#define ZR(k) zv[3 + rr + (k)]
            const float d2x = D2(PXR, c2);
            const float d1x = D1(PXR, c1);
            const float d2y = D2(ZR, c2);
            const float dph = D1(FXR, c1);
#undef PXR
#undef FXR
#undef ZR
            phn[rr] = __fadd_rn(__fmul_rn(A, comp(phc, rr)), __fmul_rn(B, d1x));
            chn[rr] = __fadd_rn(__fmul_rn(A, comp(chc, rr)), __fmul_rn(B, __fadd_rn(d2x, dph)));
            const float prop = __fadd_rn(dph, chn[rr]);
            float pp = comp(zc, rr), ppm = comp(pmv, rr);
            if (rr == 0 && fsq && !a.disk) { pp = a.side_p[x]; ppm = a.side_pm[x]; }
            const float base = __fadd_rn(-ppm, __fmul_rn(2.f, pp));
            o[rr] = __fadd_rn(base, __fmul_rn(comp(c2v, rr), __fadd_rn(__fadd_rn(d2x, d2y), prop)));
        }
        if (fsq && !a.disk) {  // free-surface row: private history keeps p3, the grid gets 0
            a.side_pm[x] = o[0];
            o[0] = 0.f;
        }
        *reinterpret_cast<float4*>(a.pm + g) = make_float4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<float4*>(a.phix_out + g) = make_float4(phn[0], phn[1], phn[2], phn[3]);
        *reinterpret_cast<float4*>(a.chix + g) = make_float4(chn[0], chn[1], chn[2], chn[3]);
    }
}

// C-PML z-strip over interior columns (rect type 2): kx = 0.  Rows with
// kz > 0 run a specialised update; interior rows of a partial float4 at the
// bottom of the band fall back to the generic cell.
template <int MODE>
__device__ __forceinline__ void zstrip_tile(const StepArgs& a, float* ps, int r, int t) {
    const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * PTZ, x0 = a.r_x0[r] + tx * PTX;
    const int zend = a.r_zd0[r] + a.r_h[r], xend = a.r_x0[r] + a.r_w[r];
    const int nr = a.zoff + a.nyt;
    const int sz0 = (min(z0, nr - 4) - 3) & ~3;
    const int sx0 = x0 - 3;  // interior columns: no clamping along x
    load_tile(a, ps, sz0, sx0, PHQ, PWX, tid);
    __syncthreads();
    const int zd = z0 + lane;
    if (zd >= zend) return;
    const int dn = a.dn;
    const int z = zd - a.zoff;
    if (z < 0 || z >= a.nyt) return;
    const int kz = (z < dn) ? (dn - z) : (z >= dn + a.ny ? z - (dn + a.ny) + 1 : 0);
    if (kz == 0) {
#pragma unroll 1
        for (int c = 0; c < PXS; ++c) {
            const int x = x0 + wy * PXS + c;
            if (x >= xend) break;
            cell_generic<MODE, PHZ>(a, ps, sz0, sx0, zd, x);
        }
        return;
    }
    const float A = __ldg(a.fA + kz - 1), B = __ldg(a.fB + kz - 1);
    const int zl = zd - sz0;
    const int czl = clampi(z, 3, a.nyt - 4) + a.zoff - sz0;
    const int sb = (z < dn) ? 0 : dn + a.ny;
    const int cj = clampi(z - sb, 3, dn - 4) + sb + a.zoff;
    const float* c1 = a.cf1;
    const float* c2 = a.cf2;
#pragma unroll 1
    for (int c = 0; c < PXS; ++c) {
        const int x = x0 + wy * PXS + c;
        if (x >= xend) break;
        const int xl = x - sx0;
        const float* colc = ps + xl * PHZ + zl;
        const float* colz = ps + xl * PHZ + czl;
#define AX(k) colc[(k) * PHZ]
#define AZ(k) colz[(k)]
        const float d2x = D2(AX, c2);
        const float d2y = D2(AZ, c2);
        const float d1 = D1(AZ, c1);
#undef AX
        const int g = x * a.ldz + zd;
        const float* ph = a.phiz_in + x * a.ldz + cj;
#define PZ(k) __ldg(ph + (k))
        const float dph = D1(PZ, c1);
#undef PZ
#undef AZ
        const float phn = __fadd_rn(__fmul_rn(A, __ldg(a.phiz_in + g)), __fmul_rn(B, d1));
        const float chn = __fadd_rn(__fmul_rn(A, a.chiz[g]), __fmul_rn(B, __fadd_rn(d2y, dph)));
        a.phiz_out[g] = phn;
        a.chiz[g] = chn;
        const float prop = __fadd_rn(dph, chn);
        const float base = __fadd_rn(-a.pm[g], __fmul_rn(2.f, colc[0]));
        a.pm[g] = __fadd_rn(base, __fmul_rn(__ldg(a.c2 + g), __fadd_rn(__fadd_rn(d2x, d2y), prop)));
    }
}

// Corner tiles and anything else (rect type 3): generic per-cell update.
template <int MODE>
__device__ __forceinline__ void generic_tile(const StepArgs& a, float* ps, int r, int t) {
    const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * PTZ, x0 = a.r_x0[r] + tx * PTX;
    const int zend = a.r_zd0[r] + a.r_h[r], xend = a.r_x0[r] + a.r_w[r];
    const int nr = a.zoff + a.nyt;
    // Stencil centres are clamped to [3, n-4]: a tile at the far edge may need
    // rows/columns before its own start.
    const int sz0 = (min(z0, nr - 4) - 3) & ~3;
    const int sx0 = min(x0, a.nxt - 4) - 3;
    load_tile(a, ps, sz0, sx0, PHQ, PWX, tid);
    __syncthreads();
    const int zd = z0 + lane;
    if (zd >= zend) return;
#pragma unroll 1
    for (int c = 0; c < PXS; ++c) {
        const int x = x0 + wy * PXS + c;
        if (x >= xend) break;
        cell_generic<MODE, PHZ>(a, ps, sz0, sx0, zd, x);
    }
}

template <int MODE>
__global__ void __launch_bounds__(NT, 5) step_kernel(const StepArgs a) {
    __shared__ __align__(16) float ps[WX * HZ];
    __shared__ int tile_id;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    if (MODE == 0 && a.rec_t >= 0) {
        // Receivers of the previous step: p is that step's p3.
        for (int i = blockIdx.x * NT + tid; i < a.nrec; i += gridDim.x * NT)
            a.rec_out[(size_t)i * a.rec_ld + a.rec_t] = a.p[a.rec_cell[i]];
    }
    // Persistent blocks take tiles in order (heaviest rect types first) from
    // this step's counter; the other counter is cleared for the next step.
    if (blockIdx.x == 0 && tid == 0) a.tile_counter[a.counter_sel ^ 1] = 0;
    const int total = a.r_first[a.nrect];
    for (;;) {
        if (tid == 0) tile_id = atomicAdd(a.tile_counter + a.counter_sel, 1);
        __syncthreads();
        const int b = tile_id;
        if (b >= total) return;
        int r = 0;
        while (r + 1 < a.nrect && b >= a.r_first[r + 1]) ++r;
        const int t = b - a.r_first[r];
        switch (a.r_type[r]) {
            case 0: interior_tile<MODE>(a, ps, r, t); break;
            case 1: xband_tile<MODE>(a, ps, r, t); break;
            case 2: zstrip_tile<MODE>(a, ps, r, t); break;
            default: generic_tile<MODE>(a, ps, r, t); break;
        }
        __syncthreads();  // shared tile and tile_id are reused
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
// Rows outside [zoff, zoff+nyt) are zeroed.
__global__ void pad_c2_kernel(const float* vp, int ny, int nx, int dn, int nyt, int nxt, int ldz, int zoff, float dt,
                              float dd, int ram_padding, float* c2) {
    const int zd = blockIdx.x * blockDim.x + threadIdx.x;
    const int x = blockIdx.y;
    if (zd >= ldz || x >= nxt) return;
    const int z = zd - zoff;
    float v = 0.f;
    const bool strip_row = z < dn || z >= dn + ny;
    if (z >= 0 && z < nyt && !(ram_padding && strip_row && x >= 2 * dn && x < dn + nx)) {
        const int j = clampi(z - dn, 0, ny - 1), i = clampi(x - dn, 0, nx - 1);
        const float c = vp[(size_t)i * ny + j];
        v = __fdiv_rn(__fmul_rn(__fmul_rn(c, c), __fmul_rn(dt, dt)), __fmul_rn(dd, dd));
    }
    c2[(size_t)x * ldz + zd] = v;
}

}  // namespace

void plan_tiles(StepArgs* a) {
    // Rects of the padded grid (device rows):
    //   type 0  interior band  rows [d0, d0+ny4) x interior columns
    //   type 1  x-strip band   rows [d0, d0+ny4) x C-PML columns
    //   type 2  z-strips       rows below the band (and above it without a free
    //                          surface) x interior columns
    //   type 3  corners        the remaining rows x C-PML columns
    // d0 = first interior row (a multiple of 4), ny4 = ny rounded down to 4.
    const int dn = a->dn, nr = a->zoff + a->nyt;
    const int d0 = dn + a->zoff;
    const int ny4 = a->ny & ~3;
    int n = 0;
    a->r_first[0] = 0;
    auto add = [&](int type, int zd0, int x0, int h, int w) {
        if (h <= 0 || w <= 0) return;
        const int tzsz = (type == 0 || type == 1) ? TZ : PTZ;
        const int txsz = (type == 0) ? TX : PTX;
        a->r_type[n] = type;
        a->r_zd0[n] = zd0; a->r_x0[n] = x0; a->r_h[n] = h; a->r_w[n] = w;
        a->r_tz[n] = (h + tzsz - 1) / tzsz;
        a->r_first[n + 1] = a->r_first[n] + a->r_tz[n] * ((w + txsz - 1) / txsz);
        ++n;
    };
    const int xr = dn + a->nx;  // first right-strip column
    add(0, d0, dn, ny4, a->nx);
    add(1, d0, 0, ny4, dn);
    add(1, d0, xr, ny4, a->nxt - xr);
    add(2, d0 + ny4, dn, nr - (d0 + ny4), a->nx);
    add(3, d0 + ny4, 0, nr - (d0 + ny4), dn);
    add(3, d0 + ny4, xr, nr - (d0 + ny4), a->nxt - xr);
    if (!a->fs) {  // with a free surface the rows above it are dead
        add(2, 0, dn, d0, a->nx);
        add(3, 0, 0, d0, dn);
        add(3, 0, xr, d0, a->nxt - xr);
    }
    a->nrect = n;
}

int step_blocks_per_sm() {
    static int nb = 0;
    if (nb == 0) {
        int n0 = 0, n1 = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n0, step_kernel<0>, NT, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n1, step_kernel<1>, NT, 0);
        nb = max(1, min(n0, n1));
    }
    return nb;
}

int launch_step(int mode, const StepArgs& a, void* stream) {
    const dim3 grid(min(a.r_first[a.nrect], a.num_sms * step_blocks_per_sm()));
    const dim3 block(32, NWARP);
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

int launch_pad_c2(const float* vp, int ny, int nx, int dn, int nyt, int nxt, int ldz, int zoff, float dt, float dd,
                  int ram_padding, float* c2, void* stream) {
    const dim3 grid((ldz + 127) / 128, nxt);
    pad_c2_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(vp, ny, nx, dn, nyt, nxt, ldz, zoff, dt, dd, ram_padding,
                                                          c2);
    return (int)cudaGetLastError();
}

}  // namespace psdm
