// Resident pass kernel for sm_100a: one cooperative launch per pass of one
// shot, with the wavefield kept on chip between time steps.
//
// The padded grid is cut into rectangular regions, one per block and about
// one per multiprocessor.  A block holds its region's levels n and n-1 (with
// a 3-column / 4-row ring of level n) in shared memory for the whole pass:
// a time step reads p and p1 from shared memory, computes level n+1 with
// the one-step kernels' arithmetic (src/solver_ac_forward_ram.f90:344-573,
// src/solver_ac_backward_ram.f90:329-545, in the reference's evaluation
// order), writes it over level n-1 in shared memory and to the global
// wavefield buffer of the step (as a one-step launch does), and publishes
// its step counter.  Before the next step it waits until every region within
// reach has published, and reloads only the ring of its window from global
// memory.  Compared with one launch per step, the grid's interior is not
// re-read from L2 every step, no launch gap separates the steps and a slow
// region delays only its neighbours.
//
// Per step a region's work is a list of warp items (plan_resident):
//   * interior float4s (four rows of one lane) swept over up to 10 columns
//     with a register window, p1 and p from shared memory, c2 from L2, the
//     snapshot or the imaging update fused;
//   * C-PML x-strip float4s and z-strip float4s (interior columns), phi
//     and chi in global memory, the next column's loads in flight;
//   * generic cells (cell_generic's arithmetic, a lane per cell and the
//     next cell's loads in flight): strip edges, corners, the free-surface
//     row, injection rows.
// The global buffers hold exactly what one launch per step leaves there, so
// the receiver gather of the last steps, the pass that follows and every
// other form see the same state.
//
// Every wait is bounded (about 1 s, or until another block gives up) and
// reports through the engine's error word.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "rtm_device.cuh"
#include "rtm_internal.h"

namespace psdm {
namespace {

constexpr int RSH = kResPitch;      // shared rows per column
constexpr int kFastColsMax = 10;    // most columns of an interior float4 item
constexpr int RHQ = RSH / 4;        // shared float4 rows per column
static_assert(RSH % 4 == 0, "float4 rows");

// Fill window positions of a level buffer from the global level `src`:
// all of it (ring_only = false) or only its ring (3 columns left and right,
// one float4 row above and below the region).  Positions outside the
// allocation read zero.
__device__ __forceinline__ void fill_window(float* B, const float* __restrict__ src, const StepArgs& a, int sz0,
                                            int sx0, int nq2, int sw, bool ring_only, int tid) {
    const int n = ring_only ? 6 * nq2 + 2 * (sw - 6) : sw * nq2;
    for (int i = tid; i < n; i += kResThreads) {
        int col, r4;
        if (!ring_only) {
            col = i / nq2;
            r4 = i - col * nq2;
        } else if (i < 6 * nq2) {
            const int c = i / nq2;
            r4 = i - c * nq2;
            col = c < 3 ? c : sw - 6 + c;
        } else {
            const int j = i - 6 * nq2;
            const int half = sw - 6;
            col = 3 + (j < half ? j : j - half);
            r4 = j < half ? 0 : nq2 - 1;
        }
        const int gx = sx0 + col, gz = sz0 + 4 * r4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gx >= 0 && gx < a.nxt && gz >= 0 && gz + 4 <= a.ldz)
            v = *reinterpret_cast<const float4*>(src + (size_t)gx * a.ldz + gz);
        *reinterpret_cast<float4*>(B + col * RSH + 4 * r4) = v;
    }
}

// Interior float4 of rows zd..zd+3 over columns x..x+ncol-1 (ncol <= 10):
// shared float4 row qr, shared column cl of x.  Level n from ps4, level n-1
// from and level n+1 to pp4 and the global buffer a.pm.
template <int MODE>
__device__ __forceinline__ void res_fast(const StepArgs& a, const SubStep& sub, const float4* __restrict__ ps4,
                                         float4* pp4, int qr, int cl, int g, int fi, int ncol,
                                         const float2 (&cc)[4]) {
    float4 win[7];
#pragma unroll
    for (int k = 0; k < 6; ++k) win[k] = ps4[(cl - 3 + k) * RHQ + qr];
    float4 c2N = __ldg(reinterpret_cast<const float4*>(a.c2 + g));
    const bool snap = MODE == 0 && sub.field != nullptr;
    const bool img = MODE == 1 && sub.field != nullptr;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint2 z2 = make_uint2(0u, 0u);
    float4 Fn = z4, In = z4;
    if (img) {
        Fn = __ldg(reinterpret_cast<const float4*>(sub.field + fi));
        In = *reinterpret_cast<const float4*>(a.image + fi);
    }
    float amax_t = 0.f;
#pragma unroll
    for (int c = 0; c < kFastColsMax; ++c) {
        if (c >= ncol) break;
        const int col = cl + c;
        win[6] = ps4[(col + 3) * RHQ + qr];
        const float4 zm = ps4[col * RHQ + qr - 1];
        const float4 zp = ps4[col * RHQ + qr + 1];
        const float4 pmv = pp4[col * RHQ + qr];
        const float4 c2v = c2N;
        if (c + 1 < ncol) c2N = __ldg(reinterpret_cast<const float4*>(a.c2 + g + a.ldz));
        const float4 Fc = Fn, Ic = In;
        if (img && c + 1 < ncol) {
            Fn = __ldg(reinterpret_cast<const float4*>(sub.field + fi + a.ldf));
            In = *reinterpret_cast<const float4*>(a.image + fi + a.ldf);
        }
        const float4 out = clean_update(win, zm, zp, pmv, c2v, cc);
        pp4[col * RHQ + qr] = out;
        *reinterpret_cast<float4*>(a.pm + g) = out;
        if (snap || img) emit4<MODE>(a, sub, fi, out, pmv, Fc, Ic, z4, z2, 1.f, amax_t);
#pragma unroll
        for (int k = 0; k < 6; ++k) win[k] = win[k + 1];
        g += a.ldz;
        fi += a.ldf;
    }
}

// The generic cell update (cell_generic's arithmetic, in the same order)
// split into a phase that issues every global load of the cell and a phase
// that computes and stores, so that a lane loads its next cell while it
// computes the current one.  p at level n and n-1 come from the shared level
// buffers (pitch RSH, origin sz0 / sx0).
struct GenIn {
    int x, zd, kx, kz;  // kx < 0: nothing to update
    float pmo, c2v, A, B;
    float phx[7], chx;  // phx[3]: phi_x at the cell, the others its strip stencil
    float phz[7], chz;
    float sp, spm;      // free-surface histories (x-strip cells of the free-surface row)
    float src;          // injection
    float F, I;         // backward: snapshot and image of an interior cell
};

template <int MODE>
__device__ __forceinline__ void res_gen_load(const StepArgs& a, const float* Pp, int sz0, int sx0, int zd, int x,
                                             GenIn& c) {
    const int dn = a.dn;
    const int z = zd - a.zoff;
    c.x = x;
    c.zd = zd;
    c.kx = -1;
    if (z < 0 || z >= a.nyt || x >= a.nxt || (a.fs && z < dn)) return;
    const int kz = (z < dn) ? (dn - z) : (z >= dn + a.ny ? z - (dn + a.ny) + 1 : 0);
    const int kx = (x < dn) ? (dn - x) : (x >= dn + a.nx ? x - (dn + a.nx) + 1 : 0);
    c.kx = kx;
    c.kz = kz;
    const int g = x * a.ldz + zd;
    c.pmo = Pp[(x - sx0) * RSH + (zd - sz0)];
    c.c2v = __ldg(a.c2 + g);
    c.src = 0.f;
    if (kx > 0 || kz > 0) {
        const int f = (kx > 0 && kz > 0) ? max(kx, kz) : (kx > 0 ? kx : kz);
        c.A = __ldg(a.fA + f - 1);
        c.B = __ldg(a.fB + f - 1);
        if (kx > 0) {
            const int sb = (x < dn) ? 0 : dn + a.nx;
            const int ci = clampi(x - sb, 3, dn - 4) + sb;
            const float* ph = a.phix_in + ci * a.ldz + zd;
#pragma unroll
            for (int k = 0; k < 7; ++k)
                if (k != 3) c.phx[k] = ph[(k - 3) * a.ldz];
            c.phx[3] = a.phix_in[g];
            c.chx = a.chix[g];
        }
        if (kz > 0) {
            const int sb = (z < dn) ? 0 : dn + a.ny;
            const int cj = clampi(z - sb, 3, dn - 4) + sb + a.zoff;
            const float* ph = a.phiz_in + x * a.ldz + cj;
#pragma unroll
            for (int k = 0; k < 7; ++k)
                if (k != 3) c.phz[k] = ph[k - 3];
            c.phz[3] = a.phiz_in[g];
            c.chz = a.chiz[g];
        }
    } else if (a.row_slot != nullptr) {
        const int rs = __ldg(a.row_slot + zd);
        if (rs >= 0) {
            const int j = __ldg(a.inj_cols + rs * a.nxt + x);
            if (j >= 0) c.src = __ldg(a.inj_trace + (size_t)j * a.inj_ld + a.inj_t);
        }
    }
    if (a.fs && z == dn && kx > 0 && !a.disk) {
        c.sp = a.side_p[x];
        c.spm = a.side_pm[x];
    }
    if (MODE == 1 && kx == 0 && kz == 0 && a.field != nullptr) {
        const int fi = (x - dn) * a.ldf + (z - dn);
        c.F = __ldg(a.field + fi);
        c.I = a.image[fi];
    }
}

template <int MODE>
__device__ __forceinline__ void res_gen_store(const StepArgs& a, const float* __restrict__ Pc, float* Pp, int sz0,
                                              int sx0, const GenIn& c) {
    if (c.kx < 0) return;
    const int dn = a.dn, x = c.x, zd = c.zd, kx = c.kx, kz = c.kz;
    const int z = zd - a.zoff;
    const bool fsrow = a.fs && z == dn;
    const int zl = zd - sz0, xl = x - sx0;
    const int cxl = clampi(x, 3, a.nxt - 4) - sx0;
    const int czl = clampi(z, 3, a.nyt - 4) + a.zoff - sz0;
    const float* colc = Pc + cxl * RSH + zl;  // x-stencil centre
    const float* colz = Pc + xl * RSH + czl;  // z-stencil centre
#define AX(k) colc[(k) * RSH]
#define AZ(k) colz[(k)]
    const float d2x = D2(AX, a.cf2);
    const float d2y = D2(AZ, a.cf2);
    const int g = x * a.ldz + zd;
    const float pc = Pc[xl * RSH + zl];
    float pp = pc, ppm = c.pmo;
    if (fsrow && kx > 0 && !a.disk) { pp = c.sp; ppm = c.spm; }
    const float base = __fadd_rn(-ppm, __fmul_rn(2.f, pp));
    float main_term, propz = 0.f;
    if (kx > 0 || kz > 0) {
        float propx = 0.f;
        if (kx > 0) {
            const float d1 = D1(AX, a.cf1);
#define PX(k) c.phx[3 + (k)]
            const float dph = D1(PX, a.cf1);
#undef PX
            const float phn = __fadd_rn(__fmul_rn(c.A, c.phx[3]), __fmul_rn(c.B, d1));
            const float chn = __fadd_rn(__fmul_rn(c.A, c.chx), __fmul_rn(c.B, __fadd_rn(d2x, dph)));
            a.phix_out[g] = phn;
            a.chix[g] = chn;
            propx = __fadd_rn(dph, chn);
        }
        if (kz > 0) {
            const float d1 = D1(AZ, a.cf1);
#define PZ(k) c.phz[3 + (k)]
            const float dph = D1(PZ, a.cf1);
#undef PZ
            const float phn = __fadd_rn(__fmul_rn(c.A, c.phz[3]), __fmul_rn(c.B, d1));
            const float chn = __fadd_rn(__fmul_rn(c.A, c.chz), __fmul_rn(c.B, __fadd_rn(d2y, dph)));
            a.phiz_out[g] = phn;
            a.chiz[g] = chn;
            propz = __fadd_rn(dph, chn);
        }
        main_term = (kx > 0) ? propx : propz;
    } else {
        main_term = c.src;
    }
#undef AX
#undef AZ
    float p3 = __fadd_rn(base, __fmul_rn(c.c2v, __fadd_rn(__fadd_rn(d2x, d2y), main_term)));
    if (kx > 0 && kz > 0) p3 = __fadd_rn(p3, __fmul_rn(c.c2v, propz));
    float out = p3;
    if (fsrow) {
        if (kx > 0) {
            if (!a.disk) { a.side_pm[x] = p3; out = 0.f; }
        } else {
            out = 0.f;
        }
    }
    a.pm[g] = out;
    Pp[xl * RSH + zl] = out;
    if (kx == 0 && kz == 0 && a.field != nullptr) {
        const int fi = (x - dn) * a.ldf + (z - dn);
        if (MODE == 0) {
            a.field[fi] = div_dt(a, __fmul_rn(__fsub_rn(out, c.pmo), 0.5f));
        } else {
            float F = c.F;
            if (a.field_w != 1.f) F = __fmul_rn(F, a.field_w);
            float inc = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out, c.pmo)), F);
            if (a.ss != 1.f) inc = __fmul_rn(inc, a.ss);
            a.image[fi] = __fadd_rn(c.I, inc);
        }
    }
}

// A generic item: lane l updates row r0 + l % nr, columns [c0 + span*k/ng,
// c0 + span*(k+1)/ng) with k = l / nr, one column at a time with the next
// column's loads in flight.
template <int MODE>
__device__ __noinline__ void res_gen_item(const StepArgs& a, const float* Pc, float* Pp, int sz0, int sx0,
                                             int zd, int xa, int xb) {
    if (xa >= xb) return;
    GenIn cur, nxt;
    res_gen_load<MODE>(a, Pp, sz0, sx0, zd, xa, cur);
#pragma unroll 1
    for (int x = xa; x < xb; ++x) {
        if (x + 1 < xb) res_gen_load<MODE>(a, Pp, sz0, sx0, zd, x + 1, nxt);
        res_gen_store<MODE>(a, Pc, Pp, sz0, sx0, cur);
        cur = nxt;
    }
}

// A z-strip item's lane: the float4 of rows zd..zd+3 (all in one C-PML
// z-strip, kx = 0, no stencil centre clamped: the rows are at least 3 rows
// from the strip's edges and from the grid's edges) over columns
// x..x+ncol-1.  The update of each row is cell_generic's for kz > 0, kx = 0
// (src/solver_PML_matrices.f90:40-75 with factor kz), in its order; phi_z,
// chi_z and c2 of the next column are loaded while the current one updates.
__device__ __noinline__ void res_zpml_item(const StepArgs& a, const float4* ps4, float4* pp4, int sz0, int sx0,
                                           int zd, int x, int ncol) {
    const int dn = a.dn;
    const int z = zd - a.zoff;
    const int qr = (zd - sz0) >> 2;
    float A[4], B[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int zr = z + r;
        const int kz = zr < dn ? dn - zr : zr - (dn + a.ny) + 1;
        A[r] = __ldg(a.fA + kz - 1);
        B[r] = __ldg(a.fB + kz - 1);
    }
    const float* c1 = a.cf1;
    const float* cf = a.cf2;
    int g = x * a.ldz + zd;
    auto ld4 = [](const float* p) { return *reinterpret_cast<const float4*>(p); };
    float4 fm = ld4(a.phiz_in + g - 4), fc = ld4(a.phiz_in + g), fp = ld4(a.phiz_in + g + 4);
    float4 ch = ld4(a.chiz + g), c2v = __ldg(reinterpret_cast<const float4*>(a.c2 + g));
#pragma unroll 1
    for (int c = 0; c < ncol; ++c) {
        float4 nfm = fm, nfc = fc, nfp = fp, nch = ch, nc2 = c2v;
        if (c + 1 < ncol) {
            const int gn = g + a.ldz;
            nfm = ld4(a.phiz_in + gn - 4);
            nfc = ld4(a.phiz_in + gn);
            nfp = ld4(a.phiz_in + gn + 4);
            nch = ld4(a.chiz + gn);
            nc2 = __ldg(reinterpret_cast<const float4*>(a.c2 + gn));
        }
        const int cl = x + c - sx0;
        float4 P[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) P[k] = ps4[(cl + k - 3) * RHQ + qr];
        const float4 zm = ps4[cl * RHQ + qr - 1], zp = ps4[cl * RHQ + qr + 1];
        const float4 pmv = pp4[cl * RHQ + qr];
        const float zv[10] = {zm.y, zm.z, zm.w, P[3].x, P[3].y, P[3].z, P[3].w, zp.x, zp.y, zp.z};
        const float fv[12] = {fm.x, fm.y, fm.z, fm.w, fc.x, fc.y, fc.z, fc.w, fp.x, fp.y, fp.z, fp.w};
        float o[4], phn[4], chn[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
#define PXR(k) comp(P[3 + (k)], r)
#define ZR(k) zv[3 + r + (k)]
#define FR(k) fv[4 + r + (k)]
            const float d2x = D2(PXR, cf);
            const float d2y = D2(ZR, cf);
            const float d1 = D1(ZR, c1);
            const float dph = D1(FR, c1);
#undef PXR
#undef ZR
#undef FR
            phn[r] = __fadd_rn(__fmul_rn(A[r], comp(fc, r)), __fmul_rn(B[r], d1));
            chn[r] = __fadd_rn(__fmul_rn(A[r], comp(ch, r)), __fmul_rn(B[r], __fadd_rn(d2y, dph)));
            const float prop = __fadd_rn(dph, chn[r]);
            const float base = __fadd_rn(-comp(pmv, r), __fmul_rn(2.f, comp(P[3], r)));
            o[r] = __fadd_rn(base, __fmul_rn(comp(c2v, r), __fadd_rn(__fadd_rn(d2x, d2y), prop)));
        }
        const float4 out = make_float4(o[0], o[1], o[2], o[3]);
        pp4[cl * RHQ + qr] = out;
        *reinterpret_cast<float4*>(a.pm + g) = out;
        *reinterpret_cast<float4*>(a.phiz_out + g) = make_float4(phn[0], phn[1], phn[2], phn[3]);
        *reinterpret_cast<float4*>(a.chiz + g) = make_float4(chn[0], chn[1], chn[2], chn[3]);
        fm = nfm;
        fc = nfc;
        fp = nfp;
        ch = nch;
        c2v = nc2;
        g += a.ldz;
    }
}

// An x-strip item's lane: the float4 of rows zd..zd+3 (interior band rows,
// x in a C-PML x-strip) over columns x0..x0+ncol-1, the next column's global
// loads in flight while the current column updates.
__device__ __noinline__ void res_xpml_item(const StepArgs& a, const float4* ps4, float4* pp4, int sx0, int qr, int zd,
                                           bool fsq, int x0, int ncol) {
    XbandIn cur, nxt;
    xband_load(a, zd, x0, false, cur);
#pragma unroll 1
    for (int c = 0; c < ncol; ++c) {
        if (c + 1 < ncol) xband_load(a, zd, x0 + c + 1, false, nxt);
        xband_compute<RHQ, true>(a, ps4, pp4, sx0, qr, zd, fsq, x0 + c, cur);
        cur = nxt;
    }
}

// All steps of one pass (MODE 0 forward, 1 backward with imaging).  Block b
// owns region b; all blocks are resident at once (cooperative launch).
template <int MODE>
__global__ void __launch_bounds__(kResThreads, 1) res_kernel(const ResParams rp) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(16) StepArgs sb[2];
    __shared__ __align__(16) PassVar sv[2];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const ResRegion R = rp.reg[blockIdx.x];
    constexpr int kWords = (int)(sizeof(StepArgs) / sizeof(long long));
    constexpr int kVar16 = (int)(sizeof(PassVar) / 16);
    for (int w = tid; w < 2 * kWords; w += kResThreads)
        reinterpret_cast<long long*>(sb)[w] = reinterpret_cast<const long long*>(rp.base)[w];
    if (tid == 0 && rp.nsteps > 0) {
        for (int q = 0; q < kVar16; ++q)
            cp_async16(reinterpret_cast<char*>(&sv[0]) + 16 * q, reinterpret_cast<const char*>(rp.var) + 16 * q);
        cp_async_commit();
    }
    __syncthreads();
    float* B[2] = {sm, sm + RSH * rp.sw};
    const int sw = R.w + 6, nq2 = R.nrows / 4 + 2;
    const int sz0 = R.zr0 - 4, sx0 = R.x0 - 3;
    fill_window(B[0], sb[0].p, sb[0], sz0, sx0, nq2, sw, false, tid);   // level 0
    fill_window(B[1], sb[0].pm, sb[0], sz0, sx0, nq2, sw, false, tid);  // level -1
    const int it0 = rp.warp_first[blockIdx.x * kResWarps + warp];
    const int it1 = rp.warp_first[blockIdx.x * kResWarps + warp + 1];
    for (int s = 0; s < rp.nsteps; ++s) {
        const int par = s & 1;
        if (tid == 0) {
            cp_async_wait_all();  // values of step s
            const PassVar& v = sv[par];
            StepArgs& t = sb[par];
            t.field = v.field;
            t.field16 = v.field16;
            t.field_iscale = v.field_iscale;
            t.field_w = v.field_w;
            t.inj_t = v.inj_t;
            t.rec_t = v.rec_t;
            if (s + 1 < rp.nsteps) {
                const char* src = reinterpret_cast<const char*>(rp.var + s + 1);
                for (int q = 0; q < kVar16; ++q)
                    cp_async16(reinterpret_cast<char*>(&sv[par ^ 1]) + 16 * q, src + 16 * q);
                cp_async_commit();
            }
        }
        bool ok = true;
        if (s > 0 && tid < R.nnbr) ok = wait_flag(rp.flags + rp.nbr[R.nbr0 + tid], s, rp.abort);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(rp.abort, 1);
                atomicCAS(rp.err, 0, 3);
                cp_async_wait_all();
            }
            return;
        }
        const StepArgs& a = sb[par];
        float* Pc = B[par];
        float* Pp = B[par ^ 1];
        if (s > 0) fill_window(Pc, a.p, a, sz0, sx0, nq2, sw, true, tid);  // the neighbours' ring of level s
        if (MODE == 0 && a.rec_t >= 0)  // own cells of level s, written by this block in the previous step
            for (int j = tid; j < R.nrec; j += kResThreads) {
                const int r = rp.rec[R.rec0 + j];
                a.rec_out[(size_t)r * a.rec_ld + a.rec_t] = a.p[a.rec_cell[r]];
            }
        __syncthreads();
        SubStep sub{};
        sub.field = a.field;
        sub.field_w = a.field_w;
        float2 cc[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) cc[k] = make_float2(a.cf2[k], a.cf2[k]);
        const float4* ps4 = reinterpret_cast<const float4*>(Pc);
        float4* pp4 = reinterpret_cast<float4*>(Pp);
        for (int it = it0; it < it1; ++it) {
            const int w0 = rp.items[2 * it], w1 = rp.items[2 * it + 1];
            const int kind = w0 & 15;
            const int first = w1 >> 16, c0 = w1 & 0xffff;
            if (kind == kResGen) {
                const int ng = (w0 >> 4) & 15, nr = (w0 >> 8) & 255, span = w0 >> 16;
                if (lane >= nr * ng) continue;
                const int k = lane / nr;
                const int xa = R.x0 + c0 + span * k / ng, xb = R.x0 + c0 + span * (k + 1) / ng;
                res_gen_item<MODE>(a, Pc, Pp, sz0, sx0, R.zr0 + first + lane - k * nr, xa, xb);
                continue;
            }
            const int ncol = (w0 >> 4) & 15, nl = w0 >> 8;
            if (lane >= nl) continue;
            const int x = R.x0 + c0;
            const int zd = R.zr0 + 4 * (first + lane);
            if (kind == kResFast) {
                const int z = zd - a.zoff;
                res_fast<MODE>(a, sub, ps4, pp4, (zd - sz0) >> 2, x - sx0, x * a.ldz + zd,
                               (x - a.dn) * a.ldf + (z - a.dn), ncol, cc);
            } else if (kind == kResZpml) {
                res_zpml_item(a, ps4, pp4, sz0, sx0, zd, x, ncol);
            } else {
                res_xpml_item(a, ps4, pp4, sx0, (zd - sz0) >> 2, zd, a.fs && zd - a.zoff == a.dn, x, ncol);
            }
        }
        __syncthreads();  // the step's writes precede the publication
        if (tid == 0) st_release(rp.flags + blockIdx.x, s + 1);
    }
    if (tid == 0) cp_async_wait_all();
}

// Dynamic shared memory of a resident block: two level buffers of sw columns.
int res_smem_bytes(int sw) {
    return 2 * RSH * sw * (int)sizeof(float);
}

}  // namespace

// ---- host side -------------------------------------------------------------

namespace {

// Relative time of one warp item of each kind, for the region split and the
// warp assignment: an interior float4 item costs its columns plus the warm-up
// of its register window, an x-strip item about 3 interior columns per
// column, a generic item one global round trip (about 4) and then about 1.5
// per column (the next column's loads overlap the current one's update).
constexpr double kCostFastCol = 1.0, kCostFastItem = 1.0, kCostXpmlCol = 2.2, kCostXpmlItem = 1.0,
                 kCostGenItem = 2.0, kCostGenCol = 2.2, kCostZpmlItem = 1.0, kCostZpmlCol = 1.8;
// Most columns of an interior float4 item (res_fast's unrolled sweep).
constexpr int kFastCols = kFastColsMax;
// Columns a lane of a generic item sweeps (its update is latency-bound).
constexpr int kGenCols = 3;

// Split n units with costs c[0..n) into k consecutive parts of about equal
// cost, each of lo..hi units.  Returns the k+1 boundaries, or an empty
// vector if impossible.
std::vector<int> split_costs(const std::vector<double>& c, int k, int lo, int hi) {
    const int n = (int)c.size();
    if (k <= 0 || (long long)k * lo > n || (long long)k * hi < n) return {};
    std::vector<double> pre(n + 1, 0.0);
    for (int i = 0; i < n; ++i) pre[i + 1] = pre[i] + c[i];
    std::vector<int> cut = {0};
    for (int p = 1; p < k; ++p) {
        const double target = pre[n] * p / k;
        const int prev = cut.back(), parts = k - p;
        int best = -1;
        double bd = 0.0;
        for (int e = prev + lo; e <= std::min(n, prev + hi); ++e) {
            const int rest = n - e;
            if ((long long)rest > (long long)parts * hi || rest < parts * lo) continue;
            const double d = std::abs(pre[e] - target);
            if (best < 0 || d < bd) { best = e; bd = d; }
        }
        if (best < 0) return {};
        cut.push_back(best);
    }
    cut.push_back(n);
    return cut;
}

// Even split of n into parts of at most `most`, and at least `parts` parts.
std::vector<int> chunks(int n, int most, int parts = 1) {
    std::vector<int> c;
    const int k = std::min(n, std::max(parts, (n + most - 1) / most));
    for (int i = 0; i < k; ++i) c.push_back(n * (i + 1) / k - n * i / k);
    return c;
}

struct Item {
    int w0, w1;
    double cost;
};

// Row classes of the live grid, by quad: 2 = interior rows without injection
// or the free surface (a type-0 rect of the step plan), 1 = other rows of the
// interior band, 0 = the rest.
struct RowClasses {
    int zlo = 0, zhi = 0;
    std::vector<char> cls;
};

// The warp items of region R.
std::vector<Item> region_items(const StepArgs& a, const RowClasses& rc, const ResRegion& R) {
    std::vector<Item> its;
    const int dn = a.dn;
    const int q0 = (R.zr0 - rc.zlo) / 4, nqr = R.nrows / 4;
    auto add_runs = [&](int kind, int qa, int qb, int xa, int xb) {
        // quads [qa, qb) (region-relative) x columns [xa, xb) (absolute)
        if (qb <= qa || xb <= xa) return;
        const std::vector<int> qc = chunks(qb - qa, 32);
        const int most = kind == kResFast ? kFastCols : (kind == kResZpml ? 4 : 2);
        const int parts = kind == kResFast ? kResWarps / (int)qc.size() : 1;  // fill the warps
        int qs = qa;
        for (int nqc : qc) {
            int xs = xa;
            for (int ncc : chunks(xb - xa, most, parts)) {
                const double cost = kind == kResFast ? kCostFastItem + kCostFastCol * ncc
                                                     : (kind == kResZpml ? kCostZpmlItem + kCostZpmlCol * ncc
                                                                         : kCostXpmlItem + kCostXpmlCol * ncc);
                its.push_back({kind | (ncc << 4) | (nqc << 8), (qs << 16) | (xs - R.x0), cost});
                xs += ncc;
            }
            qs += nqc;
        }
    };
    auto add_gen = [&](int qa, int qb, int xa, int xb) {
        // rows [4qa, 4qb) x columns [xa, xb): lanes are nr rows x ng column
        // groups, each lane sweeping up to kGenCols columns of its group
        const int nrows = 4 * (qb - qa), ncols = xb - xa;
        if (nrows <= 0 || ncols <= 0) return;
        if (nrows >= 16) {
            int rs = 4 * qa;
            for (int nr : chunks(nrows, 32)) {
                int xs = xa;
                for (int span : chunks(ncols, kGenCols)) {
                    its.push_back({kResGen | (1 << 4) | (nr << 8) | (span << 16), (rs << 16) | (xs - R.x0),
                                   kCostGenItem + kCostGenCol * span});
                    xs += span;
                }
                rs += nr;
            }
        } else {
            const int ng = std::min(std::min(32 / nrows, ncols), 15);
            const int nit = (ncols + kGenCols * ng - 1) / (kGenCols * ng);
            int xs = xa;
            for (int span : chunks(ncols, kGenCols * ng, nit)) {
                const int g = std::min(ng, span);
                its.push_back({kResGen | (g << 4) | (nrows << 8) | (span << 16), ((4 * qa) << 16) | (xs - R.x0),
                               kCostGenItem + kCostGenCol * ((span + g - 1) / g)});
                xs += span;
            }
        }
    };
    const int xi0 = std::max(R.x0, dn), xi1 = std::min(R.x0 + R.w, dn + a.nx);
    int q = 0;
    while (q < nqr) {
        const int c = rc.cls[q0 + q];
        int e = q + 1;
        while (e < nqr && rc.cls[q0 + e] == c) ++e;
        if (c == 2) add_runs(kResFast, q, e, xi0, xi1);  // interior columns
        if (c == 1 || c == 2) {                          // x-strip columns of the band
            add_runs(kResXpml, q, e, R.x0, std::min(R.x0 + R.w, std::max(R.x0, dn)));
            add_runs(kResXpml, q, e, std::max(R.x0, dn + a.nx), R.x0 + R.w);
        }
        if (c == 1) add_gen(q, e, xi0, xi1);          // band rows with injection or the free surface
        if (c == 3) {                                 // z-strip rows: float4 path on interior columns
            add_runs(kResZpml, q, e, xi0, xi1);
            add_gen(q, e, R.x0, std::min(R.x0 + R.w, std::max(R.x0, dn)));
            add_gen(q, e, std::max(R.x0, dn + a.nx), R.x0 + R.w);
        }
        if (c == 0) add_gen(q, e, R.x0, R.x0 + R.w);  // strip edges, corners, partial quads
        q = e;
    }
    return its;
}

// Longest-processing-time assignment of items to the warps of a block;
// returns the largest warp load and, if per != nullptr, the items of each warp.
double assign_warps(std::vector<Item>& its, std::vector<std::vector<int>>* per) {
    std::stable_sort(its.begin(), its.end(), [](const Item& u, const Item& v) { return u.cost > v.cost; });
    std::vector<double> load(kResWarps, 0.0);
    if (per) per->assign(kResWarps, {});
    for (size_t i = 0; i < its.size(); ++i) {
        const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[w] += its[i].cost;
        if (per) (*per)[w].push_back((int)i);
    }
    return *std::max_element(load.begin(), load.end());
}

std::vector<ResRegion> regions_of(const RowClasses& rc, const std::vector<int>& rows, const std::vector<int>& cols) {
    std::vector<ResRegion> reg;
    for (size_t i = 0; i + 1 < rows.size(); ++i)
        for (size_t j = 0; j + 1 < cols.size(); ++j) {
            ResRegion R{};
            R.zr0 = rc.zlo + 4 * rows[i];
            R.nrows = 4 * (rows[i + 1] - rows[i]);
            R.x0 = cols[j];
            R.w = cols[j + 1] - cols[j];
            reg.push_back(R);
        }
    return reg;
}

}  // namespace

bool plan_resident(const StepArgs& a, int max_regions, int max_sw, int nrec, const int* h_rec_cell, ResPlan* plan) {
    const int dn = a.dn, zoff = a.zoff;
    const int d0 = dn + zoff;  // first interior row (a multiple of 4)
    RowClasses rc;
    rc.zlo = a.fs ? d0 : (zoff & ~3);  // live device rows [zlo, zhi)
    rc.zhi = (zoff + a.nyt + 3) & ~3;
    const int nq = (rc.zhi - rc.zlo) / 4, ncolg = a.nxt;
    const int max_w = max_sw - 6;
    if (4 * nq < kResMinSide || ncolg < kResMinSide || max_w < kResMinSide || max_regions < 1) return false;
    rc.cls.assign(nq, 0);
    const int ny4 = a.ny & ~3;
    for (int zd = d0; zd < d0 + ny4; zd += 4)
        if (zd >= rc.zlo && zd < rc.zhi) rc.cls[(zd - rc.zlo) / 4] = 1;
    for (int r = 0; r < a.nrect; ++r)
        if (a.r_type[r] == 0)
            for (int zd = a.r_zd0[r]; zd < a.r_zd0[r] + a.r_h[r]; zd += 4)
                if (zd >= rc.zlo && zd < rc.zhi) rc.cls[(zd - rc.zlo) / 4] = 2;
    for (int q = 0; q < nq; ++q) {  // z-strip quads whose rows are 3 or more rows inside their strip
        bool ok = true;
        for (int r = 0; r < 4; ++r) {
            const int z = rc.zlo + 4 * q + r - zoff;
            const int sb = z < dn ? 0 : dn + a.ny;
            const bool strip = z >= 0 && z < a.nyt && (z < dn || z >= dn + a.ny) && !(a.fs && z < dn);
            ok = ok && strip && z - sb >= 3 && z - sb <= dn - 4;
        }
        if (ok) rc.cls[q] = 3;
    }
    // Marginal costs per quad and per column (for cost-balanced cuts).
    auto col_interior = [&](int x) { return x >= dn && x < dn + a.nx; };
    std::vector<double> qcost(nq, 0.0), xcost(ncolg, 0.0);
    const double ni = a.nx, ns = ncolg - a.nx;
    for (int q = 0; q < nq; ++q) {
        const int c = rc.cls[q];
        qcost[q] = c == 2 ? ni * kCostFastCol + ns * kCostXpmlCol
                          : (c == 1 ? ni * kCostGenItem / 8 + ns * kCostXpmlCol
                                    : (c == 3 ? ni * kCostZpmlCol + ns * kCostGenItem / 8 : ncolg * kCostGenItem / 8));
    }
    for (int x = 0; x < ncolg; ++x)
        for (int q = 0; q < nq; ++q) {
            const int c = rc.cls[q];
            const bool in = col_interior(x);
            xcost[x] += (c == 2 && in) ? kCostFastCol
                                       : ((c == 3 && in) ? kCostZpmlCol
                                                         : ((c == 1 || c == 2) && !in ? kCostXpmlCol : kCostGenItem / 8));
        }
    // The region grid whose busiest warp has the least work.
    double best = -1.0;
    std::vector<int> brow, bcol;
    for (int cr = 1; cr <= std::min(max_regions, nq / (kResMinSide / 4)); ++cr) {
        const std::vector<int> rows = split_costs(qcost, cr, kResMinSide / 4, kResRows / 4);
        if (rows.empty()) continue;
        const int cmax = std::min(max_regions / cr, ncolg / kResMinSide);
        for (int cc = cmax; cc >= std::max(1, cmax - 3); --cc) {
            if ((long long)cc * max_w < ncolg) break;
            const std::vector<int> cols = split_costs(xcost, cc, kResMinSide, max_w);
            if (cols.empty()) continue;
            double worst = 0.0, sum = 0.0;
            for (const ResRegion& R : regions_of(rc, rows, cols)) {
                std::vector<Item> its = region_items(a, rc, R);
                const double m = assign_warps(its, nullptr);
                worst = std::max(worst, m);
                sum += m;
            }
            worst += 0.3 * sum / std::max<size_t>(1, (rows.size() - 1) * (cols.size() - 1));
            if (best < 0 || worst < best) {
                best = worst;
                brow = rows;
                bcol = cols;
            }
        }
    }
    if (best < 0) return false;
    plan->reg = regions_of(rc, brow, bcol);
    plan->nbr.clear();
    plan->rec.clear();
    plan->items.clear();
    plan->warp_first.assign(1, 0);
    plan->sw = 0;
    for (const ResRegion& R : plan->reg) plan->sw = std::max(plan->sw, R.w + 6);
    const int nreg = (int)plan->reg.size();
    // Neighbours: regions within kTileReadHalo cells (the reach of a step's
    // reads of p, phi and the free-surface histories).
    for (int b = 0; b < nreg; ++b) {
        ResRegion& R = plan->reg[b];
        R.nbr0 = (int)plan->nbr.size();
        for (int o = 0; o < nreg; ++o) {
            if (o == b) continue;
            const ResRegion& Q = plan->reg[o];
            const bool zx = Q.zr0 < R.zr0 + R.nrows + kTileReadHalo && R.zr0 < Q.zr0 + Q.nrows + kTileReadHalo;
            const bool xx = Q.x0 < R.x0 + R.w + kTileReadHalo && R.x0 < Q.x0 + Q.w + kTileReadHalo;
            if (zx && xx) plan->nbr.push_back(o);
        }
        R.nnbr = (int)plan->nbr.size() - R.nbr0;
        if (R.nnbr > kResThreads) return false;
    }
    // Receivers by owning region.
    for (int b = 0; b < nreg; ++b) {
        ResRegion& R = plan->reg[b];
        R.rec0 = (int)plan->rec.size();
        for (int i = 0; i < nrec; ++i) {
            const int x = h_rec_cell[i] / a.ldz, zd = h_rec_cell[i] % a.ldz;
            if (zd >= R.zr0 && zd < R.zr0 + R.nrows && x >= R.x0 && x < R.x0 + R.w) plan->rec.push_back(i);
        }
        R.nrec = (int)plan->rec.size() - R.rec0;
    }
    if ((int)plan->rec.size() != nrec) return false;  // a receiver outside the live grid
    // Work items of each region by warp.
    for (int b = 0; b < nreg; ++b) {
        std::vector<Item> its = region_items(a, rc, plan->reg[b]);
        std::vector<std::vector<int>> per;
        assign_warps(its, &per);
        for (int w = 0; w < kResWarps; ++w) {
            for (int i : per[w]) {
                plan->items.push_back(its[i].w0);
                plan->items.push_back(its[i].w1);
            }
            plan->warp_first.push_back((int)plan->items.size() / 2);
        }
    }
    return true;
}

int resident_max_sw() {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
    const int stat = 2 * (int)sizeof(StepArgs) + 2 * (int)sizeof(PassVar) + 1024;
    return (optin - stat) / (2 * RSH * (int)sizeof(float));
}

template <int MODE>
int res_blocks_t(int sw) {
    const int bytes = res_smem_bytes(sw);
    if (cudaFuncSetAttribute(res_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, res_kernel<MODE>, kResThreads, bytes) != cudaSuccess)
        return 0;
    return n;
}

int resident_blocks_per_sm(int mode, int sw) {
    cudaGetLastError();
    const int n = mode == 0 ? res_blocks_t<0>(sw) : (mode == 1 ? res_blocks_t<1>(sw) : 0);
    cudaGetLastError();
    return n;
}

template <int MODE>
int launch_res_t(const ResParams& rp, cudaStream_t stream) {
    const int bytes = res_smem_bytes(rp.sw);
    cudaError_t e = cudaFuncSetAttribute(res_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return (int)e;
    void* args[] = {const_cast<ResParams*>(&rp)};
    e = cudaLaunchCooperativeKernel((const void*)res_kernel<MODE>, dim3(rp.nreg), dim3(kResThreads), args,
                                    (size_t)bytes, stream);
    return (int)e;
}

int launch_resident(int mode, const ResParams& rp, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (mode == 0) return launch_res_t<0>(rp, s);
    if (mode == 1) return launch_res_t<1>(rp, s);
    return (int)cudaErrorInvalidValue;
}

}  // namespace psdm
