// Two time steps per launch (temporal blocking) for sm_100a.
//
// The same per-cell arithmetic as the one-step kernels (rtm_step.cu), which
// follow src/solver_ac_forward_ram.f90:344-573 and
// src/solver_ac_backward_ram.f90:329-545 in the reference's evaluation
// order, organised so that a launch advances the grid by two steps:
//
//   * a tile loads level n on itself plus a 6-cell ring, computes level n+1
//     on itself plus a 3-cell ring into shared memory (the ring cells are
//     computed again, with the same arithmetic, by the tiles that own them),
//     and then level n+2 on itself;
//   * levels n-1 and n are only read, levels n+1 and n+2 go to two other
//     buffers (the wavefield rotates through four); the C-PML memory
//     variables phi and chi read level n and write level n+2 to a second
//     buffer, level n+1 living only in shared memory; the free-surface
//     histories rotate like the wavefield;
//   * both steps' snapshots (forward) or imaging updates (backward), source
//     or adjoint-source injections and receiver samples are done by the tile
//     that owns the cell, in step order.
//
// Per step and cell the wavefield crosses HBM half as often as with one
// launch per step (p, p1 and c2 are read once for two steps) and the launch
// count halves.  A launch may also do a single step (nsub = 1), which ends a
// pass with an odd number of steps.
//
// Tiles: "clean" interior tiles (rect type 0) whose tile and 3-cell ring
// hold only interior cells with no injection and no free-surface row, 120
// rows x 28 columns, level n staged in shared memory by bulk asynchronous
// copies, each thread sliding a float4 x 7-column window through registers
// with the packed FP32x2 stencil of the one-step interior tiles; and
// "generic" tiles (rect type 1, at most 26 x 32 cells) for everything else:
// C-PML strips and corners (with the phi/chi recursions of
// src/solver_PML_matrices.f90:1-111), the free-surface and injection rows,
// and the interior cells next to them: a lane per row, a warp per run of
// columns, one cell per thread at a time.
//
// Reach: a cell's update reads its neighbours within 3 cells, except where
// a stencil centre is clamped (the reference copies the derivative at
// acc+1 into the first acc cells, src/solver_space_derivs_clean.f90) or a
// strip-local phi derivative is clamped to its strip
// (src/solver_PML_matrices.f90:9-38); those reads reach up to 6 cells, but
// always towards the inside of the grid or strip.  The planner therefore
// starts tiles at every strip and grid edge and keeps them at least 8 cells
// wide and high there, so that every read of level n+1 by a tile's cells
// lies in its 3-cell ring and every read of level n by the ring lies within
// 6 cells.

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

#include "rtm_device.cuh"
#include "rtm_internal.h"

namespace psdm {
namespace {

// Clean interior tiles: TZC output rows (30 float4 rows; level n+1 is
// computed on 32 float4 rows, one per lane) by TXC columns.
constexpr int TZC = 120;
constexpr int XSC = 7;              // output columns per warp
constexpr int TXC = NWARP * XSC;    // 28
constexpr int HS0 = TZC + 16;       // rows of the level-n tile (6-row ring rounded up to 8)
constexpr int HS1 = TZC + 8;        // rows of the level n+1 tile (3-row ring rounded up to 4)
constexpr int Q0 = HS0 / 4, Q1 = HS1 / 4;
constexpr int WS0 = TXC + 12, WS1 = TXC + 6;
constexpr int kCleanFloats = HS0 * WS0 + HS1 * WS1;
// Generic tiles: at most GZ x GX cells; GZ + 6 = 32 rows, one per lane, in
// the first step.
constexpr int GZ = 26, GX = 32;
constexpr int GH0 = GZ + 12, GW0 = GX + 12;  // level n on the tile + 6
constexpr int GH1 = GZ + 6, GW1 = GX + 6;    // level n+1, phi and chi at n+1 on the tile + 3
constexpr int kGenericFloats = GH0 * GW0 + 5 * GH1 * GW1 + GW1;
constexpr int kPairFloats = kCleanFloats > kGenericFloats ? kCleanFloats : kGenericFloats;

// Largest |snapshot| of each sub-step seen by this block (float bits).
__shared__ unsigned int s_pair_amax[2];

// One phase of a clean interior tile (rows [z0, z0+nrows), a multiple of 4
// starting on a float4 boundary; columns [x0, x0+ncols)).
//   PH = 0: level n+1 on rows [z0-4, z0+nrows+4) x columns [x0-3,
//     x0+ncols+3) from level n in S0 (rows from z0-8, columns from x0-6) and
//     level n-1 from HBM, into S1 (rows from z0-4, columns from x0-3); on the
//     tile also to p_out[0], with sub-step 0's snapshot or imaging.
//   PH = 1: level n+2 on the tile from S1, with level n from S0, to p_out[1]
//     and over level n in S0 (for the receiver gather), with sub-step 1's
//     snapshot or imaging.
// Lane l owns the float4 of rows z0-4+4l (PH 0) or z0+4l (PH 1); warp w a
// run of consecutive columns, swept with a 7-column register window.
template <int MODE, int PH>
__device__ __forceinline__ void clean_phase(const PairArgs& P, float* S0, float* S1, int z0, int x0, int nrows,
                                            int ncols, const float2 (&cc)[4]) {
    const StepArgs& a = P.a;
    const SubStep& s = P.sub[PH];
    const int lane = threadIdx.x, w = threadIdx.y;
    const int nq = PH == 0 ? (nrows >> 2) + 2 : (nrows >> 2);
    const int ncl = PH == 0 ? ncols + 6 : ncols;
    const int cb = (w * ncl) >> 2, ce = ((w + 1) * ncl) >> 2;
    // at most (TXC + 6) / 4 columns per warp: the loop below is unrolled to
    // that bound, so the register window shifts by renaming
    constexpr int MAXC = PH == 0 ? (TXC + 6 + NWARP - 1) / NWARP : XSC;
    const int ncw = ce - cb;
    if (lane >= nq || ncw <= 0) return;
    const int zd = PH == 0 ? z0 - 4 + 4 * lane : z0 + 4 * lane;
    constexpr int SQ = PH == 0 ? Q0 : Q1;
    const float4* __restrict__ src = reinterpret_cast<const float4*>(PH == 0 ? S0 : S1);
    float4* S0v = reinterpret_cast<float4*>(S0);
    float4* S1v = reinterpret_cast<float4*>(S1);
    const int sr = lane + 1;  // float4 row of this thread's float4 in the source tile
    const bool rowT = PH == 1 || (lane >= 1 && lane <= (nrows >> 2));
    const int xb = PH == 0 ? x0 - 3 : x0;  // column of phase column 0
    const int tc0 = PH == 0 ? 3 : 0, tc1 = PH == 0 ? ncols + 3 : ncols;
    const int dn = a.dn;
    const bool snap = MODE == 0 && s.field != nullptr;
    const bool img = MODE == 1 && s.field != nullptr;
    const bool img16 = MODE == 2 && s.field16 != nullptr;
    const float isc = img16 ? __ldg(s.field_iscale) : 1.f;
    float amax_t = 0.f;
    int g = (xb + cb) * a.ldz + zd;
    int fi = (xb + cb - dn) * a.ldf + (zd - a.zoff - dn);
    float4 pmN = PH == 0 ? __ldg(reinterpret_cast<const float4*>(a.pm + g)) : S0v[(cb + 6) * Q0 + lane + 2];
    float4 c2N = __ldg(reinterpret_cast<const float4*>(a.c2 + g));
    float4 Fn = make_float4(0.f, 0.f, 0.f, 0.f), In = Fn, Cn = Fn;
    uint2 Fr = make_uint2(0u, 0u);
    if (rowT && cb >= tc0 && cb < tc1) {
        if (img) {
            Fn = __ldg(reinterpret_cast<const float4*>(s.field + fi));
            In = *reinterpret_cast<const float4*>(a.image + fi);
        }
        if (img16) {
            Fr = load16x4_raw(s.field16, fi);
            In = *reinterpret_cast<const float4*>(a.image + fi);
            Cn = *reinterpret_cast<const float4*>(a.comp + fi);
        }
    }
    float4 win[7];
#pragma unroll
    for (int k = 0; k < 6; ++k) win[k] = src[(cb + k) * SQ + sr];
#pragma unroll
    for (int j = 0; j < MAXC; ++j) {
        if (j >= ncw) break;
        const int c = cb + j;
        win[6] = src[(c + 6) * SQ + sr];
        const float4 zm = src[(c + 3) * SQ + sr - 1];
        const float4 zp = src[(c + 3) * SQ + sr + 1];
        const float4 pmv = pmN, c2v = c2N;
        if (j + 1 < ncw) {
            pmN = PH == 0 ? __ldg(reinterpret_cast<const float4*>(a.pm + g + a.ldz)) : S0v[(c + 7) * Q0 + lane + 2];
            c2N = __ldg(reinterpret_cast<const float4*>(a.c2 + g + a.ldz));
        }
        const float4 Fc = Fn, Ic = In, Cc = Cn;
        const uint2 Frc = Fr;
        const bool t = rowT && c >= tc0 && c < tc1;
        if (j + 1 < ncw && rowT && c + 1 >= tc0 && c + 1 < tc1) {
            if (img) {
                Fn = __ldg(reinterpret_cast<const float4*>(s.field + fi + a.ldf));
                In = *reinterpret_cast<const float4*>(a.image + fi + a.ldf);
            }
            if (img16) {
                Fr = load16x4_raw(s.field16, fi + a.ldf);
                In = *reinterpret_cast<const float4*>(a.image + fi + a.ldf);
                Cn = *reinterpret_cast<const float4*>(a.comp + fi + a.ldf);
            }
        }
        const float4 out = clean_update(win, zm, zp, pmv, c2v, cc);
        if (PH == 0) S1v[c * Q1 + lane] = out;
        if (t) {
            *reinterpret_cast<float4*>(P.p_out[PH] + g) = out;
            if (PH == 1) S0v[(c + 6) * Q0 + lane + 2] = out;
            if (snap || img || img16) emit4<MODE>(a, s, fi, out, pmv, Fc, Ic, Cc, Frc, isc, amax_t);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) win[k] = win[k + 1];
        g += a.ldz;
        fi += a.ldf;
    }
    if (snap && s.field_amax != nullptr && amax_t > 0.f) atomicMax(&s_pair_amax[PH], __float_as_uint(amax_t));
}

// Receiver samples of tile b (forward): sub-step 0's level from S1, sub-step
// 1's from S0.  (oz0, ox0) / (oz1, ox1) are the origins (device row, column)
// of S0 / S1, with pitches h0 / h1.
__device__ __forceinline__ void gather_receivers(const PairArgs& P, int b, const float* S0, int oz0, int ox0, int h0,
                                                 const float* S1, int oz1, int ox1, int h1) {
    const StepArgs& a = P.a;
    const int j0 = P.rec_first[b], j1 = P.rec_first[b + 1];
    if (j1 <= j0) return;
    __syncthreads();  // both levels complete
    const int t0 = P.sub[0].rec_t, t1 = P.nsub == 2 ? P.sub[1].rec_t : -1;
    for (int j = j0 + threadIdx.y * 32 + threadIdx.x; j < j1; j += NT) {
        const int i = P.rec_idx[j];
        const int cell = a.rec_cell[i];
        const int x = cell / a.ldz, zd = cell - x * a.ldz;
        if (t0 >= 0) a.rec_out[(size_t)i * a.rec_ld + t0] = S1[(x - ox1) * h1 + (zd - oz1)];
        if (t1 >= 0) a.rec_out[(size_t)i * a.rec_ld + t1] = S0[(x - ox0) * h0 + (zd - oz0)];
    }
}

// Clean interior tile t of rect r (tile b of the launch).  Returns false if
// its bulk copies did not complete (error reported).
template <int MODE>
__device__ __forceinline__ bool pair_clean_tile(const PairArgs& P, float* sm, uint64_t* bar, uint32_t& phase, int r,
                                                int t, int b) {
    const StepArgs& a = P.a;
    const int lane = threadIdx.x, wy = threadIdx.y;
    if (P.txc != TXC) {  // planned for another tile width: report, touch nothing
        if (lane == 0 && wy == 0) atomicExch(a.err, 2);
        return false;
    }
    const int tz = t % P.r_tz[r], tx = t / P.r_tz[r];
    const int z0 = P.r_zd0[r] + tz * TZC, x0 = P.r_x0[r] + tx * TXC;
    const int nrows = min(TZC, P.r_zd0[r] + P.r_h[r] - z0);  // a multiple of 4
    const int ncols = min(TXC, P.r_x0[r] + P.r_w[r] - x0);
    float* S0 = sm;
    float* S1 = sm + HS0 * WS0;
    if (wy == 0) {  // level n, rows [z0-8, z0+nrows+8) x columns [x0-6, x0+ncols+6)
        const uint32_t prow = (uint32_t)(nrows + 16) * 4u;
        const uint32_t bytes = (uint32_t)(ncols + 12) * prow;
        fence_proxy_async();  // the previous tile's shared accesses precede these writes
        if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
        __syncwarp();
        for (int c = lane; c < ncols + 12; c += 32)
            bulk_g2s(S0 + c * HS0, a.p + (size_t)(x0 - 6 + c) * a.ldz + (z0 - 8), prow, bar);
    }
    float2 cc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) cc[k] = make_float2(a.cf2[k], a.cf2[k]);
    const bool ok = mbar_wait_bounded(bar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
        if (lane == 0 && wy == 0) atomicExch(a.err, 1);
        return false;
    }
    clean_phase<MODE, 0>(P, S0, S1, z0, x0, nrows, ncols, cc);
    if (P.nsub == 2) {
        __syncthreads();
        clean_phase<MODE, 1>(P, S0, S1, z0, x0, nrows, ncols, cc);
    }
    if (MODE == 0 && P.rec_first != nullptr) gather_receivers(P, b, S0, z0 - 8, x0 - 6, HS0, S1, z0 - 4, x0 - 3, HS1);
    return true;
}

// Shared-memory views of a generic tile (rows [z0, z1) x columns [x0, x1)).
struct GenTile {
    float* S0;   // level n on rows [z0-6, z1+6) x columns [x0-6, x1+6), pitch GH0
    float* S1;   // level n+1 on rows [z0-3, z1+3) x columns [x0-3, x1+3), pitch GH1
    float* F1x;  // phi_x, phi_z, chi_x, chi_z at level n+1, laid out like S1
    float* F1z;
    float* X1x;
    float* X1z;
    float* SD1;  // free-surface history at level n+1 by column (from x0-3)
    int z0, z1, x0, x1;
};

// Snapshot store (forward) or imaging update (backward) of interior cell fi
// of the migration window at sub-step SUB, from its level n+1+SUB value and
// its level n+SUB-1 value pmo.
template <int MODE, int SUB>
__device__ __forceinline__ void pair_field(const PairArgs& P, int fi, float out, float pmo) {
    const StepArgs& a = P.a;
    const SubStep& s = P.sub[SUB];
    if (MODE == 0) {
        if (s.field != nullptr) {
            const float D = div_dt(a, __fmul_rn(__fsub_rn(out, pmo), 0.5f));
            s.field[fi] = D;
            if (s.field_amax != nullptr) atomicMax(&s_pair_amax[SUB], __float_as_uint(fabsf(D)));
        }
    } else if (MODE == 1) {
        if (s.field != nullptr) {
            float F = __ldg(s.field + fi);
            if (s.field_w != 1.f) F = __fmul_rn(F, s.field_w);
            float inc = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out, pmo)), F);
            if (a.ss != 1.f) inc = __fmul_rn(inc, a.ss);
            a.image[fi] = __fadd_rn(a.image[fi], inc);
        }
    } else if (s.field16 != nullptr) {
        float F = load16x1(s.field16, fi, a.kind16, __ldg(s.field_iscale));
        if (s.field_w != 1.f) F = __fmul_rn(F, s.field_w);
        float inc = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out, pmo)), F);
        if (a.ss != 1.f) inc = __fmul_rn(inc, a.ss);
        kahan(a.image[fi], a.comp[fi], inc);
    }
}

// One cell of a generic tile at sub-step SUB: the one-step kernels' generic
// cell update (cell_generic, rtm_device.cuh) with its sources moved:
//   SUB 0: stencil level n from S0, level n-1 / phi / chi at level n and the
//     free-surface histories (levels n, n-1) from HBM; results to S1 and the
//     phi / chi / history tiles, and on the tile to the level n+1 outputs;
//   SUB 1: stencil level n+1 from S1, level n from S0, phi / chi / history
//     at level n+1 from shared memory and the history at level n from HBM;
//     results to the level n+2 outputs (and over level n in S0).
template <int MODE, int SUB>
__device__ __forceinline__ void pair_cell(const PairArgs& P, const GenTile& G, int zd, int x) {
    const StepArgs& a = P.a;
    const SubStep& s = P.sub[SUB];
    const int dn = a.dn;
    const int z = zd - a.zoff;
    const int i1 = (x - (G.x0 - 3)) * GH1 + (zd - (G.z0 - 3));
    const int i0 = (x - (G.x0 - 6)) * GH0 + (zd - (G.z0 - 6));
    if (z < 0 || z >= a.nyt || x < 0 || x >= a.nxt || (a.fs && z < dn)) {
        // outside the grid, or above a free surface: never updated, zero
        if (SUB == 0) G.S1[i1] = 0.f;
        return;
    }
    const bool inT = SUB == 1 || (zd >= G.z0 && zd < G.z1 && x >= G.x0 && x < G.x1);
    const int kz = (z < dn) ? (dn - z) : (z >= dn + a.ny ? z - (dn + a.ny) + 1 : 0);
    const int kx = (x < dn) ? (dn - x) : (x >= dn + a.nx ? x - (dn + a.nx) + 1 : 0);
    const bool fsrow = a.fs && z == dn;
    const bool side = fsrow && kx > 0 && !a.disk;
    const float* SS = SUB == 0 ? G.S0 : G.S1;
    constexpr int SP = SUB == 0 ? GH0 : GH1;
    const int oz = SUB == 0 ? G.z0 - 6 : G.z0 - 3, ox = SUB == 0 ? G.x0 - 6 : G.x0 - 3;
    const int cx = clampi(x, 3, a.nxt - 4);
    const int czd = clampi(z, 3, a.nyt - 4) + a.zoff;
    const float* colc = SS + (cx - ox) * SP + (zd - oz);  // x-stencil centre
    const float* colz = SS + (x - ox) * SP + (czd - oz);  // z-stencil centre
#define AX(k) colc[(k) * SP]
#define AZ(k) colz[(k)]
    const float d2x = D2(AX, a.cf2);
    const float d2y = D2(AZ, a.cf2);
    const int g = x * a.ldz + zd;
    const float pc = SS[(x - ox) * SP + (zd - oz)];
    // Every HBM operand of a pair launch is only read during the launch
    // (its outputs go to other buffers), so read-only cached loads are safe.
    const float pmo = SUB == 0 ? __ldg(a.pm + g) : G.S0[i0];
    const float c2v = __ldg(a.c2 + g);
    float pp = pc, ppm = pmo;
    if (side) {
        if (SUB == 0) {
            pp = __ldg(a.side_p + x);
            ppm = __ldg(a.side_pm + x);
        } else {
            pp = G.SD1[x - (G.x0 - 3)];
            ppm = __ldg(a.side_p + x);
        }
    }
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
            float dph, phold, chold;
            if (SUB == 0) {
                const float* ph = a.phix_in + (size_t)ci * a.ldz + zd;
#define PX(k) __ldg(ph + (k) * a.ldz)
                dph = D1(PX, a.cf1);
#undef PX
                phold = __ldg(a.phix_in + g);
                chold = __ldg(P.chix_in + g);
            } else {
                const float* ph = G.F1x + (ci - (G.x0 - 3)) * GH1 + (zd - (G.z0 - 3));
#define PX(k) ph[(k) * GH1]
                dph = D1(PX, a.cf1);
#undef PX
                phold = G.F1x[i1];
                chold = G.X1x[i1];
            }
            const float phn = __fadd_rn(__fmul_rn(A, phold), __fmul_rn(B, d1));
            const float chn = __fadd_rn(__fmul_rn(A, chold), __fmul_rn(B, __fadd_rn(d2x, dph)));
            if (SUB == 0) {
                G.F1x[i1] = phn;
                G.X1x[i1] = chn;
                if (inT && P.nsub == 1) {
                    a.phix_out[g] = phn;
                    a.chix[g] = chn;
                }
            } else {
                a.phix_out[g] = phn;
                a.chix[g] = chn;
            }
            propx = __fadd_rn(dph, chn);
        }
        if (kz > 0) {
            const float d1 = D1(AZ, a.cf1);
            const int sb = (z < dn) ? 0 : dn + a.ny;
            const int cj = clampi(z - sb, 3, dn - 4) + sb + a.zoff;
            float dph, phold, chold;
            if (SUB == 0) {
                const float* ph = a.phiz_in + (size_t)x * a.ldz + cj;
#define PZ(k) __ldg(ph + (k))
                dph = D1(PZ, a.cf1);
#undef PZ
                phold = __ldg(a.phiz_in + g);
                chold = __ldg(P.chiz_in + g);
            } else {
                const float* ph = G.F1z + (x - (G.x0 - 3)) * GH1 + (cj - (G.z0 - 3));
#define PZ(k) ph[(k)]
                dph = D1(PZ, a.cf1);
#undef PZ
                phold = G.F1z[i1];
                chold = G.X1z[i1];
            }
            const float phn = __fadd_rn(__fmul_rn(A, phold), __fmul_rn(B, d1));
            const float chn = __fadd_rn(__fmul_rn(A, chold), __fmul_rn(B, __fadd_rn(d2y, dph)));
            if (SUB == 0) {
                G.F1z[i1] = phn;
                G.X1z[i1] = chn;
                if (inT && P.nsub == 1) {
                    a.phiz_out[g] = phn;
                    a.chiz[g] = chn;
                }
            } else {
                a.phiz_out[g] = phn;
                a.chiz[g] = chn;
            }
            propz = __fadd_rn(dph, chn);
        }
        main_term = (kx > 0) ? propx : propz;
    } else {
        float src = 0.f;
        if (a.row_slot != nullptr) {
            const int rs = __ldg(a.row_slot + zd);
            if (rs >= 0) {
                const int j = __ldg(a.inj_cols + rs * a.nxt + x);
                if (j >= 0) src = __ldg(a.inj_trace + (size_t)j * a.inj_ld + s.inj_t);
            }
        }
        main_term = src;
    }
#undef AX
#undef AZ
    float p3 = __fadd_rn(base, __fmul_rn(c2v, __fadd_rn(__fadd_rn(d2x, d2y), main_term)));
    if (kx > 0 && kz > 0) p3 = __fadd_rn(p3, __fmul_rn(c2v, propz));
    float out = p3;
    if (fsrow && (kx == 0 || !a.disk)) out = 0.f;
    if (SUB == 0) {
        G.S1[i1] = out;
        if (side) G.SD1[x - (G.x0 - 3)] = p3;
        if (inT) {
            P.p_out[0][g] = out;
            if (side) P.side_out[0][x] = p3;
        }
    } else {
        P.p_out[1][g] = out;
        G.S0[i0] = out;
        if (side) P.side_out[1][x] = p3;
    }
    if (MODE == 0 && inT && s.band != nullptr) {  // the band of this level (boundary-saved reconstruction)
        if (kz == 0 && kx >= 1 && kx <= 3)
            s.band[(x < dn ? x - (dn - 3) : 3 + x - (dn + a.nx)) * a.ny + (z - dn)] = out;
        else if (kx == 0 && kz >= 1 && kz <= 3)
            s.band[6 * a.ny + (x - dn) * 6 + (z >= dn + a.ny ? z - (dn + a.ny) : 3 + z - (dn - 3))] = out;
    }
    if (inT && kx == 0 && kz == 0) pair_field<MODE, SUB>(P, (x - dn) * a.ldf + (z - dn), out, pmo);
}

// Tile bounds of generic rect r, tile t: an even split of the rect into
// r_tz x r_tx tiles.
__host__ __device__ __forceinline__ void generic_bounds(const PairArgs& P, int r, int t, int* z0, int* z1, int* x0,
                                                        int* x1) {
    const int nz = P.r_tz[r], nxr = P.r_tx[r];
    const int tz = t % nz, tx = t / nz;
    *z0 = P.r_zd0[r] + (tz * P.r_h[r]) / nz;
    *z1 = P.r_zd0[r] + ((tz + 1) * P.r_h[r]) / nz;
    *x0 = P.r_x0[r] + (tx * P.r_w[r]) / nxr;
    *x1 = P.r_x0[r] + ((tx + 1) * P.r_w[r]) / nxr;
}

template <int MODE>
__device__ __forceinline__ void pair_generic_tile(const PairArgs& P, float* sm, int r, int t, int b) {
    const StepArgs& a = P.a;
    GenTile G;
    generic_bounds(P, r, t, &G.z0, &G.z1, &G.x0, &G.x1);
    G.S0 = sm;
    G.S1 = G.S0 + GH0 * GW0;
    G.F1x = G.S1 + GH1 * GW1;
    G.F1z = G.F1x + GH1 * GW1;
    G.X1x = G.F1z + GH1 * GW1;
    G.X1z = G.X1x + GH1 * GW1;
    G.SD1 = G.X1z + GH1 * GW1;
    const int H = G.z1 - G.z0, W = G.x1 - G.x0;
    const int H0 = H + 12, W0 = W + 12;
    const int lane = threadIdx.x, w = threadIdx.y;
    for (int xl = w; xl < W0; xl += NWARP) {
        const int x = G.x0 - 6 + xl;
        const bool xin = x >= 0 && x < a.nxt;
        for (int zl = lane; zl < H0; zl += 32) {
            const int zd = G.z0 - 6 + zl;
            G.S0[xl * GH0 + zl] = (xin && zd >= 0 && zd < a.ldz) ? __ldg(a.p + (size_t)x * a.ldz + zd) : 0.f;
        }
    }
    __syncthreads();
    // first step on rows [z0-3, z1+3) (a lane each) x columns [x0-3, x1+3)
    // (a run of columns per warp)
    const int H1 = H + 6, W1 = W + 6;
    if (lane < H1) {
        const int zd = G.z0 - 3 + lane;
        const int cb = (w * W1) / NWARP, ce = ((w + 1) * W1) / NWARP;
#pragma unroll 1
        for (int c = cb; c < ce; ++c) pair_cell<MODE, 0>(P, G, zd, G.x0 - 3 + c);
    }
    if (P.nsub == 2) {
        __syncthreads();
        if (lane < H) {
            const int zd = G.z0 + lane;
            const int cb = (w * W) / NWARP, ce = ((w + 1) * W) / NWARP;
#pragma unroll 1
            for (int c = cb; c < ce; ++c) pair_cell<MODE, 1>(P, G, zd, G.x0 + c);
        }
    }
    if (MODE == 0 && P.rec_first != nullptr)
        gather_receivers(P, b, G.S0, G.z0 - 6, G.x0 - 6, GH0, G.S1, G.z0 - 3, G.x0 - 3, GH1);
}

// ---- x-strip tiles (rect type 2): the C-PML x-strips beside a clean run
//
// Rows of a clean run (interior rows away from the free surface and the
// injection rows, float4-aligned), columns of one x-strip.  Every cell of
// the tile and its 3-cell ring has kz = 0; the ring reaches 3 interior
// columns on the strip's inner side.  A thread owns a float4 of rows of one
// column at a time (16 float4 rows of the first step per half-warp, two
// columns per warp), so the C-PML factors and the clamped stencil centres
// are uniform per half-warp and every operand moves as a float4.
constexpr int XZ = 56, XX = 28;              // tile rows (a multiple of 4) and columns at most
constexpr int XQ0 = (XZ + 16) / 4;           // float4 rows of level n (rows from z0-8)
constexpr int XQ1 = (XZ + 8) / 4;            // float4 rows of level n+1 (rows from z0-4)
constexpr int XW0 = XX + 12, XW1 = XX + 6;   // columns of level n (from x0-6) and n+1 (from x0-3)
constexpr int kXStripFloats = 4 * (XQ0 * XW0 + 3 * XQ1 * XW1);
static_assert(kXStripFloats <= kPairFloats, "x-strip tiles fit the launch's shared memory");

__host__ __device__ __forceinline__ void xstrip_bounds(const PairArgs& P, int r, int t, int* z0, int* z1, int* x0,
                                                       int* x1) {
    const int nz = P.r_tz[r], nxr = P.r_tx[r], nq = P.r_h[r] / 4;
    const int tz = t % nz, tx = t / nz;
    *z0 = P.r_zd0[r] + 4 * ((tz * nq) / nz);
    *z1 = P.r_zd0[r] + 4 * (((tz + 1) * nq) / nz);
    *x0 = P.r_x0[r] + (tx * P.r_w[r]) / nxr;
    *x1 = P.r_x0[r] + ((tx + 1) * P.r_w[r]) / nxr;
}

__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void st4(float* p, const float4& v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float4 f4(const float (&v)[4]) { return make_float4(v[0], v[1], v[2], v[3]); }

// One float4 of an x-strip tile at step SUB: rows zd..zd+3 (device), column x.
//   SUB 0: level n from S0 (float4 rows from z0-8, columns from x0-6);
//     phi, chi, p1 at level n from HBM; results into S1 / F1 / X1 (float4
//     rows from z0-4, columns from x0-3) and, on the tile, to the level n+1
//     outputs.
//   SUB 1: level n+1 from S1 / F1 / X1, p1 = level n from S0; results to the
//     level n+2 outputs and over level n in S0.
template <int MODE, int SUB>
__device__ __forceinline__ void xstrip_quad(const PairArgs& P, float4* S0, float4* S1, float4* F1, float4* X1,
                                            int z0, int x0, int x1, int zd, int x, bool inT) {
    const StepArgs& a = P.a;
    const SubStep& s = P.sub[SUB];
    const int dn = a.dn;
    const int kx = (x < dn) ? (dn - x) : (x >= dn + a.nx ? x - (dn + a.nx) + 1 : 0);
    const int cx = clampi(x, 3, a.nxt - 4);
    const float4* SS = SUB == 0 ? S0 : S1;
    const int QS = SUB == 0 ? XQ0 : XQ1;
    const int ox = SUB == 0 ? x0 - 6 : x0 - 3;
    const int rs = SUB == 0 ? (zd - (z0 - 8)) >> 2 : (zd - (z0 - 4)) >> 2;  // float4 row in the source
    const int r1 = (zd - (z0 - 4)) >> 2;                                      // float4 row in S1 / F1 / X1
    float4 W[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) W[k] = SS[(cx - 3 + k - ox) * QS + rs];
    const float4 zc = SS[(x - ox) * QS + rs];
    const float4 zm = SS[(x - ox) * QS + rs - 1];
    const float4 zp = SS[(x - ox) * QS + rs + 1];
    const int g = x * a.ldz + zd;
    const float4 pmv = SUB == 0 ? ld4(a.pm + g) : S0[(x - (x0 - 6)) * XQ0 + ((zd - (z0 - 8)) >> 2)];
    const float4 c2v = ld4(a.c2 + g);
    const float zv[10] = {zm.y, zm.z, zm.w, zc.x, zc.y, zc.z, zc.w, zp.x, zp.y, zp.z};
    float o[4], phn[4], chn[4];
    if (kx > 0) {
        const int sb = (x < dn) ? 0 : dn + a.nx;
        const int ci = clampi(x - sb, 3, dn - 4) + sb;
        float4 F[7];
        float4 phc, chc;
        if (SUB == 0) {
#pragma unroll
            for (int k = 0; k < 7; ++k)
                if (k != 3) F[k] = ld4(a.phix_in + (size_t)(ci - 3 + k) * a.ldz + zd);
            phc = ld4(a.phix_in + g);
            chc = ld4(P.chix_in + g);
        } else {
#pragma unroll
            for (int k = 0; k < 7; ++k)
                if (k != 3) F[k] = F1[(ci - 3 + k - (x0 - 3)) * XQ1 + r1];
            phc = F1[(x - (x0 - 3)) * XQ1 + r1];
            chc = X1[(x - (x0 - 3)) * XQ1 + r1];
        }
        F[3] = make_float4(0.f, 0.f, 0.f, 0.f);
        const float A = __ldg(a.fA + kx - 1), B = __ldg(a.fB + kx - 1);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
#define PXR(k) comp(W[3 + (k)], e)
#define FXR(k) comp(F[3 + (k)], e)
#define ZR(k) zv[3 + e + (k)]
            const float d2x = D2(PXR, a.cf2);
            const float d1x = D1(PXR, a.cf1);
            const float d2y = D2(ZR, a.cf2);
            const float dph = D1(FXR, a.cf1);
#undef PXR
#undef FXR
#undef ZR
            phn[e] = __fadd_rn(__fmul_rn(A, comp(phc, e)), __fmul_rn(B, d1x));
            chn[e] = __fadd_rn(__fmul_rn(A, comp(chc, e)), __fmul_rn(B, __fadd_rn(d2x, dph)));
            const float prop = __fadd_rn(dph, chn[e]);
            const float base = __fadd_rn(-comp(pmv, e), __fmul_rn(2.f, comp(zc, e)));
            o[e] = __fadd_rn(base, __fmul_rn(comp(c2v, e), __fadd_rn(__fadd_rn(d2x, d2y), prop)));
        }
    } else {  // an interior column of the ring: no C-PML term, no injection here
#pragma unroll
        for (int e = 0; e < 4; ++e) {
#define PXR(k) comp(W[3 + (k)], e)
#define ZR(k) zv[3 + e + (k)]
            const float d2x = D2(PXR, a.cf2);
            const float d2y = D2(ZR, a.cf2);
#undef PXR
#undef ZR
            const float base = __fadd_rn(-comp(pmv, e), __fmul_rn(2.f, comp(zc, e)));
            o[e] = __fadd_rn(base, __fmul_rn(comp(c2v, e), __fadd_rn(__fadd_rn(d2x, d2y), 0.f)));
            phn[e] = chn[e] = 0.f;
        }
    }
    const float4 out = f4(o);
    if (SUB == 0) {
        S1[(x - (x0 - 3)) * XQ1 + r1] = out;
        if (kx > 0) {
            F1[(x - (x0 - 3)) * XQ1 + r1] = f4(phn);
            X1[(x - (x0 - 3)) * XQ1 + r1] = f4(chn);
        }
        if (inT) {
            st4(P.p_out[0] + g, out);
            if (P.nsub == 1) {
                st4(a.phix_out + g, f4(phn));
                st4(a.chix + g, f4(chn));
            }
        }
    } else {
        st4(P.p_out[1] + g, out);
        st4(a.phix_out + g, f4(phn));
        st4(a.chix + g, f4(chn));
        S0[(x - (x0 - 6)) * XQ0 + ((zd - (z0 - 8)) >> 2)] = out;
    }
    if (inT && kx == 0) {
        const int fi = (x - dn) * a.ldf + (zd - a.zoff - dn);
#pragma unroll
        for (int e = 0; e < 4; ++e) pair_field<MODE, SUB>(P, fi + e, o[e], comp(pmv, e));
    }
    if (MODE == 0 && inT && s.band != nullptr && kx >= 1 && kx <= 3) {
        const int z = zd - a.zoff;
        float* bp = s.band + (x < dn ? x - (dn - 3) : 3 + x - (dn + a.nx)) * a.ny + (z - dn);
        bp[0] = o[0];
        bp[1] = o[1];
        bp[2] = o[2];
        bp[3] = o[3];
    }
}

template <int MODE>
__device__ __forceinline__ void pair_xstrip_tile(const PairArgs& P, float* sm, int r, int t, int b) {
    const StepArgs& a = P.a;
    int z0, z1, x0, x1;
    xstrip_bounds(P, r, t, &z0, &z1, &x0, &x1);
    float4* S0 = reinterpret_cast<float4*>(sm);
    float4* S1 = S0 + XQ0 * XW0;
    float4* F1 = S1 + XQ1 * XW1;
    float4* X1 = F1 + XQ1 * XW1;
    const int lane = threadIdx.x, w = threadIdx.y, tid = w * 32 + lane;
    const int H = z1 - z0, W = x1 - x0;
    // level n on rows [z0-8, z1+8) x columns [x0-6, x1+6), zero outside the grid
    const int nq0 = H / 4 + 4, W0 = W + 12;
    for (int i = tid; i < nq0 * W0; i += NT) {
        const int c = i / nq0, q = i - c * nq0;
        const int x = x0 - 6 + c;
        S0[c * XQ0 + q] = (x >= 0 && x < a.nxt) ? ld4(a.p + (size_t)x * a.ldz + (z0 - 8) + 4 * q)
                                                 : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    // first step: float4 rows [z0-4, z1+4) (16 per half-warp) x the columns
    // of [x0-3, x1+3) inside the grid, two columns per warp at a time
    const int hq = lane & 15, hc = (w << 1) | (lane >> 4);  // float4 row, column slot 0..7
    const int cl = max(x0 - 3, 0), cr = min(x1 + 3, a.nxt);
    if (hq < H / 4 + 2)
        for (int x = cl + hc; x < cr; x += 2 * NWARP) {
            const int zd = z0 - 4 + 4 * hq;
            const bool inT = hq >= 1 && hq <= H / 4 && x >= x0 && x < x1;
            xstrip_quad<MODE, 0>(P, S0, S1, F1, X1, z0, x0, x1, zd, x, inT);
        }
    if (P.nsub == 2) {
        __syncthreads();
        if (hq < H / 4)
            for (int x = x0 + hc; x < x1; x += 2 * NWARP)
                xstrip_quad<MODE, 1>(P, S0, S1, F1, X1, z0, x0, x1, z0 + 4 * hq, x, true);
    }
    if (MODE == 0 && P.rec_first != nullptr)
        gather_receivers(P, b, reinterpret_cast<float*>(S0), z0 - 8, x0 - 6, 4 * XQ0, reinterpret_cast<float*>(S1),
                         z0 - 4, x0 - 3, 4 * XQ1);
}

// Tile b of a launch; false if its bulk copies did not complete.
template <int MODE>
__device__ __forceinline__ bool pair_tile(const PairArgs& P, float* sm, uint64_t* bar, uint32_t& phase, int b) {
    int r = 0;
    while (r + 1 < P.nrect && b >= P.r_first[r + 1]) ++r;
    const int t = b - P.r_first[r];
    if (P.r_type[r] == 0) return pair_clean_tile<MODE>(P, sm, bar, phase, r, t, b);
    if (P.r_type[r] == 2)
        pair_xstrip_tile<MODE>(P, sm, r, t, b);
    else
        pair_generic_tile<MODE>(P, sm, r, t, b);
    return true;
}

__device__ __forceinline__ void pair_prologue_convert(const PairArgs& P, int tid) {
    const StepArgs& a = P.a;
    if (a.q_src != nullptr) quantize_part(a.q_src, a.q_amax, a.q_dst, a.q_iscale, a.q_n, a.kind16, tid);
    if (P.q_src2 != nullptr) quantize_part(P.q_src2, P.q_amax2, P.q_dst2, P.q_iscale2, P.q_n2, a.kind16, tid);
}

__device__ __forceinline__ void pair_flush_amax(const PairArgs& P) {
    for (int k = 0; k < 2; ++k)
        if (P.sub[k].field_amax != nullptr && s_pair_amax[k] != 0u) atomicMax(P.sub[k].field_amax, s_pair_amax[k]);
    s_pair_amax[0] = s_pair_amax[1] = 0u;
}

// Two steps (or one) of one shot.  Persistent blocks take tiles from this
// launch's counter (clean tiles first); the other counter is cleared for
// the next launch.
template <int MODE>
__global__ void __launch_bounds__(NT, 5) pair_kernel(const PairArgs P) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int tile_id;
    const StepArgs& a = P.a;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    grid_dependency_wait();
    if (tid == 0) {
        mbar_init(&bar, 1);
        s_pair_amax[0] = s_pair_amax[1] = 0u;
    }
    if (MODE == 0) pair_prologue_convert(P, tid);
    if (blockIdx.x == 0 && tid == 0) a.tile_counter[a.counter_sel ^ 1] = 0;
    __syncthreads();
    uint32_t phase = 0;
    const int total = P.r_first[P.nrect];
    for (;;) {
        if (tid == 0) tile_id = atomicAdd(a.tile_counter + a.counter_sel, 1);
        __syncthreads();
        const int b = tile_id;
        if (b >= total) {
            if (MODE == 0 && tid == 0) pair_flush_amax(P);
            return;
        }
        if (!pair_tile<MODE>(P, sm, &bar, phase, b)) return;
        __syncthreads();  // shared tiles and tile_id are reused
    }
}

// Two steps (or one) of several shots in one launch; see PairBatchParams.
// A slot's arguments are copied into shared memory when a block switches
// slot.  FIXED >= 0 is the instance for a launch whose slots are all in
// pass FIXED.
template <int FIXED>
__global__ void __launch_bounds__(NT, 5) pair_batch_kernel(const PairBatchParams bp) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int tile_id;
    __shared__ __align__(16) PairArgs sa;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    grid_dependency_wait();
    if (tid == 0) {
        mbar_init(&bar, 1);
        s_pair_amax[0] = s_pair_amax[1] = 0u;
    }
    for (int s = 0; s < bp.nslots; ++s) {
        if (FIXED > 0 || bp.mode[s] != 0) continue;
        const PairArgs* g = bp.args[s];
        const StepArgs& ga = g->a;
        if (ga.q_src != nullptr) quantize_part(ga.q_src, ga.q_amax, ga.q_dst, ga.q_iscale, ga.q_n, ga.kind16, tid);
        if (g->q_src2 != nullptr)
            quantize_part(g->q_src2, g->q_amax2, g->q_dst2, g->q_iscale2, g->q_n2, ga.kind16, tid);
    }
    if (blockIdx.x == 0 && tid == 0) bp.counter[bp.counter_sel ^ 1] = 0;
    __syncthreads();
    uint32_t phase = 0;
    int cur = -1;
    const int total = bp.first[bp.nslots];
    constexpr int kWords = (int)(sizeof(PairArgs) / sizeof(long long));
    static_assert(sizeof(PairArgs) % sizeof(long long) == 0, "PairArgs is copied in 8-byte words");
    for (;;) {
        if (tid == 0) tile_id = atomicAdd(bp.counter + bp.counter_sel, 1);
        __syncthreads();
        const int b = tile_id;
        if (b >= total) {
            if (tid == 0 && cur >= 0 && bp.mode[cur] == 0) pair_flush_amax(sa);
            return;
        }
        int s = 0;
        while (s + 1 < bp.nslots && b >= bp.first[s + 1]) ++s;
        if (s != cur) {  // every thread takes the same branch
            if (tid == 0 && cur >= 0 && bp.mode[cur] == 0) pair_flush_amax(sa);
            __syncthreads();  // the flush reads sa before it is replaced
            const long long* src = reinterpret_cast<const long long*>(bp.args[s]);
            long long* dst = reinterpret_cast<long long*>(&sa);
            for (int i = tid; i < kWords; i += NT) dst[i] = src[i];
            __syncthreads();
            cur = s;
        }
        const int lb = b - bp.first[s];
        bool ok;
        if (FIXED >= 0) {
            ok = pair_tile<(FIXED >= 0 ? FIXED : 0)>(sa, sm, &bar, phase, lb);
        } else {
            const int md = bp.mode[s];
            ok = md == 0 ? pair_tile<0>(sa, sm, &bar, phase, lb)
                         : (md == 1 ? pair_tile<1>(sa, sm, &bar, phase, lb) : pair_tile<2>(sa, sm, &bar, phase, lb));
        }
        if (!ok) return;
        __syncthreads();  // shared tiles, tile_id and (next switch) sa are reused
    }
}

// Reverse step of the interior: the forward update
// P(L+2) = (-P(L) + 2 P(L+1)) + c2 ((d2x + d2y) + src) solved for P(L) with
// the same c2 term, P(L) = (2 P(L+1) + c2 (...)) - P(L+2); the free-surface
// row stays zero.  One thread per interior cell (rows fastest).
__global__ void reconstruct_kernel(const ReconArgs r) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;  // interior row
    const int i = blockIdx.y;                              // interior column
    if (j >= r.ny || i >= r.nx) return;
    const int z = r.dn + j, x = r.dn + i, zd = z + r.zoff;
    const size_t g = (size_t)x * r.ldz + zd;
    const float p2 = r.pn[g];
    float out = 0.f;
    if (!(r.fs && j == 0)) {
        const float* colc = r.pc + g;
#define AX(k) __ldg(colc + (ptrdiff_t)(k) * r.ldz)
#define AZ(k) __ldg(colc + (k))
        const float d2x = D2(AX, r.cf2);
        const float d2y = D2(AZ, r.cf2);
#undef AX
#undef AZ
        float src = 0.f;
        if (r.row_slot != nullptr) {
            const int rs = __ldg(r.row_slot + zd);
            if (rs >= 0) {
                const int t = __ldg(r.inj_cols + rs * r.nxt + x);
                if (t >= 0) src = __ldg(r.inj_trace + r.inj_t);
            }
        }
        const float b = __fmul_rn(__ldg(r.c2 + g), __fadd_rn(__fadd_rn(d2x, d2y), src));
        out = __fsub_rn(__fadd_rn(__fmul_rn(2.f, __ldg(r.pc + g)), b), p2);
    }
    r.pn[g] = out;
    StepArgs da;  // the division by dt of the snapshots
    da.dt = r.dt;
    da.inv_dt = r.inv_dt;
    da.div_lo = r.div_lo;
    da.div_hi = r.div_hi;
    da.div_tiny = r.div_tiny;
    da.fast_div = r.fast_div;
    r.snap[(size_t)i * r.ldf + j] = div_dt(da, __fmul_rn(__fsub_rn(p2, out), 0.5f));
}

// The saved band of level L into its cells of pn.
__global__ void band_fill_kernel(const ReconArgs r) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nxb = 6 * r.ny;
    if (q >= nxb + 6 * r.nx) return;
    int z, x;
    if (q < nxb) {
        const int col = q / r.ny, j = q - col * r.ny;
        z = r.dn + j;
        x = col < 3 ? r.dn - 3 + col : r.dn + r.nx + (col - 3);
    } else {
        const int u = q - nxb, i = u / 6, row = u - 6 * i;
        x = r.dn + i;
        z = row < 3 ? r.dn + r.ny + row : r.dn - 3 + (row - 3);
        if (r.fs && z < r.dn) return;  // above a free surface: stays zero
    }
    r.pn[(size_t)x * r.ldz + z + r.zoff] = r.band_L[q];
}

constexpr int kPairSmemBytes = kPairFloats * (int)sizeof(float);

template <int MODE>
int pair_blocks_per_sm() {
    static int nb = 0;
    if (nb == 0) {
        cudaFuncSetAttribute(pair_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPairSmemBytes);
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pair_kernel<MODE>, NT, kPairSmemBytes);
        nb = n > 0 ? n : 1;
    }
    return nb;
}

template <int FIXED>
int pair_batch_blocks_per_sm() {
    static int nb = 0;
    if (nb == 0) {
        cudaFuncSetAttribute(pair_batch_kernel<FIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPairSmemBytes);
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pair_batch_kernel<FIXED>, NT, kPairSmemBytes);
        nb = n > 0 ? n : 1;
    }
    return nb;
}

template <class K, class A>
int launch_persistent(K kernel, const A& args, int tiles, int blocks, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(std::min(tiles, blocks));
    cfg.blockDim = dim3(32, NWARP);
    cfg.dynamicSmemBytes = (size_t)kPairSmemBytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelEx(&cfg, kernel, args);
}

}  // namespace

int prepare_pair_kernels() {
    return (pair_blocks_per_sm<0>() > 0 && pair_blocks_per_sm<1>() > 0 && pair_blocks_per_sm<2>() > 0 &&
            pair_batch_blocks_per_sm<-1>() > 0 && pair_batch_blocks_per_sm<0>() > 0 &&
            pair_batch_blocks_per_sm<1>() > 0 && pair_batch_blocks_per_sm<2>() > 0)
               ? (int)cudaGetLastError()
               : 1;
}

int launch_pair(int mode, const PairArgs& P, void* stream) {
    const int tiles = P.r_first[P.nrect];
    if (tiles <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const int sms = P.a.num_sms;
    if (mode == 0) return launch_persistent(pair_kernel<0>, P, tiles, sms * pair_blocks_per_sm<0>(), st);
    if (mode == 1) return launch_persistent(pair_kernel<1>, P, tiles, sms * pair_blocks_per_sm<1>(), st);
    return launch_persistent(pair_kernel<2>, P, tiles, sms * pair_blocks_per_sm<2>(), st);
}

int launch_reconstruct(const ReconArgs& r, void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    reconstruct_kernel<<<dim3((r.ny + 127) / 128, r.nx), 128, 0, st>>>(r);
    const int nb = band_count(r.ny, r.nx);
    band_fill_kernel<<<(nb + 255) / 256, 256, 0, st>>>(r);
    return (int)cudaGetLastError();
}

int launch_pair_batch(const PairBatchParams& bp, int num_sms, void* stream) {
    const int tiles = bp.first[bp.nslots];
    if (bp.nslots <= 0 || tiles <= 0) return 0;
    bool same = true;
    for (int s = 1; s < bp.nslots; ++s) same = same && bp.mode[s] == bp.mode[0];
    cudaStream_t st = (cudaStream_t)stream;
    if (!same) return launch_persistent(pair_batch_kernel<-1>, bp, tiles, num_sms * pair_batch_blocks_per_sm<-1>(), st);
    if (bp.mode[0] == 0)
        return launch_persistent(pair_batch_kernel<0>, bp, tiles, num_sms * pair_batch_blocks_per_sm<0>(), st);
    if (bp.mode[0] == 1)
        return launch_persistent(pair_batch_kernel<1>, bp, tiles, num_sms * pair_batch_blocks_per_sm<1>(), st);
    return launch_persistent(pair_batch_kernel<2>, bp, tiles, num_sms * pair_batch_blocks_per_sm<2>(), st);
}

bool plan_pair(PairArgs* P, const int* row_slot_host) {
    const StepArgs& a = P->a;
    P->txc = TXC;
    const int dn = a.dn, ny = a.ny, nx = a.nx, nyt = a.nyt, nxt = a.nxt, zoff = a.zoff;
    // Clean rows (logical): the tile and its 3-row ring are interior rows,
    // at least 4 rows below a free surface and 4 rows from every row that
    // holds an injection point.
    std::vector<char> ok(nyt, 0);
    for (int z = dn + 3; z < dn + ny - 3; ++z) ok[z] = 1;
    if (a.fs)
        for (int z = dn; z <= dn + 3 && z < nyt; ++z) ok[z] = 0;
    if (row_slot_host)
        for (int zd = 0; zd < a.ldz; ++zd)
            if (row_slot_host[zd] >= 0)
                for (int z = zd - zoff - 3; z <= zd - zoff + 3; ++z)
                    if (z >= 0 && z < nyt) ok[z] = 0;
    const int cx0 = dn + 3, cx1 = dn + nx - 3;
    std::vector<std::pair<int, int>> runs;  // device rows, both ends multiples of 4
    if (cx1 > cx0)
        for (int z = 0; z < nyt;) {
            if (!ok[z]) {
                ++z;
                continue;
            }
            int e = z;
            while (e < nyt && ok[e]) ++e;
            const int ds = (z + zoff + 3) / 4 * 4, de = (e + zoff) / 4 * 4;
            if (de - ds >= 4) runs.push_back({ds, de});
            z = e;
        }
    if (runs.size() > 4) {  // many injection rows: keep the four longest clean runs
        std::sort(runs.begin(), runs.end(),
                  [](const std::pair<int, int>& u, const std::pair<int, int>& v) {
                      return u.second - u.first > v.second - v.first;
                  });
        runs.resize(4);
        std::sort(runs.begin(), runs.end());
    }
    // Band cuts (device rows): live rows, strip edges, clean runs.
    const int top = (a.fs ? dn : 0) + zoff, bot = nyt + zoff;
    std::vector<int> cuts = {top, dn + zoff, dn + ny + zoff, bot};
    for (auto& rn : runs) {
        cuts.push_back(rn.first);
        cuts.push_back(rn.second);
    }
    std::sort(cuts.begin(), cuts.end());
    cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
    int n = 0;
    bool overflow = false;
    P->r_first[0] = 0;
    auto add = [&](int type, int zd0, int x0, int h, int w) {
        if (h <= 0 || w <= 0) return;
        if (n >= kPairRects) {
            overflow = true;
            return;
        }
        P->r_type[n] = type;
        P->r_zd0[n] = zd0;
        P->r_x0[n] = x0;
        P->r_h[n] = h;
        P->r_w[n] = w;
        P->r_tz[n] = type == 0 ? (h + TZC - 1) / TZC : type == 2 ? (h / 4 + XZ / 4 - 1) / (XZ / 4) : (h + GZ - 1) / GZ;
        P->r_tx[n] = type == 0 ? (w + TXC - 1) / TXC : type == 2 ? (w + XX - 1) / XX : (w + GX - 1) / GX;
        P->r_first[n + 1] = P->r_first[n] + P->r_tz[n] * P->r_tx[n];
        ++n;
    };
    for (auto& rn : runs) add(0, rn.first, cx0, rn.second - rn.first, cx1 - cx0);
    for (size_t i = 0; i + 1 < cuts.size(); ++i) {
        const int za = cuts[i], zb = cuts[i + 1];
        if (za < top || zb > bot) continue;
        bool clean = false;
        for (auto& rn : runs) clean = clean || (rn.first == za && rn.second == zb);
        if (clean) {  // the x-strips and the 3 interior columns beside them, float4 tiles
            add(2, za, 0, zb - za, cx0);
            add(2, za, cx1, zb - za, nxt - cx1);
        } else {
            add(1, za, 0, zb - za, dn);
            add(1, za, dn, zb - za, nx);
            add(1, za, dn + nx, zb - za, nxt - (dn + nx));
        }
    }
    P->nrect = n;
    return !overflow;
}

void pair_tile_rect(const PairArgs& P, int b, int* z0, int* z1, int* x0, int* x1) {
    int r = 0;
    while (r + 1 < P.nrect && b >= P.r_first[r + 1]) ++r;
    const int t = b - P.r_first[r];
    if (P.r_type[r] == 0) {
        const int tz = t % P.r_tz[r], tx = t / P.r_tz[r];
        *z0 = P.r_zd0[r] + tz * TZC;
        *x0 = P.r_x0[r] + tx * P.txc;
        *z1 = std::min(*z0 + TZC, P.r_zd0[r] + P.r_h[r]);
        *x1 = std::min(*x0 + P.txc, P.r_x0[r] + P.r_w[r]);
    } else if (P.r_type[r] == 2) {
        xstrip_bounds(P, r, t, z0, z1, x0, x1);
    } else {
        generic_bounds(P, r, t, z0, z1, x0, x1);
    }
}

void pair_rec_lists(const PairArgs& P, int nrec, const int* h_rec_cell, std::vector<int>* first,
                    std::vector<int>* idx) {
    const int n = P.r_first[P.nrect];
    std::vector<std::vector<int>> by(n);
    std::vector<int> R(4 * (size_t)n);
    for (int b = 0; b < n; ++b) pair_tile_rect(P, b, &R[4 * b], &R[4 * b + 1], &R[4 * b + 2], &R[4 * b + 3]);
    for (int i = 0; i < nrec; ++i) {
        const int x = h_rec_cell[i] / P.a.ldz, zd = h_rec_cell[i] % P.a.ldz;
        for (int b = 0; b < n; ++b)
            if (zd >= R[4 * b] && zd < R[4 * b + 1] && x >= R[4 * b + 2] && x < R[4 * b + 3]) {
                by[b].push_back(i);
                break;
            }
    }
    first->assign(n + 1, 0);
    idx->clear();
    for (int b = 0; b < n; ++b) {
        idx->insert(idx->end(), by[b].begin(), by[b].end());
        (*first)[b + 1] = (int)idx->size();
    }
}

}  // namespace psdm
