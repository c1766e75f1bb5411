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
// Work decomposition (see plan_tiles): rectangles of five tile types.
//  * interior tiles, 128 rows x 28 columns (one shot per launch) or 32
//    columns (batched launches) of the interior band: p staged in shared
//    memory with a 4-row / 3-column halo by bulk copies; each thread owns 4
//    consecutive rows (one float4) of 7 or 8 consecutive columns and slides
//    a 7-column float4 window through registers (three 16-byte shared loads
//    per 4 cells, float4 global traffic).
//  * C-PML x-strip, z-strip and corner tiles, and interior rows holding
//    injection points or the free surface (4-row bands), each with its own
//    specialised or generic per-cell update.
// Rows are offset by `zoff` so that the interior starts on a 16-byte
// boundary.  step_kernel runs one step of one shot, batch_step_kernel one
// step of several shots, pass_kernel all steps of one pass (opt-in).
//
// Memory: p1 is overwritten in place with p3; phi is ping-ponged because its
// strip stencil reads neighbours; chi is updated in place.

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <vector>

#include "rtm_device.cuh"
#include "rtm_internal.h"

namespace psdm {
namespace {

// Interior tiles: 128 rows x (4 XS) columns, each thread 4 rows x XS
// columns.  A launch of one shot has fewer tiles than resident blocks and
// gains from narrower tiles (more of them in flight); a batched launch runs
// several waves and gains from wider ones (less halo per cell).
constexpr int QZ = 32;          // float4 rows per interior tile (one warp along z)
constexpr int TZ = 4 * QZ;      // interior tile rows
constexpr int XS_ONE = 7;       // columns per thread, one shot per launch (backward passes)
constexpr int XS_FWD = 6;       // columns per thread, one shot per launch (forward passes)
// Interior tile width of the one-shot kernels of each pass: measured on the
// B200 (config 2), 6 columns make the forward step 3 % faster than 7 (10.7
// against 11.05 us) and the backward step 4 % slower (9.66 against 9.32).
template <int MODE>
__host__ __device__ constexpr int xs_one() { return MODE == 0 ? XS_FWD : XS_ONE; }
constexpr int XS_MANY = 8;      // columns per thread, batched launches
constexpr int HZ = TZ + 8;      // shared rows (16-byte aligned halo of >= 3)
constexpr int HQ = HZ / 4;      // shared float4 rows
__host__ __device__ constexpr int tile_cols(int xs) { return NWARP * xs; }      // interior tile columns
__host__ __device__ constexpr int tile_smem_cols(int xs) { return NWARP * xs + 6; }  // with a 3-column halo
// C-PML / boundary tiles: 32 rows x 16 columns, each thread 1 row x 4 columns.
constexpr int PTZ = 32;
constexpr int PXS = 4;
constexpr int PTX = NWARP * PXS;
constexpr int PHZ = PTZ + 8;
constexpr int PHQ = PHZ / 4;
constexpr int PWX = PTX + 6;
// C-PML x-strip tiles: 128 rows x (4 XXS) columns, each thread 4 rows x XXS
// columns: 2 columns in one-shot forward passes (the forward step 10.7 ->
// 10.5 us on config 2, these tiles ending last), 4 otherwise (with 2 the
// one-shot mixed backward ran 7 %, 8 FP16 shots in flight 3 % and config 4
// up to 22 % slower).
constexpr int XXS_ONE = 2, XXS_MANY = PXS;
template <int MODE, bool BATCHED>
__host__ __device__ constexpr int xxs() { return (!BATCHED && MODE == 0) ? XXS_ONE : XXS_MANY; }
// z-strip tiles: 32 rows x 32 columns (8 columns per thread); row-band
// tiles: 4 rows x 64 columns (2 cells per thread).  Sized so that, with the
// interior and x-strip tiles, a step has about as many tiles as resident
// blocks.
constexpr int ZXS = 8;
constexpr int ZTX = NWARP * ZXS;
constexpr int ZWX = ZTX + 6;
constexpr int RTX = 64;
constexpr int kRing = 3;  // columns of p1 / c2 in flight per thread (RG)

// Stage rows [sz0, sz0+4*hq) x columns [sx0, sx0+wx) of p in shared memory
// (zero outside the array).  sz0 is a multiple of 4.
__device__ __forceinline__ void load_tile_from(const float* src, const StepArgs& a, float* ps, int sz0, int sx0, int hq,
                                               int wx, int tid) {
    for (int q = tid; q < wx * hq; q += NT) {
        const int col = q / hq, r4 = q - col * hq;
        const int gx = sx0 + col, gz = sz0 + 4 * r4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gx >= 0 && gx < a.nxt && gz >= 0 && gz < a.ldz)
            v = *reinterpret_cast<const float4*>(src + gx * a.ldz + gz);
        *reinterpret_cast<float4*>(&ps[col * (4 * hq) + 4 * r4]) = v;
    }
}
__device__ __forceinline__ void load_tile(const StepArgs& a, float* ps, int sz0, int sx0, int hq, int wx, int tid) {
    load_tile_from(a.p, a, ps, sz0, sx0, hq, wx, tid);
}

// Interior tile (rect type 0): rows [zd0, zd0+h) are interior rows without
// injection and without the free-surface row, starting on a 16-byte
// boundary; columns [x0, x0+w) are interior columns.  No stencil centre is
// clamped and no C-PML term applies.  p (with its halo), p1 and c2 of the
// tile are staged in shared memory with bulk asynchronous copies, one per
// column and array, completing on the block's mbarrier; the backward pass
// reads the snapshot slot and the image with 16-byte loads one column ahead.
// Each thread updates 4 rows as two row pairs with the packed FP32x2
// instructions (per-element rounding of the scalar ones); adds that consume
// a product stay scalar so that no multiply-add is ever fused.
// Returns false if the copies did not complete (error reported).
// ST: p1 and c2 of the tile are copied into shared memory with p (batched
// launches, whose operands come from HBM rather than L2: every load of the
// tile is in flight at once), instead of being read one column ahead.
template <int MODE, int XS, bool ST = false, bool RG = false>
__device__ __forceinline__ bool interior_tile(const StepArgs& a, float* sm, uint64_t* bar, uint32_t& phase, int r,
                                              int t) {
    constexpr int TX = tile_cols(XS);
    const int lane = threadIdx.x, wy = threadIdx.y;
    if (a.itx != TX) {  // planned for the other tile width: report, touch nothing
        if (lane == 0 && wy == 0) atomicExch(a.err, 2);
        return false;
    }
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * TZ, x0 = a.r_x0[r] + tx * TX;
    const int nrows = min(TZ, a.r_zd0[r] + a.r_h[r] - z0);  // a multiple of 4
    const int ncols = min(TX, a.r_x0[r] + a.r_w[r] - x0);
    const int sz0 = z0 - 4, sx0 = x0 - 3;
    const int dn = a.dn;
    float* ps = sm;                  // p, (ncols+6) columns of HZ rows
    float* pms = ps + tile_smem_cols(XS) * HZ;  // ST: p1, then c2, ncols columns of TZ rows each
    float* c2s = pms + tile_cols(XS) * TZ;
    if (wy == 0) {
        const uint32_t prow = (uint32_t)(nrows + 8) * 4u, trow = (uint32_t)nrows * 4u;
        const uint32_t bytes = (uint32_t)(ncols + 6) * prow + (ST ? (uint32_t)ncols * trow * 2u : 0u);
        fence_proxy_async();  // the previous tile's shared reads precede these writes
        if (lane == 0) mbar_arrive_expect_tx(bar, bytes);
        __syncwarp();
        for (int c = lane; c < ncols + 6; c += 32)
            bulk_g2s(ps + c * HZ, a.p + (sx0 + c) * a.ldz + sz0, prow, bar);
        if (ST)
            for (int c = lane; c < ncols; c += 32) {
                const int gc = (x0 + c) * a.ldz + z0;
                bulk_g2s(pms + c * TZ, a.pm + gc, trow, bar);
                bulk_g2s(c2s + c * TZ, a.c2 + gc, trow, bar);
            }
    }
    const int q = 4 * lane;        // first tile row of this thread's float4
    const int c0 = wy * XS;        // first tile column of this thread
    const bool active = q < nrows && c0 < ncols;
    const int zd = z0 + q;
    const int z = zd - a.zoff;
    int fi = (x0 + c0 - dn) * a.ldf + (z - dn);
    const bool img = MODE == 1 && a.field != nullptr;
    const bool img16 = MODE == 2 && a.field16 != nullptr;
    const float isc = img16 ? __ldg(a.field_iscale) : 1.f;
    float4 Fn = make_float4(0.f, 0.f, 0.f, 0.f), In = Fn, Cn = Fn;
    if (img && active) {  // first column of the snapshot and image, while the copies land
        Fn = __ldg(reinterpret_cast<const float4*>(a.field + fi));
        In = *reinterpret_cast<const float4*>(a.image + fi);
    }
    uint2 Fr = make_uint2(0u, 0u);  // 16-bit snapshot values, converted where used
    if (img16 && active) {
        Fr = load16x4_raw(a.field16, fi);
        In = *reinterpret_cast<const float4*>(a.image + fi);
        Cn = *reinterpret_cast<const float4*>(a.comp + fi);
    }
    float amax_t = 0.f;
    // p1 and c2 of the first column, from global memory while p lands; later
    // columns are fetched one column ahead.
    float* __restrict__ pmp = a.pm;
    int g = (x0 + c0) * a.ldz + zd;
    float4 pmN = make_float4(0.f, 0.f, 0.f, 0.f), c2N = pmN;
    // RG: this thread's p1 and c2 of the next kRing columns are copied into a
    // ring of shared slots by cp.async, one commit group per column (groups
    // past the last column are empty), so that kRing columns of HBM loads
    // are in flight without holding registers.
    float4* ring = reinterpret_cast<float4*>(sm + tile_smem_cols(XS) * HZ) + (threadIdx.y * 32 + lane);
    if (RG && active) {
#pragma unroll
        for (int k = 0; k < kRing; ++k) {
            if (c0 + k < ncols && k < XS) {
                cp_async16(ring + (2 * k) * NT, pmp + g + k * a.ldz);
                cp_async16(ring + (2 * k + 1) * NT, a.c2 + g + k * a.ldz);
            }
            cp_async_commit();
        }
    } else if (active && !ST) {
        pmN = *reinterpret_cast<const float4*>(pmp + g);
        c2N = __ldg(reinterpret_cast<const float4*>(a.c2 + g));
    }
    const bool ok = mbar_wait_bounded(bar, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0 && threadIdx.y == 0) atomicExch(a.err, 1);
        if (RG) cp_async_wait_all();
        return false;
    }
    if (!active) return true;
    const int ncol = min(XS, ncols - c0);
    const float4* __restrict__ ps4 = reinterpret_cast<const float4*>(ps);
    const int qr = (q + 4) >> 2;   // shared float4 row (halo of 4 rows above)
    float4 win[7];
#pragma unroll
    for (int k = 0; k < 6; ++k) win[k] = ps4[(c0 + k) * HQ + qr];
    float2 cc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) cc[k] = make_float2(a.cf2[k], a.cf2[k]);
    const float2 two = make_float2(2.f, 2.f);
#pragma unroll
    for (int c = 0; c < XS; ++c) {
        if (c >= ncol) break;
        const int col = c0 + c;    // tile column; shared p column is col + 3
        win[6] = ps4[(col + 6) * HQ + qr];
        const float4 zm = ps4[(col + 3) * HQ + qr - 1];
        const float4 zp = ps4[(col + 3) * HQ + qr + 1];
        float4 pmv = pmN, c2v = c2N;
        if (RG) {
            cp_async_wait_group<kRing - 1>();  // column c's copies have landed
            const int sl = c % kRing;
            pmv = ring[(2 * sl) * NT];
            c2v = ring[(2 * sl + 1) * NT];
            if (c + kRing < ncol) {
                cp_async16(ring + (2 * sl) * NT, pmp + g + kRing * a.ldz);
                cp_async16(ring + (2 * sl + 1) * NT, a.c2 + g + kRing * a.ldz);
            }
            cp_async_commit();
        } else if (ST) {
            pmv = *reinterpret_cast<const float4*>(pms + col * TZ + q);
            c2v = *reinterpret_cast<const float4*>(c2s + col * TZ + q);
        } else if (c + 1 < ncol) {
            pmN = *reinterpret_cast<const float4*>(pmp + g + a.ldz);
            c2N = __ldg(reinterpret_cast<const float4*>(a.c2 + g + a.ldz));
        }
        float4 Fc = Fn, Ic = In, Cc = Cn;
        const uint2 Frc = Fr;
        if (img && c + 1 < ncol) {  // next column of the snapshot and image
            Fn = __ldg(reinterpret_cast<const float4*>(a.field + fi + a.ldf));
            In = *reinterpret_cast<const float4*>(a.image + fi + a.ldf);
        }
        if (img16 && c + 1 < ncol) {
            Fr = load16x4_raw(a.field16, fi + a.ldf);
            In = *reinterpret_cast<const float4*>(a.image + fi + a.ldf);
            Cn = *reinterpret_cast<const float4*>(a.comp + fi + a.ldf);
        }
        const float4& pc = win[3];
        // z-window rows -3..+6 around the float4: pairs (i, i+1) of
        // {zm.y, zm.z, zm.w, pc.x, pc.y, pc.z, pc.w, zp.x, zp.y, zp.z}
        const float2 z01 = make_float2(zm.y, zm.z), z12 = make_float2(zm.z, zm.w);
        const float2 z23 = make_float2(zm.w, pc.x), z34 = lo2(pc);
        const float2 z45 = make_float2(pc.y, pc.z), z56 = hi2(pc);
        const float2 z67 = make_float2(pc.w, zp.x), z78 = lo2(zp);
        const float2 z89 = make_float2(zp.y, zp.z);
        // rows 0-1: centre pair z34; rows 2-3: centre pair z56
#define XA(k) lo2(win[3 + (k)])
#define XB(k) hi2(win[3 + (k)])
        const float2 d2xA = D2P(XA, cc);
        const float2 d2xB = D2P(XB, cc);
#undef XA
#undef XB
        const float2 zA[7] = {z01, z12, z23, z34, z45, z56, z67};
        const float2 zB[7] = {z23, z34, z45, z56, z67, z78, z89};
#define ZA(k) zA[3 + (k)]
#define ZB(k) zB[3 + (k)]
        const float2 d2yA = D2P(ZA, cc);
        const float2 d2yB = D2P(ZB, cc);
#undef ZA
#undef ZB
        // -p1 + 2p: 2p is exact, so a fused form would round identically
        const float2 baseA = __fadd2_rn(neg2(lo2(pmv)), __fmul2_rn(two, lo2(pc)));
        const float2 baseB = __fadd2_rn(neg2(hi2(pmv)), __fmul2_rn(two, hi2(pc)));
        const float2 oA = add_prod(baseA, __fmul2_rn(lo2(c2v), __fadd2_rn(d2xA, d2yA)));
        const float2 oB = add_prod(baseB, __fmul2_rn(hi2(c2v), __fadd2_rn(d2xB, d2yB)));
        const float4 out = make_float4(oA.x, oA.y, oB.x, oB.y);
        *reinterpret_cast<float4*>(pmp + g) = out;
        if (MODE == 0 && a.field != nullptr) {
            const float hx = __fmul_rn(__fsub_rn(out.x, pmv.x), 0.5f);
            const float hy = __fmul_rn(__fsub_rn(out.y, pmv.y), 0.5f);
            const float hz = __fmul_rn(__fsub_rn(out.z, pmv.z), 0.5f);
            const float hw = __fmul_rn(__fsub_rn(out.w, pmv.w), 0.5f);
            bool rare = false;
            float4 sv;
            sv.x = div_dt_common(a, hx, rare);
            sv.y = div_dt_common(a, hy, rare);
            sv.z = div_dt_common(a, hz, rare);
            sv.w = div_dt_common(a, hw, rare);
            if (__any_sync(__activemask(), rare) && rare) {
                sv.x = div_dt(a, hx);
                sv.y = div_dt(a, hy);
                sv.z = div_dt(a, hz);
                sv.w = div_dt(a, hw);
            }
            *reinterpret_cast<float4*>(a.field + fi) = sv;
            if (a.field_amax != nullptr)
                amax_t = fmaxf(amax_t, fmaxf(fmaxf(fabsf(sv.x), fabsf(sv.y)), fmaxf(fabsf(sv.z), fabsf(sv.w))));
        }
        if (MODE == 2 && img16) {
            Fc = unpack16x4(Frc, a.kind16, isc);
            float Fv[4] = {Fc.x, Fc.y, Fc.z, Fc.w};
            float Iv[4] = {Ic.x, Ic.y, Ic.z, Ic.w};
            float Cv[4] = {Cc.x, Cc.y, Cc.z, Cc.w};
            const float ov[4] = {out.x, out.y, out.z, out.w};
            const float pv[4] = {pmv.x, pmv.y, pmv.z, pmv.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                float F = Fv[e];
                if (a.field_w != 1.f) F = __fmul_rn(F, a.field_w);
                float inc = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(ov[e], pv[e])), F);
                if (a.ss != 1.f) inc = __fmul_rn(inc, a.ss);
                kahan(Iv[e], Cv[e], inc);
            }
            *reinterpret_cast<float4*>(a.image + fi) = make_float4(Iv[0], Iv[1], Iv[2], Iv[3]);
            *reinterpret_cast<float4*>(a.comp + fi) = make_float4(Cv[0], Cv[1], Cv[2], Cv[3]);
        }
        if (MODE == 1 && img) {
            if (a.field_w != 1.f) {
                Fc.x = __fmul_rn(Fc.x, a.field_w); Fc.y = __fmul_rn(Fc.y, a.field_w);
                Fc.z = __fmul_rn(Fc.z, a.field_w); Fc.w = __fmul_rn(Fc.w, a.field_w);
            }
            const float2 half = make_float2(0.5f, 0.5f);
            float2 iA = __fmul2_rn(__fmul2_rn(half, __fadd2_rn(oA, neg2(lo2(pmv)))), lo2(Fc));
            float2 iB = __fmul2_rn(__fmul2_rn(half, __fadd2_rn(oB, neg2(hi2(pmv)))), hi2(Fc));
            if (a.ss != 1.f) {
                const float2 ss = make_float2(a.ss, a.ss);
                iA = __fmul2_rn(iA, ss);
                iB = __fmul2_rn(iB, ss);
            }
            const float2 rA = add_prod(lo2(Ic), iA), rB = add_prod(hi2(Ic), iB);
            *reinterpret_cast<float4*>(a.image + fi) = make_float4(rA.x, rA.y, rB.x, rB.y);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) win[k] = win[k + 1];
        g += a.ldz;
        fi += a.ldf;
    }
    if (RG) cp_async_wait_all();  // the ring is reused by the next tile
    if (MODE == 0 && a.field_amax != nullptr && a.field != nullptr) amax_note(amax_t);
    return true;
}

// Interior rows that carry the free surface or injection points (rect type
// 4): 4 rows x 64 columns per tile, generic cells, 2 per thread.
template <int MODE>
__device__ __forceinline__ void rowband_tile(const StepArgs& a, float* ps, int r, int t) {
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * 4, x0 = a.r_x0[r] + tx * RTX;
    const int zend = a.r_zd0[r] + a.r_h[r], xend = a.r_x0[r] + a.r_w[r];
    const int sz0 = z0 - 4, sx0 = x0 - 3;  // interior rows and columns: no clamping
    load_tile(a, ps, sz0, sx0, 3, RTX + 6, tid);
    __syncthreads();
    const int zd = z0 + (tid & 3);
    if (zd >= zend) return;
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
        const int x = x0 + (tid >> 2) + 32 * h;
        if (x < xend) cell_generic<MODE, 12>(a, ps, sz0, sx0, zd, x);
    }
}

// C-PML x-strip over the interior band rows (rect type 1): rows are interior
// rows (kz = 0, no row clamping), columns x-PML columns.  Each thread owns 4
// rows (one float4) of XXS columns; the C-PML factor, the clamped stencil
// centre cx and the strip-local phi centre are uniform per column.
template <int MODE, int XXS>
__device__ __forceinline__ bool xband_tile(const StepArgs& a, float* ps, int r, int t) {
    constexpr int XTX = NWARP * XXS;  // the plan's a.ixb (checked on the host before a launch)
    const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * TZ, x0 = a.r_x0[r] + tx * XTX;
    const int zend = a.r_zd0[r] + a.r_h[r], xend = a.r_x0[r] + a.r_w[r];
    const int sz0 = z0 - 4;
    const int sx0 = min(x0, a.nxt - 4) - 3;
    load_tile(a, ps, sz0, sx0, HQ, XTX + 6, tid);
    __syncthreads();
    const int zd = z0 + 4 * lane;
    if (zd >= zend) return true;
    const int dn = a.dn;
    const int z = zd - a.zoff;
    const bool fsq = a.fs && z == dn;
    const float4* __restrict__ ps4 = reinterpret_cast<const float4*>(ps);
    const int qr = (zd - sz0) >> 2;
#pragma unroll 1
    for (int c = 0; c < XXS; ++c) {
        const int x = x0 + wy * XXS + c;
        if (x >= xend) break;
        XbandIn in;
        xband_load(a, zd, x, true, in);
        xband_compute<HQ>(a, ps4, nullptr, sx0, qr, zd, fsq, x, in);
    }
    return true;
}

// C-PML z-strip over interior columns (rect type 2): kx = 0.  Rows with
// kz > 0 run a specialised update; interior rows of a partial float4 at the
// bottom of the band fall back to the generic cell.  PF: each thread loads
// the next column's global inputs while it updates the current one (the
// one-shot FP32 step kernels, where these tiles end last; the mixed-precision,
// batched and pass kernels keep the plain loop, whose lower register demand
// suits them).
template <int MODE, bool PF = false>
__device__ __forceinline__ void zstrip_tile(const StepArgs& a, float* ps, int r, int t) {
    const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * PTZ, x0 = a.r_x0[r] + tx * ZTX;
    const int zend = a.r_zd0[r] + a.r_h[r], xend = a.r_x0[r] + a.r_w[r];
    const int nr = a.zoff + a.nyt;
    const int sz0 = (min(z0, nr - 4) - 3) & ~3;
    const int sx0 = x0 - 3;  // interior columns: no clamping along x
    load_tile(a, ps, sz0, sx0, PHQ, ZWX, tid);
    __syncthreads();
    const int zd = z0 + lane;
    if (zd >= zend) return;
    const int dn = a.dn;
    const int z = zd - a.zoff;
    if (z < 0 || z >= a.nyt) return;
    const int kz = (z < dn) ? (dn - z) : (z >= dn + a.ny ? z - (dn + a.ny) + 1 : 0);
    if (kz == 0) {
#pragma unroll 1
        for (int c = 0; c < ZXS; ++c) {
            const int x = x0 + wy * ZXS + c;
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
    if constexpr (!PF) {
    #pragma unroll 1
        for (int c = 0; c < ZXS; ++c) {
            const int x = x0 + wy * ZXS + c;
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
            const float* phs = a.phiz_in + x * a.ldz;
    #define PZ(k) phs[cj + (k)]
            const float dph = D1(PZ, c1);
    #undef PZ
    #undef AZ
            const float phn = __fadd_rn(__fmul_rn(A, phs[zd]), __fmul_rn(B, d1));
            const float chn = __fadd_rn(__fmul_rn(A, a.chiz[g]), __fmul_rn(B, __fadd_rn(d2y, dph)));
            a.phiz_out[g] = phn;
            a.chiz[g] = chn;
            const float prop = __fadd_rn(dph, chn);
            const float base = __fadd_rn(-a.pm[g], __fmul_rn(2.f, colc[0]));
            a.pm[g] = __fadd_rn(base, __fmul_rn(__ldg(a.c2 + g), __fadd_rn(__fadd_rn(d2x, d2y), prop)));
        }
        return;
    }
    // global inputs of one column: phi_z around the strip-local centre cj,
    // phi_z, chi_z, level n-1 and c2 of the cell; the next column's are in
    // flight during this column's update
    struct ZIn { float f[7], ph, ch, pm, c2; };
    auto zload = [&](int x, ZIn& v) {
        const float* phs = a.phiz_in + x * a.ldz;
#pragma unroll
        for (int k = 0; k < 7; ++k)
            if (k != 3) v.f[k] = phs[cj + k - 3];
        const int g = x * a.ldz + zd;
        v.ph = phs[zd];
        v.ch = a.chiz[g];
        v.pm = a.pm[g];
        v.c2 = __ldg(a.c2 + g);
    };
    const int xb = x0 + wy * ZXS, xe = min(xb + ZXS, xend);
    if (xb >= xe) return;
    ZIn cur, nxt;
    zload(xb, cur);
#pragma unroll 1
    for (int x = xb; x < xe; ++x) {
        if (x + 1 < xe) zload(x + 1, nxt);
        const int xl = x - sx0;
        const float* colc = ps + xl * PHZ + zl;
        const float* colz = ps + xl * PHZ + czl;
#define AX(k) colc[(k) * PHZ]
#define AZ(k) colz[(k)]
        const float d2x = D2(AX, c2);
        const float d2y = D2(AZ, c2);
        const float d1 = D1(AZ, c1);
#undef AX
#undef AZ
        const int g = x * a.ldz + zd;
#define PZ(k) cur.f[3 + (k)]
        const float dph = D1(PZ, c1);
#undef PZ
        const float phn = __fadd_rn(__fmul_rn(A, cur.ph), __fmul_rn(B, d1));
        const float chn = __fadd_rn(__fmul_rn(A, cur.ch), __fmul_rn(B, __fadd_rn(d2y, dph)));
        a.phiz_out[g] = phn;
        a.chiz[g] = chn;
        const float prop = __fadd_rn(dph, chn);
        const float base = __fadd_rn(-cur.pm, __fmul_rn(2.f, colc[0]));
        a.pm[g] = __fadd_rn(base, __fmul_rn(cur.c2, __fadd_rn(__fadd_rn(d2x, d2y), prop)));
        cur = nxt;
    }
}

// The z-strip tile with every global input of its C-PML cells staged in
// shared memory before the update (one-shot FP32 launches): phi_z over the
// p tile's 40-row window (the strip-local stencils of the tile's rows lie in
// it, as the clamped p stencils do), chi_z, level n-1 and c2 over the tile's
// 32 rows, all issued as 16-byte cp.async copies together with the p tile's
// loads, so that a thread's columns wait for one round trip instead of one
// per column.  The arithmetic is zstrip_tile's, in its order.
#ifndef PSDM_ZSTRIP_STAGE
#define PSDM_ZSTRIP_STAGE 1
#endif
constexpr bool kZstripStage = PSDM_ZSTRIP_STAGE != 0;
constexpr int kZsFloats = ZWX * PHZ + ZTX * PHZ + 3 * ZTX * PTZ;
template <int MODE>
__device__ __forceinline__ void zstrip_tile_staged(const StepArgs& a, float* ps, int r, int t) {
    const int lane = threadIdx.x, wy = threadIdx.y, tid = wy * 32 + lane;
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    const int z0 = a.r_zd0[r] + tz * PTZ, x0 = a.r_x0[r] + tx * ZTX;
    const int zend = a.r_zd0[r] + a.r_h[r], xend = a.r_x0[r] + a.r_w[r];
    const int nr = a.zoff + a.nyt;
    const int sz0 = (min(z0, nr - 4) - 3) & ~3;
    const int sx0 = x0 - 3;  // interior columns: no clamping along x
    float* fs = ps + ZWX * PHZ;   // phi_z, ZTX columns of PHZ rows from sz0
    float* cs = fs + ZTX * PHZ;   // chi_z, ZTX columns of PTZ rows from z0
    float* ms = cs + ZTX * PTZ;   // level n-1
    float* c2s = ms + ZTX * PTZ;  // c2
    // phi_z window (PHZ / 4 float4 per column) and the three tile arrays
    // (PTZ / 4 each); z0 and sz0 are multiples of 4
    constexpr int kF4 = PHZ / 4, kT4 = PTZ / 4;
    for (int q = tid; q < ZTX * (kF4 + 3 * kT4); q += NT) {
        int col, arr, r4;
        if (q < ZTX * kF4) {
            col = q / kF4;
            r4 = q - col * kF4;
            arr = 0;
        } else {
            const int u = q - ZTX * kF4;
            arr = 1 + u / (ZTX * kT4);
            const int v = u - (arr - 1) * ZTX * kT4;
            col = v / kT4;
            r4 = v - col * kT4;
        }
        const int x = x0 + col;
        const int row = (arr == 0 ? sz0 : z0) + 4 * r4;
        if (x >= xend || row < 0 || row + 4 > a.ldz) continue;
        const size_t gsrc = (size_t)x * a.ldz + row;
        if (arr == 0) cp_async16(fs + col * PHZ + 4 * r4, a.phiz_in + gsrc);
        else if (arr == 1) cp_async16(cs + col * PTZ + 4 * r4, a.chiz + gsrc);
        else if (arr == 2) cp_async16(ms + col * PTZ + 4 * r4, a.pm + gsrc);
        else cp_async16(c2s + col * PTZ + 4 * r4, a.c2 + gsrc);
    }
    cp_async_commit();
    load_tile(a, ps, sz0, sx0, PHQ, ZWX, tid);
    cp_async_wait_all();
    __syncthreads();
    const int zd = z0 + lane;
    if (zd >= zend) return;
    const int dn = a.dn;
    const int z = zd - a.zoff;
    if (z < 0 || z >= a.nyt) return;
    const int kz = (z < dn) ? (dn - z) : (z >= dn + a.ny ? z - (dn + a.ny) + 1 : 0);
    if (kz == 0) {
#pragma unroll 1
        for (int c = 0; c < ZXS; ++c) {
            const int x = x0 + wy * ZXS + c;
            if (x >= xend) break;
            cell_generic<MODE, PHZ>(a, ps, sz0, sx0, zd, x);
        }
        return;
    }
    const float A = __ldg(a.fA + kz - 1), B = __ldg(a.fB + kz - 1);
    const int zl = zd - sz0;
    const int czl = clampi(z, 3, a.nyt - 4) + a.zoff - sz0;
    const int sb = (z < dn) ? 0 : dn + a.ny;
    const int cjl = clampi(z - sb, 3, dn - 4) + sb + a.zoff - sz0;  // phi_z stencil centre in the window
    const int tl = zd - z0;                                          // row in the tile arrays
    const float* c1 = a.cf1;
    const float* c2 = a.cf2;
#pragma unroll 1
    for (int c = 0; c < ZXS; ++c) {
        const int cl = wy * ZXS + c;  // tile column
        const int x = x0 + cl;
        if (x >= xend) break;
        const int xl = x - sx0;
        const float* colc = ps + xl * PHZ + zl;
        const float* colz = ps + xl * PHZ + czl;
        const float* phs = fs + cl * PHZ;
#define AX(k) colc[(k) * PHZ]
#define AZ(k) colz[(k)]
#define PZ(k) phs[cjl + (k)]
        const float d2x = D2(AX, c2);
        const float d2y = D2(AZ, c2);
        const float d1 = D1(AZ, c1);
        const float dph = D1(PZ, c1);
#undef AX
#undef AZ
#undef PZ
        const int g = x * a.ldz + zd;
        const float phn = __fadd_rn(__fmul_rn(A, phs[zl]), __fmul_rn(B, d1));
        const float chn = __fadd_rn(__fmul_rn(A, cs[cl * PTZ + tl]), __fmul_rn(B, __fadd_rn(d2y, dph)));
        a.phiz_out[g] = phn;
        a.chiz[g] = chn;
        const float prop = __fadd_rn(dph, chn);
        const float base = __fadd_rn(-ms[cl * PTZ + tl], __fmul_rn(2.f, colc[0]));
        a.pm[g] = __fadd_rn(base, __fmul_rn(c2s[cl * PTZ + tl], __fadd_rn(__fadd_rn(d2x, d2y), prop)));
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

template <int XS>
constexpr int smem_floats() {
    return tile_smem_cols(XS) * HZ;  // the p tile of an interior tile (boundary tiles use less)
}

template <int MODE>
__global__ void __launch_bounds__(NT, 5) step_kernel(const StepArgs a) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int tile_id;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    grid_dependency_wait();
    if (tid == 0) {
        mbar_init(&bar, 1);
        s_blk_amax = 0u;
    }
    // Receivers of the previous step (p is that step's p3, read-only during
    // this step): spread over the blocks, a receiver per thread, loaded before
    // the tiles and stored after them so that the load's latency overlaps the
    // tiles' work.
    int rec_i = -1;
    float rec_v = 0.f;
    if (MODE == 0 && a.rec_t >= 0) {
        if (a.nrec <= (int)gridDim.x * NT) {
            const int i = blockIdx.x + (int)gridDim.x * tid;
            if (i < a.nrec) {
                rec_i = i;
                rec_v = a.p[a.rec_cell[i]];
            }
        } else {
            for (int i = blockIdx.x * NT + tid; i < a.nrec; i += gridDim.x * NT)
                a.rec_out[(size_t)i * a.rec_ld + a.rec_t] = a.p[a.rec_cell[i]];
        }
    }
    if (MODE == 0 && a.q_src != nullptr) quantize_part(a.q_src, a.q_amax, a.q_dst, a.q_iscale, a.q_n, a.kind16, tid);
    // Persistent blocks take tiles in order (heaviest rect types first) from
    // this step's counter; the other counter is cleared for the next step.
    if (blockIdx.x == 0 && tid == 0) a.tile_counter[a.counter_sel ^ 1] = 0;
    __syncthreads();
    uint32_t phase = 0;
    const int total = a.r_first[a.nrect];
    for (;;) {
        if (tid == 0) tile_id = atomicAdd(a.tile_counter + a.counter_sel, 1);
        __syncthreads();
        const int b = tile_id;
        if (b >= total) {
            if (MODE == 0 && tid == 0 && a.field_amax != nullptr && s_blk_amax != 0u)
                atomicMax(a.field_amax, s_blk_amax);
            if (MODE == 0 && rec_i >= 0) a.rec_out[(size_t)rec_i * a.rec_ld + a.rec_t] = rec_v;
            return;
        }
        int r = 0;
        while (r + 1 < a.nrect && b >= a.r_first[r + 1]) ++r;
        const int t = b - a.r_first[r];
        switch (a.r_type[r]) {
            case 0:
                if (!interior_tile<MODE, xs_one<MODE>()>(a, sm, &bar, phase, r, t)) return;
                break;
            case 1:
                if (!xband_tile<MODE, xxs<MODE, false>()>(a, sm, r, t)) return;
                break;
            case 2:
                if (kZstripStage && MODE != 2) zstrip_tile_staged<MODE>(a, sm, r, t);
                else zstrip_tile<MODE, MODE != 2>(a, sm, r, t);
                break;
            case 4: rowband_tile<MODE>(a, sm, r, t); break;
            default: generic_tile<MODE>(a, sm, r, t); break;
        }
        __syncthreads();  // shared tile and tile_id are reused
    }
}

// One tile (block-local index b of the step described by `a`).  Returns
// false if its bulk copies did not complete.
#ifndef PSDM_BATCH_STAGE
#define PSDM_BATCH_STAGE 0
#endif
// With PSDM_BATCH_STAGE=1, batched launches stage p1 and c2 of interior tiles
// with p.  Off by default: the 52 KB tile leaves 4 blocks per SM instead of 5,
// and on the B200 8 FP16 shots in flight ran at 5.73 against 6.32 shots/s
// without it (config 4: 3.62 against 4.66).
constexpr bool kBatchStage = PSDM_BATCH_STAGE != 0;
// Batched launches whose slots are all in one pass, whose interior operands
// come from HBM, prefetch p1 and c2 kRing columns ahead through a shared ring
// (interior_tile's RG): 8 FP16 shots in flight ran at 6.75 against 6.33
// shots/s without it on the B200.  The instance for slots in different
// passes keeps one column ahead in registers (with the ring config 4 ran at
// 3.3-3.8 against 4.2-4.5 shots/s).
#ifndef PSDM_BATCH_RING
#define PSDM_BATCH_RING 1
#endif
constexpr bool kBatchRing = PSDM_BATCH_RING != 0 && !kBatchStage;
constexpr int batch_smem_floats() {
    return smem_floats<XS_MANY>() + (kBatchStage ? 2 * TZ * tile_cols(XS_MANY) : 0) +
           (kBatchRing ? 4 * 2 * kRing * NT : 0);
}

template <int MODE, int XS = XS_MANY, bool ST = (XS == XS_MANY && kBatchStage),
          bool RG = (XS == XS_MANY && kBatchRing)>
__device__ __forceinline__ bool run_tile(const StepArgs& a, float* sm, uint64_t* bar, uint32_t& phase, int b) {
    int r = 0;
    while (r + 1 < a.nrect && b >= a.r_first[r + 1]) ++r;
    const int t = b - a.r_first[r];
    switch (a.r_type[r]) {
        case 0: return interior_tile<MODE, XS, ST, RG>(a, sm, bar, phase, r, t);
        case 1: return xband_tile<MODE, xxs<MODE, XS == XS_MANY>()>(a, sm, r, t);
        case 2: zstrip_tile<MODE>(a, sm, r, t); return true;
        case 4: rowband_tile<MODE>(a, sm, r, t); return true;
        default: generic_tile<MODE>(a, sm, r, t); return true;
    }
}

// One time step of several shots (slots) in one launch.  The tiles of all
// slots form one work list, slot s owning tiles [first[s], first[s+1]);
// persistent blocks take tiles from one counter, so a block moves on to the
// next slot's tiles while others are still waiting for their copies, and a
// step of many shots fills the GPU in several waves.  Each slot's step
// arguments live in device memory; a block copies them into shared memory
// when it switches slot.  Slots may be in different passes (mode 0 / 1 / 2);
// FIXED >= 0 is the instance for a launch whose slots are all in pass FIXED,
// compiled without the other passes' code (fewer registers and spills).
template <int FIXED>
__global__ void __launch_bounds__(NT, 5) batch_step_kernel(const BatchParams bp) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int tile_id;
    __shared__ __align__(16) StepArgs sa;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    grid_dependency_wait();
    if (tid == 0) {
        mbar_init(&bar, 1);
        s_blk_amax = 0u;
    }
    // Deferred receiver gathers of the forward slots (p = previous step's p3),
    // and their pending snapshot quantizations.
    for (int s = 0; s < bp.nslots; ++s) {
        if (FIXED > 0 || bp.mode[s] != 0) continue;
        const StepArgs* g = bp.args[s];
        const float* qs = g->q_src;
        if (qs != nullptr) quantize_part(qs, g->q_amax, g->q_dst, g->q_iscale, g->q_n, g->kind16, tid);
        const int rec_t = g->rec_t, nrec = g->nrec;
        if (rec_t < 0 || nrec <= 0) continue;
        const float* p = g->p;
        const int* cell = g->rec_cell;
        float* out = g->rec_out;
        const int ld = g->rec_ld;
        for (int i = blockIdx.x * NT + tid; i < nrec; i += gridDim.x * NT)
            out[(size_t)i * ld + rec_t] = p[cell[i]];
    }
    if (blockIdx.x == 0 && tid == 0) bp.counter[bp.counter_sel ^ 1] = 0;
    __syncthreads();
    uint32_t phase = 0;
    int cur = -1;
    const int total = bp.first[bp.nslots];
    constexpr int kWords = (int)(sizeof(StepArgs) / sizeof(long long));
    static_assert(sizeof(StepArgs) % sizeof(long long) == 0, "StepArgs is copied in 8-byte words");
    for (;;) {
        if (tid == 0) tile_id = atomicAdd(bp.counter + bp.counter_sel, 1);
        __syncthreads();
        const int b = tile_id;
        if (b >= total) {
            if (tid == 0 && cur >= 0 && bp.mode[cur] == 0 && sa.field_amax != nullptr && s_blk_amax != 0u)
                atomicMax(sa.field_amax, s_blk_amax);
            return;
        }
        int s = 0;
        while (s + 1 < bp.nslots && b >= bp.first[s + 1]) ++s;
        if (s != cur) {  // every thread takes the same branch
            if (tid == 0 && cur >= 0 && bp.mode[cur] == 0 && sa.field_amax != nullptr && s_blk_amax != 0u)
                atomicMax(sa.field_amax, s_blk_amax);
            __syncthreads();  // the flush reads sa before it is replaced
            if (tid == 0) s_blk_amax = 0u;
            const long long* src = reinterpret_cast<const long long*>(bp.args[s]);
            long long* dst = reinterpret_cast<long long*>(&sa);
            for (int i = tid; i < kWords; i += NT) dst[i] = src[i];
            __syncthreads();
            cur = s;
        }
        const int lb = b - bp.first[s];
        bool ok;
        if (FIXED >= 0) {
            ok = run_tile<(FIXED >= 0 ? FIXED : 0)>(sa, sm, &bar, phase, lb);
        } else {
            // slots in different passes: no p1/c2 ring (measured slower in this instance)
            const int md = bp.mode[s];
            ok = md == 0 ? run_tile<0, XS_MANY, kBatchStage, false>(sa, sm, &bar, phase, lb)
                         : (md == 1 ? run_tile<1, XS_MANY, kBatchStage, false>(sa, sm, &bar, phase, lb)
                                    : run_tile<2, XS_MANY, kBatchStage, false>(sa, sm, &bar, phase, lb));
        }
        if (!ok) return;
        __syncthreads();  // shared tile, tile_id and (next switch) sa are reused
    }
}

// ---- one launch per pass (dataflow form)

// All steps of one pass.  Block b owns tiles b, b + gridDim.x, ...; before
// step i of a tile it waits until each neighbour tile has completed i steps
// (the neighbours wrote the p, phi and side values this step reads, and
// have read the values this step overwrites), and after it publishes i + 1.
// Receivers are gathered at the start of a step by the owner of their cell,
// from p = the previous step's p3, like step_kernel does.  All blocks must be
// resident at once (cooperative launch).
template <int MODE>
__global__ void __launch_bounds__(NT, 5) pass_kernel(const PassParams pp) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ __align__(16) StepArgs sb[2];
    __shared__ __align__(16) PassVar sv[2];
    const int tid = threadIdx.y * 32 + threadIdx.x;
    constexpr int kWords = (int)(sizeof(StepArgs) / sizeof(long long));
    constexpr int kVar16 = (int)(sizeof(PassVar) / 16);
    if (tid == 0) mbar_init(&bar, 1);
    for (int w = tid; w < 2 * kWords; w += NT)
        reinterpret_cast<long long*>(sb)[w] = reinterpret_cast<const long long*>(pp.base)[w];
    if (tid == 0 && pp.nsteps > 0) {
        for (int q = 0; q < kVar16; ++q)
            cp_async16(reinterpret_cast<char*>(&sv[0]) + 16 * q, reinterpret_cast<const char*>(pp.var) + 16 * q);
        cp_async_commit();
    }
    __syncthreads();
    uint32_t phase = 0;
    for (int i = 0; i < pp.nsteps; ++i) {
        const int par = i & 1;
        if (tid == 0) {
            cp_async_wait_all();  // values of step i
            const PassVar& v = sv[par];
            StepArgs& t = sb[par];
            t.field = v.field;
            t.field16 = v.field16;
            t.field_iscale = v.field_iscale;
            t.field_w = v.field_w;
            t.inj_t = v.inj_t;
            t.rec_t = v.rec_t;
            if (i + 1 < pp.nsteps) {
                const char* src = reinterpret_cast<const char*>(pp.var + i + 1);
                for (int q = 0; q < kVar16; ++q)
                    cp_async16(reinterpret_cast<char*>(&sv[par ^ 1]) + 16 * q, src + 16 * q);
                cp_async_commit();
            }
        }
        __syncthreads();
        const StepArgs& a = sb[par];
        if (MODE == 0 && a.rec_t >= 0) {  // own cells, written by this block in the previous step
            for (int T = blockIdx.x; T < pp.ntiles; T += gridDim.x)
                for (int j = pp.rec_first[T] + tid; j < pp.rec_first[T + 1]; j += NT) {
                    const int r = pp.rec_idx[j];
                    a.rec_out[(size_t)r * a.rec_ld + a.rec_t] = a.p[a.rec_cell[r]];
                }
        }
        for (int T = blockIdx.x; T < pp.ntiles; T += gridDim.x) {
            bool ok = true;
            for (int k = pp.nbr_first[T] + tid; k < pp.nbr_first[T + 1]; k += NT)
                ok = wait_flag(pp.flags + pp.nbr[k], i, pp.abort) && ok;
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicExch(pp.abort, 1);
                    atomicCAS(pp.err, 0, 3);
                    cp_async_wait_all();
                }
                return;
            }
            if (threadIdx.y == 0) fence_proxy_async_global();  // warp 0 issues the tile's bulk copies
            if (!run_tile<MODE, xs_one<MODE>()>(a, sm, &bar, phase, T)) {
                if (tid == 0) {
                    atomicExch(pp.abort, 1);
                    atomicCAS(pp.err, 0, 1);
                    cp_async_wait_all();
                }
                return;
            }
            __syncthreads();  // the tile's writes precede the publication; shared tile reused
            if (tid == 0) st_release(pp.flags + T, i + 1);  // cumulative over the block's writes
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

void plan_tiles(StepArgs* a, const int* row_slot_host, bool batched, bool forward) {
    const int TX = tile_cols(batched ? XS_MANY : (forward ? XS_FWD : XS_ONE));
    a->itx = TX;
    a->ixb = NWARP * ((!batched && forward) ? XXS_ONE : XXS_MANY);
    // Rects of the padded grid (device rows), heaviest first:
    //   type 0  interior band rows without injection / free surface
    //   type 1  x-strip band   rows [d0, d0+ny4) x C-PML columns
    //   type 2  z-strips       rows below the band (and above it without a free
    //                          surface) x interior columns
    //   type 4  interior band rows with injection points or the free surface
    //   type 3  corners        the remaining rows x C-PML columns
    // d0 = first interior row (a multiple of 4), ny4 = ny rounded down to 4.
    const int dn = a->dn, nr = a->zoff + a->nyt;
    const int d0 = dn + a->zoff;
    const int ny4 = a->ny & ~3;
    const int nq = ny4 / 4;
    // special float4 rows of the band
    std::vector<char> special(nq, 0);
    if (a->fs && nq > 0) special[0] = 1;
    if (row_slot_host)
        for (int q = 0; q < nq; ++q)
            for (int k = 0; k < 4; ++k)
                if (row_slot_host[d0 + 4 * q + k] >= 0) special[q] = 1;
    // runs of equal kind; too many runs: one special run spanning them all
    std::vector<std::pair<int, int>> runs;  // (start quad, kind) boundaries
    for (int q = 0; q < nq; ++q)
        if (q == 0 || special[q] != special[q - 1]) runs.push_back({q, special[q]});
    int nspecial = 0;
    for (auto& rn : runs) nspecial += rn.second;
    if (nspecial > 3) {
        int first = -1, last = -1;
        for (int q = 0; q < nq; ++q)
            if (special[q]) { if (first < 0) first = q; last = q; }
        for (int q = first; q <= last; ++q) special[q] = 1;
        runs.clear();
        for (int q = 0; q < nq; ++q)
            if (q == 0 || special[q] != special[q - 1]) runs.push_back({q, special[q]});
    }
    int n = 0;
    a->r_first[0] = 0;
    auto add = [&](int type, int zd0, int x0, int h, int w) {
        if (h <= 0 || w <= 0) return;
        const int tzsz = (type == 0 || type == 1) ? TZ : (type == 4 ? 4 : PTZ);
        const int txsz = type == 0 ? TX : (type == 4 ? RTX : (type == 2 ? ZTX : (type == 1 ? a->ixb : PTX)));
        a->r_type[n] = type;
        a->r_zd0[n] = zd0; a->r_x0[n] = x0; a->r_h[n] = h; a->r_w[n] = w;
        a->r_tz[n] = (h + tzsz - 1) / tzsz;
        a->r_first[n + 1] = a->r_first[n] + a->r_tz[n] * ((w + txsz - 1) / txsz);
        ++n;
    };
    const int xr = dn + a->nx;  // first right-strip column
    for (int kind = 0; kind < 2; ++kind) {
        if (kind == 1) {  // C-PML x-band after the interior runs
            add(1, d0, 0, ny4, dn);
            add(1, d0, xr, ny4, a->nxt - xr);
            add(2, d0 + ny4, dn, nr - (d0 + ny4), a->nx);
            if (!a->fs) add(2, 0, dn, d0, a->nx);
        }
        for (size_t i = 0; i < runs.size(); ++i) {
            if (runs[i].second != kind) continue;
            const int q0 = runs[i].first;
            const int q1 = (i + 1 < runs.size()) ? runs[i + 1].first : nq;
            add(kind == 0 ? 0 : 4, d0 + 4 * q0, dn, 4 * (q1 - q0), a->nx);
        }
    }
    add(3, d0 + ny4, 0, nr - (d0 + ny4), dn);
    add(3, d0 + ny4, xr, nr - (d0 + ny4), a->nxt - xr);
    if (!a->fs) {  // with a free surface the rows above it are dead
        add(3, 0, 0, d0, dn);
        add(3, 0, xr, d0, a->nxt - xr);
    }
    a->nrect = n;
}

// Dynamic shared memory of the one-shot step kernel: an interior tile's p
// tile, or a staged z-strip tile.
constexpr int step_smem_floats() { return smem_floats<XS_ONE>() > kZsFloats ? smem_floats<XS_ONE>() : kZsFloats; }

template <int MODE>
int blocks_per_sm() {
    static int nb = 0;
    if (nb == 0) {
        const int bytes = step_smem_floats() * (int)sizeof(float);
        cudaFuncSetAttribute(step_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, step_kernel<MODE>, NT, bytes);
        nb = n > 0 ? n : 1;
    }
    return nb;
}

template <int FIXED>
int batch_blocks_per_sm() {
    static int nb = 0;
    if (nb == 0) {
        const int bytes = batch_smem_floats() * (int)sizeof(float);
        cudaFuncSetAttribute(batch_step_kernel<FIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_step_kernel<FIXED>, NT, bytes);
        nb = n > 0 ? n : 1;
    }
    return nb;
}

template <int MODE>
int launch_mode(const StepArgs& a, cudaStream_t stream) {
    if (a.ixb != NWARP * xxs<MODE, false>()) return (int)cudaErrorInvalidValue;  // a plan for another launch form
    const int bytes = step_smem_floats() * (int)sizeof(float);
    const dim3 grid(min(a.r_first[a.nrect], a.num_sms * blocks_per_sm<MODE>()));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(32, NWARP);
    cfg.dynamicSmemBytes = (size_t)bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelEx(&cfg, step_kernel<MODE>, a);
}

template <int MODE>
int pass_blocks_per_sm_t() {
    static int nb = -1;
    if (nb < 0) {
        const int bytes = smem_floats<XS_ONE>() * (int)sizeof(float);
        cudaFuncSetAttribute(pass_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pass_kernel<MODE>, NT, bytes) != cudaSuccess) n = 0;
        nb = n;
    }
    return nb;
}

template <int MODE>
int launch_pass_t(const PassParams& pp, int grid, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(32, NWARP);
    cfg.dynamicSmemBytes = (size_t)smem_floats<XS_ONE>() * sizeof(float);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelEx(&cfg, pass_kernel<MODE>, pp);
}

int prepare_step_kernels() {
    // Kernel attributes and occupancy are set up once, outside any stream
    // capture.
    return (blocks_per_sm<0>() > 0 && blocks_per_sm<1>() > 0 && blocks_per_sm<2>() > 0 &&
            batch_blocks_per_sm<-1>() > 0 && batch_blocks_per_sm<0>() > 0 && batch_blocks_per_sm<1>() > 0 &&
            batch_blocks_per_sm<2>() > 0 && pass_blocks_per_sm_t<0>() >= 0 && pass_blocks_per_sm_t<1>() >= 0 &&
            pass_blocks_per_sm_t<2>() >= 0)
               ? (int)cudaGetLastError()
               : 1;
}

int pass_blocks_per_sm(int mode) {
    if (mode == 0) return pass_blocks_per_sm_t<0>();
    if (mode == 1) return pass_blocks_per_sm_t<1>();
    return pass_blocks_per_sm_t<2>();
}

int launch_pass(int mode, const PassParams& pp, int grid, void* stream) {
    if (grid <= 0 || pp.nsteps <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (mode == 0) return launch_pass_t<0>(pp, grid, st);
    if (mode == 1) return launch_pass_t<1>(pp, grid, st);
    return launch_pass_t<2>(pp, grid, st);
}

void tile_rect(const StepArgs& a, int b, int* z0, int* z1, int* x0, int* x1) {
    int r = 0;
    while (r + 1 < a.nrect && b >= a.r_first[r + 1]) ++r;
    const int t = b - a.r_first[r], type = a.r_type[r];
    const int tzsz = (type == 0 || type == 1) ? TZ : (type == 4 ? 4 : PTZ);
    const int txsz = type == 0 ? a.itx : (type == 4 ? RTX : (type == 2 ? ZTX : (type == 1 ? a.ixb : PTX)));
    const int tz = t % a.r_tz[r], tx = t / a.r_tz[r];
    *z0 = a.r_zd0[r] + tz * tzsz;
    *x0 = a.r_x0[r] + tx * txsz;
    *z1 = min(*z0 + tzsz, a.r_zd0[r] + a.r_h[r]);
    *x1 = min(*x0 + txsz, a.r_x0[r] + a.r_w[r]);
}

// Neighbour lists of a plan (tiles within kTileReadHalo cells of each other,
// the reach of every tile's reads) and the receivers held by each tile, both
// as offset arrays.
void pass_lists(const StepArgs& a, int nrec, const int* h_rec_cell, std::vector<int>* nbr_first,
                std::vector<int>* nbr, std::vector<int>* rec_first, std::vector<int>* rec_idx) {
    const int n = a.r_first[a.nrect];
    std::vector<std::array<int, 4>> R(n);
    for (int b = 0; b < n; ++b) tile_rect(a, b, &R[b][0], &R[b][1], &R[b][2], &R[b][3]);
    const int H = kTileReadHalo;
    nbr_first->assign(n + 1, 0);
    nbr->clear();
    for (int b = 0; b < n; ++b) {
        for (int c = 0; c < n; ++c)
            if (c != b && R[c][0] < R[b][1] + H && R[b][0] - H < R[c][1] && R[c][2] < R[b][3] + H &&
                R[b][2] - H < R[c][3])
                nbr->push_back(c);
        (*nbr_first)[b + 1] = (int)nbr->size();
    }
    // A cell in no tile is never updated: its p stays 0, as the zeroed traces
    // already hold.
    std::vector<std::vector<int>> by(n);
    for (int i = 0; i < nrec; ++i) {
        const int x = h_rec_cell[i] / a.ldz, zd = h_rec_cell[i] % a.ldz;
        for (int b = 0; b < n; ++b)
            if (zd >= R[b][0] && zd < R[b][1] && x >= R[b][2] && x < R[b][3]) {
                by[b].push_back(i);
                break;
            }
    }
    rec_first->assign(n + 1, 0);
    rec_idx->clear();
    for (int b = 0; b < n; ++b) {
        rec_idx->insert(rec_idx->end(), by[b].begin(), by[b].end());
        (*rec_first)[b + 1] = (int)rec_idx->size();
    }
}

int launch_step(int mode, const StepArgs& a, void* stream) {
    if (a.r_first[a.nrect] <= 0) return 0;
    if (mode == 0) return launch_mode<0>(a, (cudaStream_t)stream);
    if (mode == 1) return launch_mode<1>(a, (cudaStream_t)stream);
    return launch_mode<2>(a, (cudaStream_t)stream);
}

__global__ void quantize_kernel(const float* src, const unsigned int* amax, void* dst, float* iscale, int n,
                                int kind16) {
    quantize_part(src, amax, dst, iscale, n, kind16, threadIdx.y * 32 + threadIdx.x);
}

int launch_quantize(const float* src, const unsigned int* amax, void* dst, float* iscale, int n, int kind16,
                    void* stream) {
    if (n <= 0) return 0;
    const int blocks = min((n / 4 + NT - 1) / NT, 148 * 8);
    quantize_kernel<<<blocks, dim3(32, NWARP), 0, (cudaStream_t)stream>>>(src, amax, dst, iscale, n, kind16);
    return (int)cudaGetLastError();
}

template <int FIXED>
int launch_batch(const BatchParams& bp, int num_sms, cudaStream_t stream) {
    const int total = bp.first[bp.nslots];
    const int bytes = batch_smem_floats() * (int)sizeof(float);
    const dim3 grid(min(total, num_sms * batch_blocks_per_sm<FIXED>()));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(32, NWARP);
    cfg.dynamicSmemBytes = (size_t)bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelEx(&cfg, batch_step_kernel<FIXED>, bp);
}

int launch_batch_step(const BatchParams& bp, int num_sms, void* stream) {
    const int total = bp.first[bp.nslots];
    if (bp.nslots <= 0 || total <= 0) return 0;
    bool same = true;
    for (int s = 1; s < bp.nslots; ++s) same = same && bp.mode[s] == bp.mode[0];
    cudaStream_t st = (cudaStream_t)stream;
    if (!same) return launch_batch<-1>(bp, num_sms, st);
    if (bp.mode[0] == 0) return launch_batch<0>(bp, num_sms, st);
    if (bp.mode[0] == 1) return launch_batch<1>(bp, num_sms, st);
    return launch_batch<2>(bp, num_sms, st);
}

// A bounded wait on copies that are never issued: the mbarrier expects 16
// bytes that no copy delivers, so the wait gives up after its time limit and
// reports through `err` exactly as a step kernel does.  Nothing is in flight,
// so returning is safe.
__global__ void wait_timeout_probe_kernel(int* err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    mbar_arrive_expect_tx(&bar, 16u);
    if (!mbar_wait_bounded(&bar, 0u)) atomicExch(err, 1);
}

int launch_wait_timeout_probe(int* err, void* stream) {
    wait_timeout_probe_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(err);
    return (int)cudaGetLastError();
}

// The snapshot quotient x / dt of the forward kernels for n inputs: q[i] by
// the interior tiles' form (div_dt_common for a float4, div_dt for all four
// when any of them is rare), q[n + i] by div_dt alone.  n is a multiple of 4.
__global__ void dt_quotients_kernel(const StepArgs a, const float* x, float* q, int n) {
    const int i = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= n) return;
    const float4 v = *reinterpret_cast<const float4*>(x + i);
    bool rare = false;
    float4 sv;
    sv.x = div_dt_common(a, v.x, rare);
    sv.y = div_dt_common(a, v.y, rare);
    sv.z = div_dt_common(a, v.z, rare);
    sv.w = div_dt_common(a, v.w, rare);
    if (rare) sv = make_float4(div_dt(a, v.x), div_dt(a, v.y), div_dt(a, v.z), div_dt(a, v.w));
    *reinterpret_cast<float4*>(q + i) = sv;
    *reinterpret_cast<float4*>(q + n + i) = make_float4(div_dt(a, v.x), div_dt(a, v.y), div_dt(a, v.z), div_dt(a, v.w));
}

int launch_dt_quotients(float dt, float inv_dt, float div_lo, float div_hi, int fast_div, const float* x, float* q,
                        int n, void* stream) {
    if (n <= 0 || n % 4) return (int)cudaErrorInvalidValue;
    StepArgs a{};
    a.dt = dt;
    a.inv_dt = inv_dt;
    a.div_lo = div_lo;
    a.div_hi = div_hi;
    a.fast_div = fast_div;
    dt_quotients_kernel<<<(n / 4 + 127) / 128, 128, 0, (cudaStream_t)stream>>>(a, x, q, n);
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
