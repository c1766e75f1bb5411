// Device helpers shared by the step kernels (rtm_step.cu), the two-step
// kernels (rtm_pair.cu) and the resident pass kernel (rtm_resident.cu): the
// reference's stencil sums in its evaluation order, the snapshot division,
// the 16-bit snapshot format, Kahan summation, the bulk asynchronous copies
// that complete on an mbarrier, the generic per-cell update, the packed
// interior update of one float4 of rows and its snapshot / imaging step.
// Everything here has internal linkage: each translation unit gets its own
// copy.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "rtm_internal.h"

namespace psdm {
namespace {

constexpr int NWARP = 4;        // warps per block
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

// x / dt, correctly rounded (see fast_div_exact).  Inputs below div_lo
// (which includes every input whose quotient is subnormal) are scaled by 2^64
// first, which is exact: the scaled quotient q1 is correctly rounded to 24
// bits, q1 * 2^-64 is exact when the true quotient is normal, and when it is
// subnormal the only double-rounding case -- q1 * 2^-64 landing exactly half
// way between two subnormals -- is resolved with the sign of the exact
// residual x*2^64 - q1*dt.  Zero keeps its sign; only inputs above div_hi, or
// a dt that failed the host check, use the IEEE division.
__device__ __forceinline__ float div_dt(const StepArgs& a, float x) {
    const float ax = fabsf(x);
    if (ax == 0.f) return __fmul_rn(x, a.inv_dt);
    if (!a.fast_div || ax > a.div_hi) return __fdiv_rn(x, a.dt);
    const bool small = ax < a.div_lo;
    const float xs = small ? __fmul_rn(x, 0x1p64f) : x;
    const float q0 = __fmul_rn(xs, a.inv_dt);
    const float e = __fmaf_rn(-q0, a.dt, xs);
    const float q1 = __fmaf_rn(e, a.inv_dt, q0);
    if (!small) return q1;
    float q = __fmul_rn(q1, 0x1p-64f);
    const float diff = __fsub_rn(q1, __fmul_rn(q, 0x1p64f));  // exact
    if (fabsf(diff) == 0x1p-86f) {                             // half a subnormal step
        const float e1 = __fmaf_rn(-q1, a.dt, xs);             // sign of (true - q1)
        if (e1 != 0.f && signbit(e1) == signbit(diff)) q = __fadd_rn(q, copysignf(0x1p-149f, diff));
    }
    return q;
}

// x / dt for the common inputs -- x = +-0 (kept with its sign) or |x| in
// [div_lo, div_hi] with the fast form enabled -- without branches; `rare`
// is set for any other input, which div_dt then handles.
__device__ __forceinline__ float div_dt_common(const StepArgs& a, float x, bool& rare) {
    const float ax = fabsf(x);
    const float q0 = __fmul_rn(x, a.inv_dt);
    const float e = __fmaf_rn(-q0, a.dt, x);
    const float q1 = __fmaf_rn(e, a.inv_dt, q0);
    rare = rare || !(ax == 0.f || (a.fast_div && ax >= a.div_lo && ax <= a.div_hi));
    return ax == 0.f ? x : q1;
}

// Programmatic dependent launch: a step is launched with programmatic
// stream serialization, so its launch is processed while the previous step
// finishes; it touches nothing before the previous launch has completed and
// its writes are visible.  (Triggering the dependent launch early made the
// single-shot step slower: the waiting blocks take resident slots.)
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ float comp(const float4& v, int r) {
    return r == 0 ? v.x : (r == 1 ? v.y : (r == 2 ? v.z : v.w));
}

// ---- mixed-precision form: 16-bit snapshots and Kahan image -------------------

// Largest |snapshot| seen by this block since the last flush (float bits; the
// order of non-negative floats is the order of their bit patterns).
__shared__ unsigned int s_blk_amax;

__device__ __forceinline__ void amax_note(float v) { atomicMax(&s_blk_amax, __float_as_uint(fabsf(v))); }

// Scale exponent k for a snapshot of largest magnitude A (bits): A * 2^k in
// [2^14, 2^15), clamped to [-126, 126]; k = 0 for an all-zero snapshot.
__device__ __forceinline__ int snapshot_scale_exp(unsigned int bits) {
    if (bits == 0u) return 0;
    const int e = (int)((bits >> 23) & 0xffu) - 127;
    return min(126, max(-126, 14 - e));
}
__device__ __forceinline__ float pow2f(int k) { return __uint_as_float((unsigned int)(k + 127) << 23); }

// q_dst[i] = round16(q_src[i] * 2^k), i < n (n a multiple of 4), over the
// launch's blocks; block 0 writes 2^-k.
__device__ __forceinline__ void quantize_part(const float* __restrict__ src, const unsigned int* amax, void* dst,
                                              float* iscale, int n, int kind16, int tid) {
    const int k = snapshot_scale_exp(__ldg(amax));
    const float sc = pow2f(k);
    if (blockIdx.x == 0 && tid == 0) *iscale = pow2f(-k);
    const float4* s4 = reinterpret_cast<const float4*>(src);
    uint2* d4 = reinterpret_cast<uint2*>(dst);
    for (int i = blockIdx.x * NT + tid; i < n / 4; i += gridDim.x * NT) {
        const float4 v = __ldg(s4 + i);
        const float x0 = __fmul_rn(v.x, sc), x1 = __fmul_rn(v.y, sc), x2 = __fmul_rn(v.z, sc),
                    x3 = __fmul_rn(v.w, sc);
        uint2 o;
        if (kind16 == 1) {
            const __half2 a = __floats2half2_rn(x0, x1), b = __floats2half2_rn(x2, x3);
            o.x = *reinterpret_cast<const unsigned int*>(&a);
            o.y = *reinterpret_cast<const unsigned int*>(&b);
        } else {
            const __nv_bfloat162 a = __floats2bfloat162_rn(x0, x1), b = __floats2bfloat162_rn(x2, x3);
            o.x = *reinterpret_cast<const unsigned int*>(&a);
            o.y = *reinterpret_cast<const unsigned int*>(&b);
        }
        d4[i] = o;
    }
}

__device__ __forceinline__ float2 unpack16(unsigned int w, int kind16) {
    if (kind16 == 1) return __half22float2(*reinterpret_cast<const __half2*>(&w));
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
}

// Four consecutive snapshot values (16-byte aligned group) as floats.
__device__ __forceinline__ uint2 load16x4_raw(const void* base, int fi) {
    return __ldg(reinterpret_cast<const uint2*>(static_cast<const unsigned short*>(base) + fi));
}
__device__ __forceinline__ float4 unpack16x4(const uint2 w, int kind16, float isc) {
    const float2 a = unpack16(w.x, kind16), b = unpack16(w.y, kind16);
    return make_float4(__fmul_rn(a.x, isc), __fmul_rn(a.y, isc), __fmul_rn(b.x, isc), __fmul_rn(b.y, isc));
}

__device__ __forceinline__ float load16x1(const void* base, int fi, int kind16, float isc) {
    const unsigned short h = __ldg(static_cast<const unsigned short*>(base) + fi);
    const float v = kind16 == 1 ? __half2float(__ushort_as_half(h)) : __bfloat162float(__ushort_as_bfloat16(h));
    return __fmul_rn(v, isc);
}

// img += inc with Kahan compensation c: y = inc - c, t = img + y,
// c = (t - img) - y, img = t.
__device__ __forceinline__ void kahan(float& img, float& c, float inc) {
    const float y = __fsub_rn(inc, c);
    const float t = __fadd_rn(img, y);
    c = __fsub_rn(__fsub_rn(t, img), y);
    img = t;
}

// ---- bulk asynchronous copies (global -> shared) completing on an mbarrier

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the phase `parity` of `bar` for at most ~1 s.  Returns false on
// timeout (the copies never completed); the caller reports it.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > 1000000000ull) return false;
    }
}

__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 neg2(const float2& v) { return make_float2(-v.x, -v.y); }
// sum_{k=0..3} c[k] * (a(+k) + a(-k)) on a pair, in the reference's order.
// Tap sums and products are packed; the running sum is accumulated with
// scalar adds: the compiler may fuse a packed multiply into a following
// packed add (FFMA2) even when both are written with explicit rounding,
// which would change the result, and it never fuses scalar RN adds.
__device__ __forceinline__ float2 sum4(const float2& t0, const float2& t1, const float2& t2, const float2& t3) {
    return make_float2(__fadd_rn(__fadd_rn(__fadd_rn(t0.x, t1.x), t2.x), t3.x),
                       __fadd_rn(__fadd_rn(__fadd_rn(t0.y, t1.y), t2.y), t3.y));
}
#define D2P(AT, c)                                                        \
    sum4(__fmul2_rn(__fadd2_rn(AT(0), AT(0)), (c)[0]),                    \
         __fmul2_rn(__fadd2_rn(AT(1), AT(-1)), (c)[1]),                   \
         __fmul2_rn(__fadd2_rn(AT(2), AT(-2)), (c)[2]),                   \
         __fmul2_rn(__fadd2_rn(AT(3), AT(-3)), (c)[3]))
// a + b with b a fresh product: scalar adds (see above).
__device__ __forceinline__ float2 add_prod(const float2& a, const float2& b) {
    return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}

// Any cell of the grid: C-PML strips and corners, free-surface row,
// injection, interior.  zd = device row (logical z = zd - zoff); the p tile
// has SH rows per column and origin (sz0, sx0).  RES: level n-1 of the cell
// is read from the shared tile pps (same origin and pitch as ps) instead of
// a.pm, and the new level is stored there as well as to a.pm.
template <int MODE, int SH, bool RES = false>
__device__ __forceinline__ void cell_generic(const StepArgs& a, const float* __restrict__ ps, int sz0, int sx0, int zd,
                                             int x, float* pps = nullptr) {
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
    const float pmo = RES ? pps[xl * SH + zl] : a.pm[g];
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
#define PX(k) ph[(k) * a.ldz]
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
#define PZ(k) ph[(k)]
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
    if (RES) pps[xl * SH + zl] = out;

    if (kx == 0 && kz == 0 && a.field != nullptr) {
        const int fi = (x - dn) * a.ldf + (z - dn);
        if (MODE == 0) {
            const float D = div_dt(a, __fmul_rn(__fsub_rn(out, pmo), 0.5f));
            a.field[fi] = D;
            if (a.field_amax != nullptr) amax_note(D);
        } else {
            float F = __ldg(a.field + fi);
            if (a.field_w != 1.f) F = __fmul_rn(F, a.field_w);
            float inc = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out, pmo)), F);
            if (a.ss != 1.f) inc = __fmul_rn(inc, a.ss);
            a.image[fi] = __fadd_rn(a.image[fi], inc);
        }
    }
    if (MODE == 2 && kx == 0 && kz == 0 && a.field16 != nullptr) {
        const int fi = (x - dn) * a.ldf + (z - dn);
        float F = load16x1(a.field16, fi, a.kind16, __ldg(a.field_iscale));
        if (a.field_w != 1.f) F = __fmul_rn(F, a.field_w);
        float inc = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(out, pmo)), F);
        if (a.ss != 1.f) inc = __fmul_rn(inc, a.ss);
        kahan(a.image[fi], a.comp[fi], inc);
    }
}

// The packed FP32x2 interior update of the one-step interior tiles for one
// float4 of rows: win = the 7 x-neighbour columns (centre win[3]), zm / zp =
// the float4s above and below the centre, pmv = level n-1 of the float4,
// c2v = its c2.  Tap sums and products are packed; every add that consumes
// a fresh product is scalar, so no multiply-add is ever fused.
__device__ __forceinline__ float4 clean_update(const float4 (&win)[7], const float4& zm, const float4& zp,
                                               const float4& pmv, const float4& c2v, const float2 (&cc)[4]) {
    const float4& pc = win[3];
    const float2 z01 = make_float2(zm.y, zm.z), z12 = make_float2(zm.z, zm.w);
    const float2 z23 = make_float2(zm.w, pc.x), z34 = lo2(pc);
    const float2 z45 = make_float2(pc.y, pc.z), z56 = hi2(pc);
    const float2 z67 = make_float2(pc.w, zp.x), z78 = lo2(zp);
    const float2 z89 = make_float2(zp.y, zp.z);
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
    const float2 two = make_float2(2.f, 2.f);
    const float2 baseA = __fadd2_rn(neg2(lo2(pmv)), __fmul2_rn(two, lo2(pc)));
    const float2 baseB = __fadd2_rn(neg2(hi2(pmv)), __fmul2_rn(two, hi2(pc)));
    const float2 oA = add_prod(baseA, __fmul2_rn(lo2(c2v), __fadd2_rn(d2xA, d2yA)));
    const float2 oB = add_prod(baseB, __fmul2_rn(hi2(c2v), __fadd2_rn(d2xB, d2yB)));
    return make_float4(oA.x, oA.y, oB.x, oB.y);
}

// Snapshot (forward) or imaging update (backward) of one float4 of interior
// cells at offset fi of the pitched snapshot / image: out = the new level,
// pmv = the level two steps back.  Fc / Ic / Cc / Frc: prefetched snapshot,
// image, compensation and raw 16-bit snapshot values.
template <int MODE>
__device__ __forceinline__ void emit4(const StepArgs& a, const SubStep& s, int fi, const float4& out,
                                      const float4& pmv, float4 Fc, const float4& Ic, const float4& Cc,
                                      const uint2& Frc, float isc, float& amax_t) {
    if (MODE == 0) {
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
        *reinterpret_cast<float4*>(s.field + fi) = sv;
        if (s.field_amax != nullptr)
            amax_t = fmaxf(amax_t, fmaxf(fmaxf(fabsf(sv.x), fabsf(sv.y)), fmaxf(fabsf(sv.z), fabsf(sv.w))));
    } else if (MODE == 1) {
        if (s.field_w != 1.f) {
            Fc.x = __fmul_rn(Fc.x, s.field_w); Fc.y = __fmul_rn(Fc.y, s.field_w);
            Fc.z = __fmul_rn(Fc.z, s.field_w); Fc.w = __fmul_rn(Fc.w, s.field_w);
        }
        const float2 half = make_float2(0.5f, 0.5f);
        const float2 oA = lo2(out), oB = hi2(out);
        float2 iA = __fmul2_rn(__fmul2_rn(half, __fadd2_rn(oA, neg2(lo2(pmv)))), lo2(Fc));
        float2 iB = __fmul2_rn(__fmul2_rn(half, __fadd2_rn(oB, neg2(hi2(pmv)))), hi2(Fc));
        if (a.ss != 1.f) {
            const float2 ss = make_float2(a.ss, a.ss);
            iA = __fmul2_rn(iA, ss);
            iB = __fmul2_rn(iB, ss);
        }
        const float2 rA = add_prod(lo2(Ic), iA), rB = add_prod(hi2(Ic), iB);
        *reinterpret_cast<float4*>(a.image + fi) = make_float4(rA.x, rA.y, rB.x, rB.y);
    } else {
        const float4 F4 = unpack16x4(Frc, a.kind16, isc);
        float Fv[4] = {F4.x, F4.y, F4.z, F4.w};
        float Iv[4] = {Ic.x, Ic.y, Ic.z, Ic.w};
        float Cv[4] = {Cc.x, Cc.y, Cc.z, Cc.w};
        const float ov[4] = {out.x, out.y, out.z, out.w};
        const float pv[4] = {pmv.x, pmv.y, pmv.z, pmv.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            float F = Fv[e];
            if (s.field_w != 1.f) F = __fmul_rn(F, s.field_w);
            float inc = __fmul_rn(__fmul_rn(0.5f, __fsub_rn(ov[e], pv[e])), F);
            if (a.ss != 1.f) inc = __fmul_rn(inc, a.ss);
            kahan(Iv[e], Cv[e], inc);
        }
        *reinterpret_cast<float4*>(a.image + fi) = make_float4(Iv[0], Iv[1], Iv[2], Iv[3]);
        *reinterpret_cast<float4*>(a.comp + fi) = make_float4(Cv[0], Cv[1], Cv[2], Cv[3]);
    }
}

// One column x of a C-PML x-strip (kz = 0) for the float4 of rows zd..zd+3
// (a multiple of 4), split into its global loads (xband_load: phi_x around
// the strip-local stencil centre, phi_x, chi_x and c2 of the cells, and level
// n-1 unless it comes from shared memory) and its update (xband_compute), so
// that callers can load the next column while they update this one.  p at
// level n comes from the shared tile ps4 (HQP float4 rows per column, origin
// column sx0, float4 row qr of zd).  RES: level n-1 is read from, and the new
// level also stored to, the shared tile pps4.
struct XbandIn {
    float4 F[7];  // phi_x stencil around the strip-local centre (F[3] unused)
    float4 phc, chc, c2v, pmv;
    float A, B;
};

__device__ __forceinline__ void xband_load(const StepArgs& a, int zd, int x, bool load_pm, XbandIn& in) {
    const int dn = a.dn;
    const int kx = (x < dn) ? (dn - x) : (x - (dn + a.nx) + 1);
    const int sb = (x < dn) ? 0 : dn + a.nx;
    const int ci = clampi(x - sb, 3, dn - 4) + sb;
    in.A = __ldg(a.fA + kx - 1);
    in.B = __ldg(a.fB + kx - 1);
    const int g = x * a.ldz + zd;
#pragma unroll
    for (int k = 0; k < 7; ++k)
        if (k != 3) in.F[k] = *reinterpret_cast<const float4*>(a.phix_in + (ci + k - 3) * a.ldz + zd);
    in.F[3] = make_float4(0.f, 0.f, 0.f, 0.f);
    in.phc = *reinterpret_cast<const float4*>(a.phix_in + g);
    in.chc = *reinterpret_cast<const float4*>(a.chix + g);
    in.c2v = __ldg(reinterpret_cast<const float4*>(a.c2 + g));
    if (load_pm) in.pmv = *reinterpret_cast<const float4*>(a.pm + g);
}

template <int HQP, bool RES = false>
__device__ __forceinline__ void xband_compute(const StepArgs& a, const float4* __restrict__ ps4, float4* pps4, int sx0,
                                              int qr, int zd, bool fsq, int x, const XbandIn& in) {
    const float* c1 = a.cf1;
    const float* c2 = a.cf2;
    const int cx = clampi(x, 3, a.nxt - 4);
    const int g = x * a.ldz + zd;
    float4 P[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) P[k] = ps4[(cx + k - 3 - sx0) * HQP + qr];
    const float4 zc = ps4[(x - sx0) * HQP + qr];
    const float4 zm = ps4[(x - sx0) * HQP + qr - 1];
    const float4 zp = ps4[(x - sx0) * HQP + qr + 1];
    const float4 pmv = RES ? pps4[(x - sx0) * HQP + qr] : in.pmv;
    const float zv[10] = {zm.y, zm.z, zm.w, zc.x, zc.y, zc.z, zc.w, zp.x, zp.y, zp.z};
    float o[4], phn[4], chn[4];
#pragma unroll
    for (int rr = 0; rr < 4; ++rr) {
#define PXR(k) comp(P[3 + (k)], rr)
#define FXR(k) comp(in.F[3 + (k)], rr)
#define ZR(k) zv[3 + rr + (k)]
        const float d2x = D2(PXR, c2);
        const float d1x = D1(PXR, c1);
        const float d2y = D2(ZR, c2);
        const float dph = D1(FXR, c1);
#undef PXR
#undef FXR
#undef ZR
        phn[rr] = __fadd_rn(__fmul_rn(in.A, comp(in.phc, rr)), __fmul_rn(in.B, d1x));
        chn[rr] = __fadd_rn(__fmul_rn(in.A, comp(in.chc, rr)), __fmul_rn(in.B, __fadd_rn(d2x, dph)));
        const float prop = __fadd_rn(dph, chn[rr]);
        float pp = comp(zc, rr), ppm = comp(pmv, rr);
        if (rr == 0 && fsq && !a.disk) { pp = a.side_p[x]; ppm = a.side_pm[x]; }
        const float base = __fadd_rn(-ppm, __fmul_rn(2.f, pp));
        o[rr] = __fadd_rn(base, __fmul_rn(comp(in.c2v, rr), __fadd_rn(__fadd_rn(d2x, d2y), prop)));
    }
    if (fsq && !a.disk) {  // free-surface row: private history keeps p3, the grid gets 0
        a.side_pm[x] = o[0];
        o[0] = 0.f;
    }
    const float4 out = make_float4(o[0], o[1], o[2], o[3]);
    *reinterpret_cast<float4*>(a.pm + g) = out;
    if (RES) pps4[(x - sx0) * HQP + qr] = out;
    *reinterpret_cast<float4*>(a.phix_out + g) = make_float4(phn[0], phn[1], phn[2], phn[3]);
    *reinterpret_cast<float4*>(a.chix + g) = make_float4(chn[0], chn[1], chn[2], chn[3]);
}

// ---- step counters of the one-launch-per-pass forms

__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Later bulk copies (async proxy) of this thread see what its generic-proxy
// acquire made visible.
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Wait until *flag >= need: relaxed polls, then one acquire load.  Gives up
// after ~1 s, or at once when another block has given up (abort, a device
// word: polling the host-mapped error word would cost a PCIe round trip).
__device__ bool wait_flag(const int* flag, int need, const int* abort) {
    if (ld_relaxed(flag) < need) {
        const uint64_t t0 = globaltimer_ns();
        for (int it = 0;; ++it) {
            if (ld_relaxed(flag) >= need) break;
            if ((it & 15) == 15 && (ld_relaxed(abort) != 0 || globaltimer_ns() - t0 > 1000000000ull)) return false;
        }
    }
    return ld_acquire(flag) >= need;  // the flag only grows
}

}  // namespace
}  // namespace psdm
