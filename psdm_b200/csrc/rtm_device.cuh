// Device helpers shared by the step kernels (rtm_step.cu) and the two-step
// kernels (rtm_pair.cu): the reference's stencil sums in its evaluation
// order, the snapshot division, the 16-bit snapshot format, Kahan summation
// and the bulk asynchronous copies that complete on an mbarrier.  Everything
// here has internal linkage: each translation unit gets its own copy.
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

}  // namespace
}  // namespace psdm
