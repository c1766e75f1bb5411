// Conditioning of a shot's observed traces on the device: resampling from
// the data time step to the propagation time step (Akima's local cubic
// interpolation), the sea-floor cut, the multiple cut and the half-cosine
// taper with zero padding -- the per-shot block of
// src/calculate_PSDM_RTM.f90:316-355 that prepares Data_target for the
// backward pass (the frequency filter, freq_filter in auxiliar.f90:498-531,
// stays on the host).  One block per trace; every output sample is computed
// independently, in FP32 with the same operations and order as the CPU
// restatement it is checked against.

#include <cuda_runtime.h>

#include "rtm_internal.h"

namespace psdm {
namespace {

// Akima's (1970) interpolation of y sampled at x_k = k*dx, k < n.  End
// slopes: m[-1] = 2m[0] - m[1], m[-2] = 2m[-1] - m[0], mirrored at the far
// end; outside the data the end interval's cubic is used.
struct AkimaDev {
    const float* y;
    int n;
    float dx;
    __device__ float x(int k) const { return float(k) * dx; }
    __device__ float mi(int k) const { return (__ldg(y + k + 1) - __ldg(y + k)) / (x(k + 1) - x(k)); }
    __device__ float m(int k) const {
        if (k < 0) {
            const float m0 = mi(0), m1 = mi(1);
            const float mm1 = 2.f * m0 - m1;
            return k == -1 ? mm1 : 2.f * mm1 - m0;
        }
        if (k > n - 2) {
            const float a = mi(n - 2), b = mi(n - 3);
            const float mp = 2.f * a - b;
            return k == n - 1 ? mp : 2.f * mp - a;
        }
        return mi(k);
    }
    __device__ float slope_at(int k) const {
        const float mk2 = m(k - 2), mk1 = m(k - 1), mk = m(k), mk1p = m(k + 1);
        const float w1 = fabsf(mk1p - mk), w2 = fabsf(mk1 - mk2);
        if (w1 + w2 == 0.f) return 0.5f * (mk1 + mk);
        return (w1 * mk1 + w2 * mk) / (w1 + w2);
    }
    __device__ float at(float t) const {
        if (n == 1) return __ldg(y);
        if (n == 2) return __ldg(y) + (t - x(0)) * ((__ldg(y + 1) - __ldg(y)) / (x(1) - x(0)));
        if (t == x(n - 1)) return __ldg(y + n - 1);
        int j = (int)(t / dx);
        j = min(max(j, 0), n - 2);
        while (j > 0 && t < x(j)) --j;
        while (j < n - 2 && t >= x(j + 1)) ++j;
        const float h = x(j + 1) - x(j), d = t - x(j);
        const float tj = slope_at(j), tj1 = slope_at(j + 1), mj = m(j);
        const float p2 = (3.f * mj - 2.f * tj - tj1) / h;
        const float p3 = (tj + tj1 - 2.f * mj) / (h * h);
        return __ldg(y + j) + d * (tj + d * (p2 + d * p3));
    }
};

__global__ void condition_kernel(CondArgs c) {
    const int i = blockIdx.x;
    const float* f = c.field + (size_t)i * c.nt_data;
    float* tr = c.out + (size_t)i * c.nt_taper;
    const AkimaDev ak{f, c.nt_data, c.dt_data};
    const int cut = max(1, min(c.nt_cut[i], c.nt_taper));
    const int nsf = c.nt_sf[i];
    for (int s0 = threadIdx.x; s0 < c.nt_taper; s0 += blockDim.x) {
        const int s = s0 + 1;  // 1-based sample, as in the reference's loops
        float v = 0.f;
        if (s <= c.nt_prop2) {
            if (c.resample)
                v = ak.at(float(s0) * c.dt_prop);
            else if (s <= c.nt_data)
                v = __ldg(f + s0);
        }
        if (c.cut_sf > 0 && s <= nsf) v = 0.f;
        // taper_pad_trace (src/filters.f90:20-48) over the first `end` samples
        int end = 0;
        if (c.cut_multiple == 0) {
            if (c.taper_option != 0) end = c.nt_prop2;
        } else {
            end = cut;
            if (s >= cut) v = 0.f;
        }
        if (end > 0) {
            const int i0 = max(1, end - c.N_taper + 1);
            if (s >= i0 && s <= end && s - i0 < c.N_taper) v = v * __ldg(c.w + (s - i0));
            if (c.N_zeros > 0 && s > end) v = 0.f;
        }
        tr[s0] = v;
    }
}

}  // namespace

int launch_condition(const CondArgs& c, void* stream) {
    if (c.nrec <= 0 || c.nt_taper <= 0) return 0;
    condition_kernel<<<c.nrec, 256, 0, (cudaStream_t)stream>>>(c);
    return (int)cudaGetLastError();
}

}  // namespace psdm
