// Frequency filter of recorded traces on the device: the reference's
// freq_filter (src/auxiliar.f90:498-531) with filters_function1D and its
// order-6 Butterworth response (src/filters.f90:50-232).  Each trace is
// placed at the end of a zero buffer 24 times its length, transformed,
// multiplied by the response (and by 1/n, the forward scaling of the
// reference's FFT), transformed back, and the real part of the last nt
// samples is kept; see filter_traces for the half-spectrum form used here.  The transforms are cuFFT's (a library FFT, like the
// reference's vendored FFTPACK); the results agree with the reference's
// arithmetic to FP32 rounding, not bit for bit.

#include <cuda_runtime.h>
#include <cuComplex.h>
#include <cufft.h>

#include <cmath>
#include <complex>
#include <vector>

#include "../../include/psdm_rtm.h"
#include "rtm_internal.h"

namespace psdm {

// Butterworth response H[ts] (butterworth, filters.f90:129-232) for the
// filter filters_function1D sets up: order n = 6 (even), high-pass start
// fs = 40 Hz, band edges f1 and fc, f0 = sqrt(f1 fc), Q = f0 / (fc - f1),
// frequency step fe/ts accumulated in single precision as the reference does.
void butterworth_response(int ts, float fe, int typef, float f1, float fc, std::complex<float>* H) {
    using cf = std::complex<float>;
    const int n = 6;
    const float pi = 3.14159265f, fs = 40.f;
    const float f2 = fc;
    const float f0 = std::sqrt(f1 * f2);
    const float Q = f0 / (f2 - f1);
    const cf I(0.f, 1.f);
    std::vector<cf> Bn(ts, cf(1.f, 0.f));
    float f = 0.f;
    for (int j = 0; j < ts / 2 + 1; ++j) {
        for (int k = 1; k <= n / 2; ++k) {
            const float c = std::cos((float(2 * k + n - 1) * pi) / float(2 * n));
            cf s;
            if (typef == 1)
                s = (I * f) / fc;
            else if (typef == 2)
                s = fs / (I * f);
            else
                s = Q * ((I * f) / f0 + f0 / (I * f));
            Bn[j] = Bn[j] * (s * s - 2.f * s * c + 1.f);
        }
        f = f + fe / float(ts);
    }
    for (int j = 0; j < ts / 2 + 1; ++j) H[j] = cf(1.f, 0.f) / Bn[j];
    H[0] = typef == 1 ? cf(1.f, 0.f) : cf(0.f, 0.f);
    for (int j = 2; j <= ts / 2; ++j) H[ts / 2 + j - 1] = std::conj(H[ts / 2 + 1 - (j - 1) - 1]);
}

namespace {

// Real input rows of ts samples, the trace at the end of each.
__global__ void pad_traces(const float* tr, int nt, int ts, int num, float* x) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)ts * num) return;
    const int t = (int)(i % ts), r = (int)(i / ts);
    const int off = ts - nt;
    x[i] = t >= off ? tr[(size_t)r * nt + (t - off)] : 0.f;
}

// The non-negative half of the spectrum times H / ts (the forward scaling
// of the reference's transform).
__global__ void apply_response(cufftComplex* X, const cufftComplex* H, int nh, int num, float scale) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nh * num) return;
    const cufftComplex h = H[i % nh], v = X[i];
    const float re = v.x * scale, im = v.y * scale;
    X[i] = make_cuComplex(re * h.x - im * h.y, re * h.y + im * h.x);
}

__global__ void unpad_traces(const float* x, int nt, int ts, int num, const int* keep, float* tr) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nt * num) return;
    const int t = (int)(i % nt), r = (int)(i / nt);
    if (!keep[r]) return;  // an all-zero trace is left as it is (is_not_cero)
    tr[i] = x[(size_t)r * ts + (ts - nt) + t];
}

__global__ void nonzero_traces(const float* tr, int nt, int num, int* keep) {
    const int r = blockIdx.x;
    if (r >= num) return;
    int any = 0;
    for (int t = threadIdx.x; t < nt && !any; t += blockDim.x) any = tr[(size_t)r * nt + t] != 0.f;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) keep[r] = any;
}

}  // namespace

size_t filter_work_floats(int ts, int num) {
    const size_t real = ((size_t)ts * num + 3) & ~(size_t)3;  // complex half starts 16-byte aligned
    return real + (size_t)(ts / 2 + 1) * num * 2;
}

// The reference transforms the real trace as a complex one and keeps the real
// part of the inverse.  The product of a real trace's spectrum with the
// response is Hermitian in every bin but ts/2, where only its real part
// reaches the real output, so the half-spectrum transforms (real to complex,
// complex to real, which reads the real part of bin ts/2) give the same
// result at half the work.
int filter_traces(float* d_tr, int nt, int num, const void* d_H, float* d_x, int* d_keep, int ts, const int* plans,
                  void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const int nh = ts / 2 + 1;
    float* x = d_x;
    cufftComplex* X = reinterpret_cast<cufftComplex*>(d_x + (((size_t)ts * num + 3) & ~(size_t)3));
    const size_t total = (size_t)ts * num;
    nonzero_traces<<<num, 256, 0, st>>>(d_tr, nt, num, d_keep);
    pad_traces<<<(int)((total + 255) / 256), 256, 0, st>>>(d_tr, nt, ts, num, x);
    if (cufftSetStream(plans[0], st) != CUFFT_SUCCESS || cufftSetStream(plans[1], st) != CUFFT_SUCCESS) return 1;
    if (cufftExecR2C(plans[0], x, X) != CUFFT_SUCCESS) return 2;
    apply_response<<<(int)(((size_t)nh * num + 255) / 256), 256, 0, st>>>(X, static_cast<const cufftComplex*>(d_H), nh,
                                                                          num, 1.f / float(ts));
    if (cufftExecC2R(plans[1], X, x) != CUFFT_SUCCESS) return 3;
    unpad_traces<<<(int)(((size_t)nt * num + 255) / 256), 256, 0, st>>>(x, nt, ts, num, d_keep, d_tr);
    return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

int make_fft_plans(int ts, int num, int* plans) {
    cufftHandle a, b;
    int n[1] = {ts};
    const int nh = ts / 2 + 1;
    if (cufftPlanMany(&a, 1, n, nullptr, 1, ts, nullptr, 1, nh, CUFFT_R2C, num) != CUFFT_SUCCESS) return 1;
    if (cufftPlanMany(&b, 1, n, nullptr, 1, nh, nullptr, 1, ts, CUFFT_C2R, num) != CUFFT_SUCCESS) {
        cufftDestroy(a);
        return 1;
    }
    plans[0] = a;
    plans[1] = b;
    return 0;
}

void destroy_fft_plans(int* plans) {
    cufftDestroy(plans[0]);
    cufftDestroy(plans[1]);
}

}  // namespace psdm

extern "C" int psdm_butterworth_response(int32_t ts, float fe, int32_t typef, float f1, float f2, float* H) {
    if (!H || ts < 2 || (ts & 1) || typef < 1 || typef > 3) {
        psdm::set_last_error("psdm_butterworth_response: null output, odd or short length, or typef not 1..3");
        return PSDM_ERR_ARG;
    }
    psdm::butterworth_response(ts, fe, typef, f1, f2, reinterpret_cast<std::complex<float>*>(H));
    return PSDM_OK;
}
