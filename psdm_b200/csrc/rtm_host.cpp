// Host-side set-up arithmetic of the RTM path, in the reference's FP32
// evaluation order (coefficients are computed once per shot on the host and
// handed to the device kernels).
//
//   psdm_fd_coef          src/solver_FD_coeffs.f90:1-73
//   psdm_pml_coeffs       src/solver_PML_coeffs.f90:1-75
//   psdm_ricker_mcs       src/get_mcs_data.f90:318-351
//   psdm_dynamic_window   src/dynamic_window.f90:1-52
//   psdm_taper_pad_trace  src/filters.f90:20-48
//   psdm_optimization_dt  src/optimization.f90:24-32
//   psdm_normalize_psdm   src/auxiliar_PSDM.f90:1-20
//   psdm_trace_windows    src/calculate_PSDM_RTM.f90:231-291

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/psdm_rtm.h"
#include "rtm_internal.h"

namespace psdm {

void pml_profiles_f32(int acc, int dPML, float dt, float d, int dn, float* fA, float* fB) {
    // Profile over strip index i in [acc+1, dPML+acc] (1-based, 1 = next to
    // the interior); zero for i <= acc; the last value beyond dPML+acc.
    for (int i = 0; i < dn; ++i) { fA[i] = 0.f; fB[i] = 0.f; }
    const float pi = 3.14159265f;
    const float refl = 0.00001f;
    const float w = float(dPML - 1) * d;
    const float s0 = -((6000.f * logf(refl)) / (2.f * w));
    for (int i = acc + 1; i <= dPML + acc; ++i) {
        const float y = float(i - (acc + 1)) * d;
        const float r = y / w;
        const float alpha = 30.f * pi * (1.f - r);
        const float sigma = s0 * (r * r);
        const float A = expf(-((sigma + alpha) * dt));
        fA[i - 1] = A;
        fB[i - 1] = ((A - 1.f) * sigma) / (sigma + alpha);
    }
    for (int i = dPML + acc + 1; i <= dn; ++i) { fA[i - 1] = fA[dPML + acc - 1]; fB[i - 1] = fB[dPML + acc - 1]; }
}

// FD coefficients of src/solver_FD_coeffs.f90:14-19,43-50,68 (acc = 3) as
// double-precision rationals; the centre tap of the 2nd derivative halved.
void fd_coef_f64(int num, double* c) {
    if (num == 1) {
        c[0] = 0.0; c[1] = 3.0 / 4.0; c[2] = -3.0 / 20.0; c[3] = 1.0 / 60.0;
    } else {
        c[0] = (-49.0 / 18.0) / 2.0; c[1] = 3.0 / 2.0; c[2] = -3.0 / 20.0; c[3] = 1.0 / 90.0;
    }
}

void pml_profiles_f64(int acc, int dPML, double dt, double d, int dn, double* fA, double* fB) {
    for (int i = 0; i < dn; ++i) { fA[i] = 0.0; fB[i] = 0.0; }
    const double pi = 3.14159265;
    const double refl = 0.00001;
    const double w = double(dPML - 1) * d;
    const double s0 = -((6000.0 * log(refl)) / (2.0 * w));
    for (int i = acc + 1; i <= dPML + acc; ++i) {
        const double y = double(i - (acc + 1)) * d;
        const double r = y / w;
        const double alpha = 30.0 * pi * (1.0 - r);
        const double sigma = s0 * (r * r);
        const double A = exp(-((sigma + alpha) * dt));
        fA[i - 1] = A;
        fB[i - 1] = ((A - 1.0) * sigma) / (sigma + alpha);
    }
    for (int i = dPML + acc + 1; i <= dn; ++i) { fA[i - 1] = fA[dPML + acc - 1]; fB[i - 1] = fB[dPML + acc - 1]; }
}

// Division by a fixed y as q0 = RN(x*r), e = x - q0*y (exact, one FMA),
// q = RN(q0 + e*r) with r = RN(1/y).  By Markstein's theorem this is the
// correctly rounded x/y when no intermediate leaves the normal range; the
// check below confirms it for every significand of one binade of x (the
// result scales exactly with powers of two of x), so for |x| in [lo, hi]
// the kernels may use it in place of an IEEE division.
bool fast_div_exact(float y, float* r, float* lo, float* hi, float* tiny) {
    volatile float one = 1.0f;
    const float rr = one / y;
    *r = rr;
    *lo = ldexpf(1.0f, -90);
    *hi = std::min(ldexpf(1.0f, 100), ldexpf(y, 120));
    // below lo the kernels scale x by 2^64 (every nonzero float then lies in
    // [2^-85, 2^-26], inside [lo, hi]); tiny is kept for reference only
    *tiny = ldexpf(1.0f, -149);
    if (!(y > 0.f) || !std::isfinite(y) || !std::isfinite(rr)) return false;
    for (uint32_t m = 0; m < (1u << 23); ++m) {
        const uint32_t bits = 0x3f800000u | m;
        float x;
        std::memcpy(&x, &bits, sizeof(x));
        const float q0 = x * rr;
        const float e = std::fmaf(-q0, y, x);
        const float q = std::fmaf(e, rr, q0);
        volatile float xv = x;
        if (q != xv / y) return false;
    }
    return true;
}

float taper_weight(int n, int N_taper) {
    const float pi = 4.0f * atanf(1.0f);
    return 0.5f * (1.0f + cosf((pi * float(n)) / float(N_taper)));
}

}  // namespace psdm

extern "C" {

void psdm_fd_coef(int32_t num, int32_t accuracy, float* coef) {
    for (int i = 0; i <= accuracy; ++i) coef[i] = 0.f;
    if (num == 1) {
        if (accuracy == 3) { coef[1] = 3.f / 4.f; coef[2] = -3.f / 20.f; coef[3] = 1.f / 60.f; }
        if (accuracy == 4) { coef[1] = 4.f / 5.f; coef[2] = -1.f / 5.f; coef[3] = 4.f / 105.f; coef[4] = -1.f / 280.f; }
    }
    if (num == 2) {
        if (accuracy == 3) { coef[0] = -49.f / 18.f; coef[1] = 3.f / 2.f; coef[2] = -3.f / 20.f; coef[3] = 1.f / 90.f; }
        if (accuracy == 4) {
            coef[0] = -205.f / 72.f; coef[1] = 8.f / 5.f; coef[2] = -1.f / 5.f; coef[3] = 8.f / 315.f; coef[4] = -1.f / 560.f;
        }
        if (accuracy == 5) {
            coef[0] = -5269.f / 1800.f; coef[1] = 5.f / 3.f; coef[2] = -5.f / 21.f; coef[3] = 5.f / 126.f;
            coef[4] = -5.f / 1008.f; coef[5] = 1.f / 3150.f;
        }
        coef[0] = coef[0] / 2.f;
    }
}

void psdm_pml_coeffs(int32_t acc, int32_t dPML, float dt, float d, int32_t dn, float* factorA,
                     float* factorB, float* corners) {
    psdm::pml_profiles_f32(acc, dPML, dt, d, dn, factorA, factorB);
    if (!corners) return;
    // Every corner cell uses the profile at max(kx, kz), both counted from the
    // interior (k = 1 next to it); the reference builds the same tables by
    // symmetric filling (solver_PML_coeffs.f90:36-70).
    const size_t dd = (size_t)dn * dn;
    float* ldA = corners + 0 * dd; float* rdA = corners + 1 * dd;
    float* luA = corners + 2 * dd; float* ruA = corners + 3 * dd;
    float* ldB = corners + 4 * dd; float* rdB = corners + 5 * dd;
    float* luB = corners + 6 * dd; float* ruB = corners + 7 * dd;
    for (int i = 1; i <= dn; ++i)        // column
        for (int j = 1; j <= dn; ++j) {  // row
            const size_t q = (size_t)(i - 1) * dn + (j - 1);
            const int k_rd = std::max(i, j);                    // below-right: kz = j, kx = i
            const int k_ld = std::max(j, dn - i + 1);           // below-left: kz = j, kx = dn-i+1
            const int k_lu = std::max(dn - j + 1, dn - i + 1);  // above-left
            const int k_ru = std::max(dn - j + 1, i);           // above-right
            rdA[q] = factorA[k_rd - 1]; rdB[q] = factorB[k_rd - 1];
            ldA[q] = factorA[k_ld - 1]; ldB[q] = factorB[k_ld - 1];
            luA[q] = factorA[k_lu - 1]; luB[q] = factorB[k_lu - 1];
            ruA[q] = factorA[k_ru - 1]; ruB[q] = factorB[k_ru - 1];
        }
}

void psdm_ricker_mcs(int32_t nt, float dt, float f0, float t0, float* S0) {
    const float pi = 3.14159265f;
    const float tmax = 10.f / f0;
    for (int i = 0; i < nt; ++i) {
        const float t = float(i) * dt;
        const float a = (pi * f0) * (t - t0);
        const float a2 = a * a;
        float s = (1.f - 2.f * a2) * expf(-(1.f * a2));
        if (t >= tmax) s = 0.f;
        S0[i] = s;
    }
}

void psdm_dynamic_window(int32_t NumRec, int32_t nxSou, const int32_t* nxRec, float dd, int32_t nx,
                         float dd_space, int32_t* nx_w, int32_t* x_i, int32_t* x_f) {
    const int ddx = 1 + (int)floorf(dd_space / dd);
    int lo = nxSou, hi = nxSou;
    for (int r = 0; r < NumRec; ++r) { lo = std::min(lo, (int)nxRec[r]); hi = std::max(hi, (int)nxRec[r]); }
    const int xi = std::max(1, lo - ddx + 1);
    const int xf = std::min((int)nx, hi + ddx);
    *x_i = xi;
    *x_f = xf;
    *nx_w = xf - xi + 1;
}

void psdm_trace_windows(const psdm_conditioning* c, int32_t NumRec, int32_t nxSou, int32_t nySou,
                        const int32_t* nxRec, const int32_t* nyRec, const float* Batmodel, float dmodel_prop,
                        float dt_prop, int32_t nt_prop, int32_t* nt_cut, int32_t* nt_sf, int32_t* lens) {
    // Defaults of calculate_PSDM_RTM.f90:123-124 and :64-65.
    for (int j = 0; j < NumRec; ++j) {
        nt_cut[j] = nt_prop;
        nt_sf[j] = 1;
    }
    // Half the source-receiver offset and the mean depth below source and
    // receiver of the sea floor at the midpoint: the legs of the sea-floor
    // reflection (:233-251 for the multiple, :259-277 for the direct wave).
    auto leg = [&](int j) {
        const float offset = fabsf(float(nxSou) * dmodel_prop - float(nxRec[j]) * dmodel_prop);
        const int mid_x = (int)ceilf(0.5f * float(nxSou + nxRec[j]));
        const float bat = Batmodel[mid_x - 1];
        const float D_src = bat - float(nySou) * dmodel_prop;
        const float D_rec = bat - float(nyRec[j]) * dmodel_prop;
        const float half = offset * 0.5f, depth = 0.5f * (D_src + D_rec);
        return sqrtf(half * half + depth * depth);
    };
    if (c->cut_multiple > 0)
        for (int j = 0; j < NumRec; ++j) nt_cut[j] = (int)ceilf((0.9f * ((4.0f * leg(j)) / 1500.f)) / dt_prop);
    if (c->cut_sf > 0)
        for (int j = 0; j < NumRec; ++j) nt_sf[j] = (int)ceilf((1.1f * ((2.0f * leg(j)) / 1500.f)) / dt_prop);
    int nt_prop2 = nt_prop, nt_taper = nt_prop, N_taper = 1, N_zeros = 0;
    if (c->taper_option != 0 || c->cut_multiple != 0) {  // :286-291
        N_taper = std::max(1, (int)(c->T_taper / dt_prop));
        N_zeros = std::max(0, (int)(c->T_zeros / dt_prop));
        int mx = NumRec > 0 ? nt_cut[0] : nt_prop;
        for (int j = 1; j < NumRec; ++j) mx = std::max(mx, (int)nt_cut[j]);
        nt_prop2 = std::min((int)nt_prop, mx);
        nt_taper = nt_prop2 + N_zeros;
    }
    lens[0] = nt_prop2;
    lens[1] = nt_taper;
    lens[2] = N_taper;
    lens[3] = N_zeros;
}

void psdm_taper_pad_trace(float* trace, int32_t nt_prop, int32_t N_taper, int32_t N_zeros, int32_t nt_new) {
    const int i0 = std::max(1, nt_prop - N_taper + 1);
    for (int n = 0; n < N_taper; ++n)
        if (i0 + n <= nt_prop) trace[i0 + n - 1] = trace[i0 + n - 1] * psdm::taper_weight(n, N_taper);
    if (N_zeros > 0)
        for (int i = nt_prop; i < nt_new; ++i) trace[i] = 0.f;
}

void psdm_optimization_dt(float dmodel_prop, float vmax, float tfin, int32_t store_snap, float* dt_prop,
                          int32_t* nt_prop, int32_t* nt_snap) {
    const float dt = (dmodel_prop / vmax) / 2.f;
    int ntp = 1 + (int)ceilf(tfin / dt);
    const int nts = (int)ceilf((1.f * float(ntp)) / float(store_snap));
    *dt_prop = dt;
    *nt_snap = nts;
    *nt_prop = nts * store_snap;
}

void psdm_normalize_psdm(int32_t nx, int32_t ny, const float* PSDM_sum, const float* Cov_sum, float* PSDM) {
    const size_t n = (size_t)nx * ny;
    for (size_t q = 0; q < n; ++q) PSDM[q] = (Cov_sum[q] > 0.f) ? PSDM_sum[q] / Cov_sum[q] : 0.f;
}

}  // extern "C"
