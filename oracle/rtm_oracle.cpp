// CPU oracle for the PSDM reverse-time-migration (RTM) propagators.
//
// TEST INFRASTRUCTURE ONLY.  The engine is checked against it; it is never the product:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// it.  The CUDA engine in psdm_b200/ never links or calls it.
//
// It is a step-by-step CPU restatement of the reference's Fortran solvers,
// keeping the reference's data structures (full-grid derivative arrays,
// strip-private PML histories, index vectors) and its floating-point
// evaluation order, so that an FP32 build reproduces the reference's
// arithmetic operation by operation.  It is templated on the real type: the
// float build restates the reference; the double build is the FP64 oracle for
// the mixed-precision engine.
//
// Parity status: the reference is Fortran 90 + MPI and no Fortran compiler
// exists on either machine, and the reference ships no tests, fixtures or
// data.  Parity with the reference's own outputs is therefore UNPINNED; the
// oracle is pinned instead by known-answer tests derived from the formulas
// (exact FD coefficients, closed-form PML profiles and Ricker wavelet, the
// analytic 2-D Green's function, mirror symmetry, PML reflection level, and
// FP32-vs-FP64 consistency) in tests/test_oracle_*.py.
//
// Reference files restated (paths inside the PSDM project):
//   src/solver_FD_coeffs.f90:1-73            finite_difference_coef
//   src/solver_PML_coeffs.f90:1-75           PML_coeffs
//   src/solver_space_derivs_clean.f90:1-140  space_deriv2x/2y, space_derivx/y
//   src/solver_PML_matrices.f90:1-111        pml_matrices_x/_y/_xycorner
//   src/solver_ac_forward_ram.f90:4-637      forward propagator, RAM strategy
//   src/solver_ac_backward_ram.f90:4-598     backward propagator + imaging
//   src/solver_ac_forward_disk.f90:294-312   disk-strategy model padding
//   src/solver_ac_forward_disk.f90:440-517   disk-strategy scatter order
//   src/dynamic_window.f90:1-183             window + solver wrappers
//   src/get_mcs_data.f90:318-351             Ricker_mcs
//   src/filters.f90:20-48                    taper_pad_trace
//   src/calculate_PSDM_RTM.f90:395-466       per-shot forward/taper/backward
//   src/auxiliar_PSDM.f90:1-20               normalize_psdm
//
// The mixed-precision form (MixedOpts, rtm_shot_mixed) has no reference
// counterpart: it restates the engine's FP16/BF16-snapshot form so that the
// float build checks the engine bit for bit and the double build is its FP64
// oracle.
//
// Build: oracle/Makefile (g++ -O3 -ffp-contract=off, no -ffast-math).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

// Column-major 2-D array with 1-based (row, col) access, as in Fortran.
template <class T>
struct Arr2 {
    std::vector<T> v;
    int n1 = 0, n2 = 0;
    Arr2() = default;
    Arr2(int a, int b) : v((size_t)a * (size_t)b, T(0)), n1(a), n2(b) {}
    inline T& operator()(int j, int i) { return v[(size_t)(i - 1) * n1 + (j - 1)]; }
    inline const T& operator()(int j, int i) const { return v[(size_t)(i - 1) * n1 + (j - 1)]; }
    void zero() { std::fill(v.begin(), v.end(), T(0)); }
};

// src/solver_FD_coeffs.f90:1-73.  coef has acc+1 entries (1-based in the
// reference, 0-based here).  The second-derivative centre tap is halved
// (:68) because the stencil applies it as p(i)+p(i).
template <class T>
void fd_coef(int num, int acc, T* coef) {
    for (int i = 0; i <= acc; ++i) coef[i] = T(0);
    if (num == 1) {
        if (acc == 1) { coef[0] = T(0); coef[1] = T(0); /* 1/2 is integer division in the reference: 0 */ }
        if (acc == 3) { coef[0] = T(0); coef[1] = T(3) / T(4); coef[2] = T(-3) / T(20); coef[3] = T(1) / T(60); }
        if (acc == 4) { coef[0] = T(0); coef[1] = T(4) / T(5); coef[2] = T(-1) / T(5); coef[3] = T(4) / T(105); coef[4] = T(-1) / T(280); }
        if (acc == 5) { for (int i = 0; i <= 5; ++i) coef[i] = T(0); }
    }
    if (num == 2) {
        if (acc == 3) { coef[0] = T(-49) / T(18); coef[1] = T(3) / T(2); coef[2] = T(-3) / T(20); coef[3] = T(1) / T(90); }
        if (acc == 4) { coef[0] = T(-205) / T(72); coef[1] = T(8) / T(5); coef[2] = T(-1) / T(5); coef[3] = T(8) / T(315); coef[4] = T(-1) / T(560); }
        if (acc == 5) { coef[0] = T(-5269) / T(1800); coef[1] = T(5) / T(3); coef[2] = T(-5) / T(21); coef[3] = T(5) / T(126); coef[4] = T(-5) / T(1008); coef[5] = T(1) / T(3150); }
        coef[0] = coef[0] / T(2);
    }
}

template <class T> inline T t_exp(T x);
template <> inline float t_exp<float>(float x) { return expf(x); }
template <> inline double t_exp<double>(double x) { return exp(x); }
template <class T> inline T t_log(T x);
template <> inline float t_log<float>(float x) { return logf(x); }
template <> inline double t_log<double>(double x) { return log(x); }
template <class T> inline T t_cos(T x);
template <> inline float t_cos<float>(float x) { return cosf(x); }
template <> inline double t_cos<double>(double x) { return cos(x); }
template <class T> inline T t_atan(T x);
template <> inline float t_atan<float>(float x) { return atanf(x); }
template <> inline double t_atan<double>(double x) { return atan(x); }

// src/solver_PML_coeffs.f90:1-75.  factorA/B are zero for i <= acc (the
// caller zero-initialises them, solver_ac_forward_ram.f90:166) and hold the
// last profile value beyond dPML+acc.  Corner matrices are (dn x dn),
// column-major, 1-based.
template <class T>
void pml_coeffs(int acc, int dPML, T dt, T d, int dn, T* fA, T* fB,
                Arr2<T>& ldA, Arr2<T>& rdA, Arr2<T>& luA, Arr2<T>& ruA,
                Arr2<T>& ldB, Arr2<T>& rdB, Arr2<T>& luB, Arr2<T>& ruB) {
    // fA, fB: 1-based arrays of length dn passed as pointer to element 1.
    std::vector<T> yPML(dn + 1, T(0)), alpha(dn + 1, T(0)), sigma(dn + 1, T(0));
    const T pi = T(3.14159265);
    const T Refl = T(0.00001);
    const T wPML = T(dPML - 1) * d;
    for (int i = 1 + acc; i <= dPML + acc; ++i) {
        yPML[i] = T(i - (acc + 1)) * d;
        alpha[i] = T(30) * pi * (T(1) - (yPML[i] / wPML));
        const T r = yPML[i] / wPML;
        sigma[i] = (-((T(6000) * t_log<T>(Refl)) / (T(2) * wPML))) * (r * r);
    }
    for (int i = 1 + acc; i <= dPML + acc; ++i) {
        fA[i - 1] = t_exp<T>(-((sigma[i] + alpha[i]) * dt));
        fB[i - 1] = ((fA[i - 1] - T(1)) * sigma[i]) / (sigma[i] + alpha[i]);
    }
    for (int i = dPML + acc + 1; i <= dn; ++i) {
        fA[i - 1] = fA[dPML + acc - 1];
        fB[i - 1] = fB[dPML + acc - 1];
    }
    for (int i = 1; i <= dn; ++i)
        for (int j = 1; j <= i; ++j) { rdA(j, i) = fA[i - 1]; rdB(j, i) = fB[i - 1]; }
    for (int i = 1; i <= dn; ++i)
        if (i + 1 <= dn)
            for (int j = i + 1; j <= dn; ++j) { rdA(j, i) = rdA(i, j); rdB(j, i) = rdB(i, j); }
    for (int i = 1; i <= dn; ++i)
        for (int j = 1; j <= dn - i + 1; ++j) { ldA(j, i) = fA[dn - i]; ldB(j, i) = fB[dn - i]; }
    for (int ix = 1; ix <= dn - 1; ++ix) {
        const int j = 2 + (ix - 1);
        for (int i = dn - (ix - 1); i <= dn; ++i) { ldA(j, i) = fA[j - 1]; ldB(j, i) = fB[j - 1]; }
    }
    for (int j = 1; j <= dn; ++j)
        for (int i = 1; i <= dn; ++i) {
            luA(j, i) = ldA(dn - j + 1, i); luB(j, i) = ldB(dn - j + 1, i);
            ruA(j, i) = rdA(dn - j + 1, i); ruB(j, i) = rdB(dn - j + 1, i);
        }
}

// src/solver_space_derivs_clean.f90:1-37 (k outer, accumulate from zero).
template <class T>
void space_deriv2x(int acc, const T* coef, int nyt, int nxt, const Arr2<T>& p, Arr2<T>& d) {
    const int i1 = 1 + acc, i2 = nxt - acc;
    d.zero();
    for (int k = 1; k <= acc + 1; ++k)
        for (int i = i1; i <= i2; ++i)
            for (int j = 1; j <= nyt; ++j)
                d(j, i) = d(j, i) + (p(j, i + (k - 1)) + p(j, i - (k - 1))) * coef[k - 1];
    for (int i = 1; i <= i1 - 1; ++i)
        for (int j = 1; j <= nyt; ++j) d(j, i) = d(j, acc + 1);
    for (int i = i2 + 1; i <= nxt; ++i)
        for (int j = 1; j <= nyt; ++j) d(j, i) = d(j, nxt - acc);
}

// src/solver_space_derivs_clean.f90:39-69.
template <class T>
void space_deriv2y(int acc, const T* coef, int nyt, int nxt, const Arr2<T>& p, Arr2<T>& d) {
    const int j1 = 1 + acc, j2 = nyt - acc;
    d.zero();
    for (int i = 1; i <= nxt; ++i) {
        for (int j = j1; j <= j2; ++j)
            for (int k = 1; k <= acc + 1; ++k)
                d(j, i) = d(j, i) + (p(j + (k - 1), i) + p(j - (k - 1), i)) * coef[k - 1];
        for (int j = 1; j <= j1 - 1; ++j) d(j, i) = d(acc + 1, i);
        for (int j = 1 + j2; j <= nyt; ++j) d(j, i) = d(nyt - acc, i);
    }
}

// src/solver_space_derivs_clean.f90:71-107.
template <class T>
void space_derivx(int acc, const T* coef, int nyt, int nxt, const Arr2<T>& p, Arr2<T>& d) {
    const int i1 = 1 + acc, i2 = nxt - acc;
    d.zero();
    for (int k = 1; k <= acc + 1; ++k)
        for (int i = i1; i <= i2; ++i)
            for (int j = 1; j <= nyt; ++j)
                d(j, i) = d(j, i) + (p(j, i + (k - 1)) - p(j, i - (k - 1))) * coef[k - 1];
    for (int i = 1; i <= i1 - 1; ++i)
        for (int j = 1; j <= nyt; ++j) d(j, i) = d(j, acc + 1);
    for (int i = 1 + i2; i <= nxt; ++i)
        for (int j = 1; j <= nyt; ++j) d(j, i) = d(j, nxt - acc);
}

// src/solver_space_derivs_clean.f90:109-140.
template <class T>
void space_derivy(int acc, const T* coef, int nyt, int nxt, const Arr2<T>& p, Arr2<T>& d) {
    const int j1 = 1 + acc, j2 = nyt - acc;
    d.zero();
    for (int i = 1; i <= nxt; ++i) {
        for (int j = j1; j <= j2; ++j)
            for (int k = 1; k <= acc + 1; ++k)
                d(j, i) = d(j, i) + (p(j + (k - 1), i) - p(j - (k - 1), i)) * coef[k - 1];
        for (int j = 1; j <= j1 - 1; ++j) d(j, i) = d(acc + 1, i);
        for (int j = 1 + j2; j <= nyt; ++j) d(j, i) = d(nyt - acc, i);
    }
}

// One C-PML strip or corner with its private histories.
template <class T>
struct Strip {
    int ny = 0, nx = 0;
    Arr2<T> p1, p, p3;                   // *_pml_p_1, *_pml_p, *_pml_p_3
    Arr2<T> phx1, phx, chx1, chx;        // phi/chi along x
    Arr2<T> phy1, phy, chy1, chy;        // phi/chi along y (z)
    void init(int a, int b) {
        ny = a; nx = b;
        p1 = Arr2<T>(a, b); p = Arr2<T>(a, b); p3 = Arr2<T>(a, b);
        phx1 = Arr2<T>(a, b); phx = Arr2<T>(a, b); chx1 = Arr2<T>(a, b); chx = Arr2<T>(a, b);
        phy1 = Arr2<T>(a, b); phy = Arr2<T>(a, b); chy1 = Arr2<T>(a, b); chy = Arr2<T>(a, b);
    }
    // Time actualisation, solver_ac_forward_ram.f90:512-565.
    void rotate() {
        p1.v = p.v; p.v = p3.v;
        phx1.v = phx.v; chx1.v = chx.v;
        phy1.v = phy.v; chy1.v = chy.v;
    }
};

// src/solver_PML_matrices.f90:1-39 (pml_matrices_x).  idir 1: factor index i
// (strip column, 1 adjacent to the interior); idir 2: factor nvx-i+1.
template <class T>
void pml_matrices_x(int idir, int acc, const T* coef1, int nvy, int nvx,
                    const std::vector<int>& vy, const std::vector<int>& vx,
                    const T* fA, const T* fB, const Arr2<T>& deriv, const Arr2<T>& deriv2,
                    Arr2<T>& phi, const Arr2<T>& phi_1, Arr2<T>& chi, const Arr2<T>& chi_1,
                    Arr2<T>& prop) {
    Arr2<T> dphi(nvy, nvx);
    prop.zero();
    space_derivx<T>(acc, coef1, nvy, nvx, phi, dphi);
    for (int i = 1; i <= nvx; ++i) {
        const int fi = (idir == 1) ? i : (nvx - i + 1);
        const T A = fA[fi - 1], B = fB[fi - 1];
        for (int j = 1; j <= nvy; ++j) {
            phi(j, i) = A * phi_1(j, i) + B * deriv(vy[j - 1], vx[i - 1]);
            chi(j, i) = A * chi_1(j, i) + B * (deriv2(vy[j - 1], vx[i - 1]) + dphi(j, i));
        }
    }
    for (size_t q = 0; q < prop.v.size(); ++q) prop.v[q] = dphi.v[q] + chi.v[q];
}

// src/solver_PML_matrices.f90:41-80 (pml_matrices_y).
template <class T>
void pml_matrices_y(int idir, int acc, const T* coef1, int nvy, int nvx,
                    const std::vector<int>& vy, const std::vector<int>& vx,
                    const T* fA, const T* fB, const Arr2<T>& deriv, const Arr2<T>& deriv2,
                    Arr2<T>& phi, const Arr2<T>& phi_1, Arr2<T>& chi, const Arr2<T>& chi_1,
                    Arr2<T>& prop) {
    Arr2<T> dphi(nvy, nvx);
    prop.zero();
    space_derivy<T>(acc, coef1, nvy, nvx, phi, dphi);
    for (int i = 1; i <= nvx; ++i)
        for (int j = 1; j <= nvy; ++j) {
            const int fj = (idir == 1) ? j : (nvy - j + 1);
            const T A = fA[fj - 1], B = fB[fj - 1];
            phi(j, i) = A * phi_1(j, i) + B * deriv(vy[j - 1], vx[i - 1]);
            chi(j, i) = A * chi_1(j, i) + B * (deriv2(vy[j - 1], vx[i - 1]) + dphi(j, i));
        }
    for (size_t q = 0; q < prop.v.size(); ++q) prop.v[q] = dphi.v[q] + chi.v[q];
}

// src/solver_PML_matrices.f90:82-111 (pml_matrices_xycorner); id 1 = x, 2 = y.
template <class T>
void pml_matrices_corner(int id, int acc, const T* coef1, int nvy, int nvx,
                         const std::vector<int>& vy, const std::vector<int>& vx,
                         const Arr2<T>& fA, const Arr2<T>& fB, const Arr2<T>& deriv, const Arr2<T>& deriv2,
                         Arr2<T>& phi, const Arr2<T>& phi_1, Arr2<T>& chi, const Arr2<T>& chi_1,
                         Arr2<T>& prop) {
    Arr2<T> dphi(nvy, nvx);
    prop.zero();
    if (id == 1) space_derivx<T>(acc, coef1, nvy, nvx, phi, dphi);
    if (id == 2) space_derivy<T>(acc, coef1, nvy, nvx, phi, dphi);
    for (int i = 1; i <= nvx; ++i)
        for (int j = 1; j <= nvy; ++j) {
            phi(j, i) = fA(j, i) * phi_1(j, i) + fB(j, i) * deriv(vy[j - 1], vx[i - 1]);
            chi(j, i) = fA(j, i) * chi_1(j, i) + fB(j, i) * (deriv2(vy[j - 1], vx[i - 1]) + dphi(j, i));
        }
    for (size_t q = 0; q < prop.v.size(); ++q) prop.v[q] = dphi.v[q] + chi.v[q];
}

// S3 = -S1 + 2 S + c2 (d2x + d2y + prop) on a strip (solver_ac_forward_ram.f90:376-438).
template <class T>
void strip_update(Strip<T>& s, const std::vector<int>& vy, const std::vector<int>& vx,
                  const Arr2<T>& c2, const Arr2<T>& d2x, const Arr2<T>& d2y, const Arr2<T>& prop) {
    for (int i = 1; i <= s.nx; ++i)
        for (int j = 1; j <= s.ny; ++j) {
            const int y = vy[j - 1], x = vx[i - 1];
            s.p3(j, i) = (-s.p1(j, i) + T(2) * s.p(j, i)) + c2(y, x) * ((d2x(y, x) + d2y(y, x)) + prop(j, i));
        }
}

// Corner second direction: S3 = S3 + c2 * prop (solver_ac_forward_ram.f90:407,416,429,438).
template <class T>
void strip_add(Strip<T>& s, const std::vector<int>& vy, const std::vector<int>& vx,
               const Arr2<T>& c2, const Arr2<T>& prop) {
    for (int i = 1; i <= s.nx; ++i)
        for (int j = 1; j <= s.ny; ++j)
            s.p3(j, i) = s.p3(j, i) + c2(vy[j - 1], vx[i - 1]) * prop(j, i);
}

template <class T>
void scatter(Arr2<T>& p3, const Strip<T>& s, const std::vector<int>& vy, const std::vector<int>& vx) {
    for (int i = 1; i <= s.nx; ++i)
        for (int j = 1; j <= s.ny; ++j) p3(vy[j - 1], vx[i - 1]) = s.p3(j, i);
}

// ---- mixed-precision form (no reference counterpart) ------------------------
//
// Options of the engine's mixed-precision form, restated here so that the
// float build emulates the engine bit for bit and the double build is its
// FP64 oracle:
//   pair_mode 1: snapshots every store_snap forward steps (slot m at forward
//     step k = store_snap*m + 1, as the reference stores them) and imaging at
//     the backward steps paired with them in time, k_b = nt + 1 - store_snap*m
//     (for store_snap = 1 this is the reference's pairing);
//   q16: snapshots rounded to binary16 (1) or bfloat16 (2) after scaling by a
//     power of two 2^k chosen from the snapshot's largest magnitude A so that
//     A*2^k lies in [2^14, 2^15); read back as float(h) * 2^-k;
//   kahan: the image is summed with compensated (Kahan) summation.
//   coef64: the float build takes its FD coefficients and C-PML profiles
//     from the double-precision set-up, rounded once (the engine's set-up of
//     the form).
struct MixedOpts {
    int pair_mode = 0;
    int q16 = 0;
    int kahan = 0;
    int coef64 = 0;
};

// x rounded to the nearest binary16 (mant = 10, emin = -14) or bfloat16
// (mant = 7, emin = -126) value, ties to even, returned as a float; |x| is
// far below either format's overflow threshold here.
inline float round_to_format(float x, int mant, int emin) {
    const double a = std::fabs((double)x);
    if (a == 0.0) return x;
    int e = 0;
    std::frexp(a, &e);  // a = f * 2^e, f in [0.5, 1)
    const int E = std::max(e - 1, emin);
    const double ulp = std::ldexp(1.0, E - mant);
    const double q = std::nearbyint(a / ulp) * ulp;  // a / ulp is exact
    return (float)std::copysign(q, (double)x);
}

// Scale exponent k for a snapshot whose largest magnitude is amax.
inline int snapshot_scale_exp(float amax) {
    if (!(amax > 0.f)) return 0;
    uint32_t b;
    std::memcpy(&b, &amax, 4);
    const int E = (int)((b >> 23) & 0xffu) - 127;  // floor(log2 amax); -127 for subnormals
    return std::min(126, std::max(-126, 14 - E));
}

inline float pow2f(int k) {
    uint32_t b = (uint32_t)(k + 127) << 23;  // k in [-126, 127]
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

// Quantize one snapshot in place (float build only).
template <class T>
void quantize_snapshot(T* F, size_t n, int q16) {
    if (q16 == 0 || sizeof(T) != sizeof(float)) return;
    float amax = 0.f;
    for (size_t i = 0; i < n; ++i) amax = std::max(amax, (float)std::fabs((float)F[i]));
    const int k = snapshot_scale_exp(amax);
    const float sc = pow2f(k), isc = pow2f(-k);
    const int mant = q16 == 1 ? 10 : 7, emin = q16 == 1 ? -14 : -126;
    for (size_t i = 0; i < n; ++i) F[i] = (T)(round_to_format((float)F[i] * sc, mant, emin) * isc);
}

// The propagator, src/solver_ac_forward_ram.f90:4-637 (iprop = 1) and
// src/solver_ac_backward_ram.f90:4-598 (iprop = 2).  disk_mode = 1 follows
// the disk variants' order (solver_ac_forward_disk.f90:506-517), in which the
// strips are scattered after the free-surface row is zeroed.
//
// Geometry is in window coordinates (1-based, as the dynamic_window wrappers
// pass it).  Forward: S(nt) single source, Rec_point(nt, NumRec) out,
// Fields(ny, nx, nt_snap) out.  Backward: Sadj(nt, NumRec) in,
// Fields(ny, nx, nt_snap) in, kernel(ny, nx) accumulated.
template <class T>
void solver_ac(int iprop, int disk_mode, int dPML, int fs, int NumRec,
               const int* nxSou, const int* nySou, const int* nxRec, const int* nyRec,
               const T* S /*forward: S(nt); backward: Sadj(nt,NumRec)*/,
               T dmodel, T dt, int ny, int nx, const T* ctmp_in,
               int store_snap, int nt_snap, int nt, T* Fields, T* out /*Rec or kernel*/,
               T* p_dump = nullptr /*(nyt, nxt) padded p after the last step, optional*/,
               const MixedOpts* mo = nullptr /*mixed-precision form; null = the reference*/,
               const T* mixed_weights = nullptr /*mixed form: weight of slot m at [m-1], or null*/) {
    const int acc = 3;
    const int dn = dPML + 2 * acc;
    const int dnx = dn, dny = dn, dny2 = dn;
    const int free_surface = fs;

    std::vector<int> nxs, nys, nxreco(NumRec), nyreco(NumRec);
    if (iprop == 1) {
        nxs = {dn + nxSou[0]}; nys = {dny2 + nySou[0]};
        for (int r = 0; r < NumRec; ++r) { nxreco[r] = dn + nxRec[r]; nyreco[r] = dny2 + nyRec[r]; }
    } else {
        nxs.resize(NumRec); nys.resize(NumRec);
        for (int r = 0; r < NumRec; ++r) { nxs[r] = dn + nxRec[r]; nys[r] = dny2 + nyRec[r]; }
    }
    const int nxt = nx + 2 * dn;
    const int nyt = dny2 + ny + dn;

    std::vector<int> mx(nx), my(ny), yu(dny2), yd(dny), xl(dnx), xr(dnx);
    for (int i = 0; i < nx; ++i) mx[i] = dnx + 1 + i;
    for (int i = 0; i < ny; ++i) my[i] = dny2 + 1 + i;
    for (int i = 0; i < dny2; ++i) yu[i] = 1 + i;
    for (int i = 0; i < dny; ++i) yd[i] = dny2 + ny + 1 + i;
    for (int i = 0; i < dnx; ++i) xl[i] = 1 + i;
    for (int i = 0; i < dnx; ++i) xr[i] = dnx + nx + 1 + i;

    std::vector<T> coef1(acc + 1), coef2(acc + 1);
    Arr2<T> source(nyt, nxt), p_1(nyt, nxt), p(nyt, nxt), p_3(nyt, nxt), c2(nyt, nxt);
    Arr2<T> d2x(nyt, nxt), d2y(nyt, nxt), d1x(nyt, nxt), d1y(nyt, nxt);
    Arr2<T> x_prop(ny, dn), y_prop(dn, nx), corner_prop(dn, dn);
    std::vector<T> fA(dn, T(0)), fB(dn, T(0));
    Arr2<T> luA(dn, dn), luB(dn, dn), ruA(dn, dn), ruB(dn, dn), ldA(dn, dn), ldB(dn, dn), rdA(dn, dn), rdB(dn, dn);
    Strip<T> syu, syd, sxl, sxr, slu, sru, sld, srd;
    syu.init(dn, nx); syd.init(dn, nx); sxl.init(ny, dn); sxr.init(ny, dn);
    slu.init(dn, dn); sru.init(dn, dn); sld.init(dn, dn); srd.init(dn, dn);

    // Model padding; c2, solver_ac_forward_ram.f90:319.
    {
        Arr2<T> c(nyt, nxt);
        auto ct = [&](int j, int i) { return ctmp_in[(size_t)(i - 1) * ny + (j - 1)]; };
        if (!disk_mode) {
            // RAM solvers, solver_ac_forward_ram.f90:282-309.  The top and
            // bottom loops run j = 1..dnx only, so c stays 0 in those strips
            // beyond the first dn interior columns.
            for (int j = 1; j <= nx; ++j) for (int i = 1; i <= ny; ++i) c(dny2 + i, dnx + j) = ct(i, j);
            for (int j = 1; j <= dnx; ++j) for (int i = 1; i <= dny2; ++i) {
                c(i, j) = ct(1, 1); c(i, dnx + j) = ct(1, j); c(i, dnx + nx + j) = ct(1, nx);
            }
            for (int j = 1; j <= dnx; ++j) for (int i = 1; i <= dny; ++i) {
                c(i + dny2 + ny, dnx + j) = ct(ny, j); c(i + dny2 + ny, j) = ct(ny, 1); c(i + dny2 + ny, dnx + nx + j) = ct(ny, nx);
            }
            for (int j = 1; j <= dnx; ++j) for (int i = 1; i <= ny; ++i) {
                c(dny2 + i, j) = ct(i, 1); c(dny2 + i, dnx + nx + j) = ct(i, nx);
            }
        } else {
            // Disk solvers, solver_ac_forward_disk.f90:294-312 (full width).
            for (int j = 1; j <= nx; ++j) for (int i = 1; i <= ny; ++i) c(dny2 + i, dnx + j) = ct(i, j);
            for (int i = 1; i <= dny2; ++i) {
                for (int j = 1; j <= nx; ++j) c(i, dnx + j) = ct(1, j);
                for (int j = 1; j <= dnx; ++j) { c(i, j) = ct(1, 1); c(i, dnx + nx + j) = ct(1, nx); }
            }
            for (int i = dny2 + ny + 1; i <= dny2 + ny + dny; ++i) {
                for (int j = 1; j <= nx; ++j) c(i, dn + j) = ct(ny, j);
                for (int j = 1; j <= dn; ++j) { c(i, j) = ct(ny, 1); c(i, dnx + nx + j) = ct(ny, nx); }
            }
            for (int i = 1; i <= dnx; ++i)
                for (int j = 1; j <= ny; ++j) { c(dny2 + j, i) = ct(j, 1); c(dny2 + j, dnx + nx + i) = ct(j, nx); }
        }
        for (size_t q = 0; q < c.v.size(); ++q) c2.v[q] = ((c.v[q] * c.v[q]) * (dt * dt)) / (dmodel * dmodel);
    }

    pml_coeffs<T>(acc, dPML, dt, dmodel, dn, fA.data(), fB.data(), ldA, rdA, luA, ruA, ldB, rdB, luB, ruB);

    int l = 0;
    int snap = (iprop == 1) ? 0 : nt_snap;
    fd_coef<T>(1, acc, coef1.data());
    fd_coef<T>(2, acc, coef2.data());
    if (mo && mo->coef64 && sizeof(T) == sizeof(float)) {
        std::vector<double> a64(dn, 0.0), b64(dn, 0.0), c1(acc + 1), c2(acc + 1);
        Arr2<double> t[8] = {Arr2<double>(dn, dn), Arr2<double>(dn, dn), Arr2<double>(dn, dn), Arr2<double>(dn, dn),
                             Arr2<double>(dn, dn), Arr2<double>(dn, dn), Arr2<double>(dn, dn), Arr2<double>(dn, dn)};
        pml_coeffs<double>(acc, dPML, double(dt), double(dmodel), dn, a64.data(), b64.data(), t[0], t[1], t[2], t[3],
                           t[4], t[5], t[6], t[7]);
        Arr2<T>* dst[8] = {&ldA, &rdA, &luA, &ruA, &ldB, &rdB, &luB, &ruB};
        for (int q = 0; q < 8; ++q)
            for (size_t i = 0; i < dst[q]->v.size(); ++i) dst[q]->v[i] = T(t[q].v[i]);
        for (int i = 0; i < dn; ++i) { fA[i] = T(a64[i]); fB[i] = T(b64[i]); }
        fd_coef<double>(1, acc, c1.data());
        fd_coef<double>(2, acc, c2.data());
        for (int k = 0; k <= acc; ++k) { coef1[k] = T(c1[k]); coef2[k] = T(c2[k]); }
    }

    if (iprop == 1)
        for (size_t q = 0; q < (size_t)nt * NumRec; ++q) out[q] = T(0);

    const size_t fstride = (size_t)ny * nx;
    std::vector<T> comp((mo && mo->kahan && iprop == 2) ? fstride : 0, T(0));
    const T* mixed_w = mixed_weights;
    for (int k = 2; k <= nt; ++k) {
        l = l + 1;
        if (iprop == 1) source(nys[0], nxs[0]) = S[k - 2];
        if (iprop == 2)
            for (int j = 0; j < NumRec; ++j) source(nys[j], nxs[j]) = S[(size_t)j * nt + (k - 2)];

        space_deriv2x<T>(acc, coef2.data(), nyt, nxt, p, d2x);
        space_deriv2y<T>(acc, coef2.data(), nyt, nxt, p, d2y);
        space_derivx<T>(acc, coef1.data(), nyt, nxt, p, d1x);
        space_derivy<T>(acc, coef1.data(), nyt, nxt, p, d1y);

        pml_matrices_x<T>(1, acc, coef1.data(), ny, dn, my, xr, fA.data(), fB.data(), d1x, d2x, sxr.phx, sxr.phx1, sxr.chx, sxr.chx1, x_prop);
        strip_update<T>(sxr, my, xr, c2, d2x, d2y, x_prop);
        pml_matrices_x<T>(2, acc, coef1.data(), ny, dn, my, xl, fA.data(), fB.data(), d1x, d2x, sxl.phx, sxl.phx1, sxl.chx, sxl.chx1, x_prop);
        strip_update<T>(sxl, my, xl, c2, d2x, d2y, x_prop);
        pml_matrices_y<T>(1, acc, coef1.data(), dn, nx, yd, mx, fA.data(), fB.data(), d1y, d2y, syd.phy, syd.phy1, syd.chy, syd.chy1, y_prop);
        strip_update<T>(syd, yd, mx, c2, d2x, d2y, y_prop);

        if (free_surface == 0) {
            pml_matrices_y<T>(2, acc, coef1.data(), dn, nx, yu, mx, fA.data(), fB.data(), d1y, d2y, syu.phy, syu.phy1, syu.chy, syu.chy1, y_prop);
            strip_update<T>(syu, yu, mx, c2, d2x, d2y, y_prop);
            pml_matrices_corner<T>(1, acc, coef1.data(), dn, dn, yu, xl, luA, luB, d1x, d2x, slu.phx, slu.phx1, slu.chx, slu.chx1, corner_prop);
            strip_update<T>(slu, yu, xl, c2, d2x, d2y, corner_prop);
            pml_matrices_corner<T>(2, acc, coef1.data(), dn, dn, yu, xl, luA, luB, d1y, d2y, slu.phy, slu.phy1, slu.chy, slu.chy1, corner_prop);
            strip_add<T>(slu, yu, xl, c2, corner_prop);
            pml_matrices_corner<T>(1, acc, coef1.data(), dn, dn, yu, xr, ruA, ruB, d1x, d2x, sru.phx, sru.phx1, sru.chx, sru.chx1, corner_prop);
            strip_update<T>(sru, yu, xr, c2, d2x, d2y, corner_prop);
            pml_matrices_corner<T>(2, acc, coef1.data(), dn, dn, yu, xr, ruA, ruB, d1y, d2y, sru.phy, sru.phy1, sru.chy, sru.chy1, corner_prop);
            strip_add<T>(sru, yu, xr, c2, corner_prop);
        }

        pml_matrices_corner<T>(1, acc, coef1.data(), dn, dn, yd, xl, ldA, ldB, d1x, d2x, sld.phx, sld.phx1, sld.chx, sld.chx1, corner_prop);
        strip_update<T>(sld, yd, xl, c2, d2x, d2y, corner_prop);
        pml_matrices_corner<T>(2, acc, coef1.data(), dn, dn, yd, xl, ldA, ldB, d1y, d2y, sld.phy, sld.phy1, sld.chy, sld.chy1, corner_prop);
        strip_add<T>(sld, yd, xl, c2, corner_prop);
        pml_matrices_corner<T>(1, acc, coef1.data(), dn, dn, yd, xr, rdA, rdB, d1x, d2x, srd.phx, srd.phx1, srd.chx, srd.chx1, corner_prop);
        strip_update<T>(srd, yd, xr, c2, d2x, d2y, corner_prop);
        pml_matrices_corner<T>(2, acc, coef1.data(), dn, dn, yd, xr, rdA, rdB, d1y, d2y, srd.phy, srd.phy1, srd.chy, srd.chy1, corner_prop);
        strip_add<T>(srd, yd, xr, c2, corner_prop);

        // Interior, solver_ac_forward_ram.f90:443-444.
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const int y = my[j], x = mx[i];
                p_3(y, x) = (-p_1(y, x) + T(2) * p(y, x)) + ((d2x(y, x) + d2y(y, x)) + source(y, x)) * c2(y, x);
            }

        auto scatter_all = [&]() {
            scatter<T>(p_3, syu, yu, mx); scatter<T>(p_3, slu, yu, xl); scatter<T>(p_3, sru, yu, xr);
            scatter<T>(p_3, syd, yd, mx); scatter<T>(p_3, sld, yd, xl); scatter<T>(p_3, srd, yd, xr);
            scatter<T>(p_3, sxl, my, xl); scatter<T>(p_3, sxr, my, xr);
        };
        if (!disk_mode) scatter_all();

        // Free surface, :463-473.
        if (free_surface != 0)
            for (int i = 1; i <= nxt; ++i) p_3(1 + dny2, i) = T(0);

        if (iprop == 1 && l == store_snap) {
            snap = snap + 1;
            T* F = Fields + (size_t)(snap - 1) * fstride;
            for (int i = 1; i <= nx; ++i)
                for (int j = 1; j <= ny; ++j)
                    F[(size_t)(i - 1) * ny + (j - 1)] = ((p_3(dny2 + j, dnx + i) - p_1(dny2 + j, dnx + i)) * T(0.5)) / dt;
            if (mo) quantize_snapshot<T>(F, fstride, mo->q16);
            l = 0;
        }
        if (iprop == 2 && mo && mo->pair_mode == 1) {
            // Mixed form: slot m pairs with backward step k = nt + 1 - store_snap*m.
            const int r = nt + 1 - k;
            const int m = (r % store_snap == 0) ? r / store_snap : 0;
            if (m >= 1 && m <= nt_snap) {
                const T* F = Fields + (size_t)(m - 1) * fstride;
                const T ss = T(store_snap);
                for (int i = 1; i <= nx; ++i)
                    for (int j = 1; j <= ny; ++j) {
                        const size_t q = (size_t)(i - 1) * ny + (j - 1);
                        if (mixed_w && mixed_w[m - 1] == T(0)) continue;
                        T Fv = F[q];
                        if (mixed_w && mixed_w[m - 1] != T(1)) Fv = Fv * mixed_w[m - 1];
                        const T inc = ((T(0.5) * (p_3(dny2 + j, dnx + i) - p_1(dny2 + j, dnx + i))) * Fv) * ss;
                        T& kk = out[q];
                        if (mo->kahan) {
                            T& cc = comp[q];
                            const T y = inc - cc;
                            const T t = kk + y;
                            cc = (t - kk) - y;
                            kk = t;
                        } else {
                            kk = kk + inc;
                        }
                    }
            }
        } else if (iprop == 2 && l == store_snap) {
            snap = snap - 1;
            const T* F = Fields + (size_t)(snap - 1) * fstride;
            const T ss = T(store_snap);
            for (int i = 1; i <= nx; ++i)
                for (int j = 1; j <= ny; ++j) {
                    T& kk = out[(size_t)(i - 1) * ny + (j - 1)];
                    kk = kk + ((T(0.5) * (p_3(dny2 + j, dnx + i) - p_1(dny2 + j, dnx + i))) * F[(size_t)(i - 1) * ny + (j - 1)]) * ss;
                }
            l = 0;
        }

        if (disk_mode) scatter_all();

        p_1.v = p.v;
        p.v = p_3.v;
        syu.rotate(); syd.rotate(); sxl.rotate(); sxr.rotate();
        slu.rotate(); sru.rotate(); sld.rotate(); srd.rotate();

        if (iprop != 2)
            for (int r = 0; r < NumRec; ++r) out[(size_t)r * nt + (k - 2)] = p_3(nyreco[r], nxreco[r]);
    }
    if (iprop == 1)
        for (int r = 0; r < NumRec; ++r) out[(size_t)r * nt + (nt - 1)] = out[(size_t)r * nt + (nt - 2)];
    if (p_dump) std::copy(p.v.begin(), p.v.end(), p_dump);
}

// src/dynamic_window.f90:1-52 with NumSou = 1.
void dynamic_window(int NumRec, int nxSou, const int* nxRec, float dd, int nx, float dd_space,
                    int* nx_w, int* x_i, int* x_f) {
    const int ddx = 1 + (int)std::floor(dd_space / dd);
    int mn = nxSou, mx = nxSou;
    for (int r = 0; r < NumRec; ++r) { mn = std::min(mn, nxRec[r]); mx = std::max(mx, nxRec[r]); }
    int xi = mn - ddx + 1;
    if (xi <= 0) xi = 1;
    int xf = mx + ddx;
    if (xf > nx) xf = nx;
    *x_i = xi; *x_f = xf; *nx_w = xf - xi + 1;
}

// src/filters.f90:20-48.
template <class T>
void taper_pad_trace(T* trace, int nt_prop, int N_taper, int N_zeros, int nt_new) {
    const T pi = T(4) * t_atan<T>(T(1));
    const int i0 = std::max(1, nt_prop - N_taper + 1);
    for (int n = 0; n <= N_taper - 1; ++n)
        if (i0 + n <= nt_prop) {
            const T w = T(0.5) * (T(1) + t_cos<T>((pi * T(n)) / T(N_taper)));
            trace[i0 + n - 1] = trace[i0 + n - 1] * w;
        }
    if (N_zeros > 0)
        for (int i = nt_prop + 1; i <= nt_new; ++i) trace[i - 1] = T(0);
}

// The per-shot block of src/calculate_PSDM_RTM.f90:395-466 (RAM strategy or
// disk-strategy ordering): forward, optional Fields taper, time-reversed
// back-source, backward with imaging.  Geometry is in model coordinates; the
// window is recomputed as the dynamic_window wrappers do.
template <class T>
void rtm_shot(int disk_mode, int dPML, int fs, int NumRec, int nxSou, int nySou,
              const int* nxRec, const int* nyRec, const T* Data_source /*nt_prop2*/,
              const T* Data_target /*(nt_taper, NumRec)*/, T dd, T dt, int ny, int nx,
              int nx_w, const T* Vp_w, float added_space, int store_snap, int nt_snap,
              int nt_prop2, int nt_taper, int taper_option, int N_taper, int N_zeros,
              T* PSDM_w /*(ny, nx_w) out*/, T* Data_synth /*(nt_prop2, NumRec) out or null*/) {
    int nxw2, xi, xf;
    dynamic_window(NumRec, nxSou, nxRec, (float)dd, nx, added_space, &nxw2, &xi, &xf);
    std::vector<int> nxs{nxSou - xi + 1}, nys{nySou}, nxr(NumRec), nyr(NumRec);
    for (int r = 0; r < NumRec; ++r) { nxr[r] = nxRec[r] - xi + 1; nyr[r] = nyRec[r]; }
    std::vector<T> Fields((size_t)ny * nx_w * nt_taper, T(0));
    std::vector<T> synth((size_t)nt_prop2 * NumRec, T(0));
    solver_ac<T>(1, disk_mode, dPML, fs, NumRec, nxs.data(), nys.data(), nxr.data(), nyr.data(),
                 Data_source, dd, dt, ny, nx_w, Vp_w, store_snap, nt_snap, nt_prop2, Fields.data(), synth.data());
    if (Data_synth) std::copy(synth.begin(), synth.end(), Data_synth);
    if (taper_option != 0) {
        std::vector<T> tr(nt_taper);
        const size_t fs2 = (size_t)ny * nx_w;
        for (size_t c = 0; c < fs2; ++c) {
            for (int t = 0; t < nt_taper; ++t) tr[t] = Fields[(size_t)t * fs2 + c];
            taper_pad_trace<T>(tr.data(), nt_prop2, N_taper, N_zeros, nt_taper);
            for (int t = 0; t < nt_taper; ++t) Fields[(size_t)t * fs2 + c] = tr[t];
        }
    }
    std::vector<T> back((size_t)nt_taper * NumRec);
    for (int r = 0; r < NumRec; ++r)
        for (int t = 0; t < nt_taper; ++t)
            back[(size_t)r * nt_taper + t] = Data_target[(size_t)r * nt_taper + (nt_taper - 1 - t)];
    for (size_t q = 0; q < (size_t)ny * nx_w; ++q) PSDM_w[q] = T(0);
    solver_ac<T>(2, disk_mode, dPML, fs, NumRec, nxs.data(), nys.data(), nxr.data(), nyr.data(),
                 back.data(), dd, dt, ny, nx_w, Vp_w, store_snap, nt_taper, nt_taper, Fields.data(), PSDM_w);
}

// Per-shot RTM in the mixed-precision form (see MixedOpts): forward with
// snapshots every store_snap steps (quantized in the float build when
// mo.q16 != 0), taper weights per slot taken at the slot's time sample
// store_snap*m, time-reversed back-source, backward imaging at the paired
// steps.  Slots whose weight is zero contribute nothing.
template <class T>
void rtm_shot_mixed(const MixedOpts& mo, int disk_mode, int dPML, int fs, int NumRec, int nxSou, int nySou,
                    const int* nxRec, const int* nyRec, const T* Data_source, const T* Data_target, T dd, T dt,
                    int ny, int nx, int nx_w, const T* Vp_w, float added_space, int store_snap, int nt_prop2,
                    int nt_taper, int taper_option, int N_taper, int N_zeros, T* PSDM_w, T* Fields_out) {
    int nxw2, xi, xf;
    dynamic_window(NumRec, nxSou, nxRec, (float)dd, nx, added_space, &nxw2, &xi, &xf);
    std::vector<int> nxs{nxSou - xi + 1}, nys{nySou}, nxr(NumRec), nyr(NumRec);
    for (int r = 0; r < NumRec; ++r) { nxr[r] = nxRec[r] - xi + 1; nyr[r] = nyRec[r]; }
    const int nsnap = (nt_prop2 - 1) / store_snap;
    const size_t fs2 = (size_t)ny * nx_w;
    std::vector<T> Fields(fs2 * std::max(nsnap, 1), T(0));
    std::vector<T> synth((size_t)nt_prop2 * NumRec, T(0));
    solver_ac<T>(1, disk_mode, dPML, fs, NumRec, nxs.data(), nys.data(), nxr.data(), nyr.data(), Data_source, dd,
                 dt, ny, nx_w, Vp_w, store_snap, nsnap, nt_prop2, Fields.data(), synth.data(), nullptr, &mo);
    if (Fields_out) std::copy(Fields.begin(), Fields.begin() + fs2 * nsnap, Fields_out);
    std::vector<T> wts(nt_taper, T(1));
    if (taper_option != 0) taper_pad_trace<T>(wts.data(), nt_prop2, N_taper, N_zeros, nt_taper);
    std::vector<T> wslot(std::max(nsnap, 1), T(1));
    for (int m = 1; m <= nsnap; ++m) wslot[m - 1] = wts[(size_t)store_snap * m - 1];
    std::vector<T> back((size_t)nt_taper * NumRec);
    for (int r = 0; r < NumRec; ++r)
        for (int t = 0; t < nt_taper; ++t)
            back[(size_t)r * nt_taper + t] = Data_target[(size_t)r * nt_taper + (nt_taper - 1 - t)];
    for (size_t q = 0; q < fs2; ++q) PSDM_w[q] = T(0);
    solver_ac<T>(2, disk_mode, dPML, fs, NumRec, nxs.data(), nys.data(), nxr.data(), nyr.data(), back.data(), dd,
                 dt, ny, nx_w, Vp_w, store_snap, nsnap, nt_taper, Fields.data(), PSDM_w, nullptr, &mo, wslot.data());
}

template <class T>
std::vector<T> widen(const float* a, size_t n) {
    std::vector<T> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = T(a[i]);
    return v;
}

}  // namespace

extern "C" {

void orc_fd_coef_f(int num, int acc, float* coef) { fd_coef<float>(num, acc, coef); }
void orc_fd_coef_d(int num, int acc, double* coef) { fd_coef<double>(num, acc, coef); }

// Corner outputs are (dn x dn) column-major: ld, rd, lu, ru for A then B.
void orc_pml_coeffs_f(int acc, int dPML, float dt, float d, int dn, float* fA, float* fB, float* corners /*8*dn*dn*/) {
    Arr2<float> m[8];
    for (auto& a : m) a = Arr2<float>(dn, dn);
    pml_coeffs<float>(acc, dPML, dt, d, dn, fA, fB, m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7]);
    for (int q = 0; q < 8; ++q) std::copy(m[q].v.begin(), m[q].v.end(), corners + (size_t)q * dn * dn);
}
void orc_pml_coeffs_d(int acc, int dPML, double dt, double d, int dn, double* fA, double* fB, double* corners) {
    Arr2<double> m[8];
    for (auto& a : m) a = Arr2<double>(dn, dn);
    pml_coeffs<double>(acc, dPML, dt, d, dn, fA, fB, m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7]);
    for (int q = 0; q < 8; ++q) std::copy(m[q].v.begin(), m[q].v.end(), corners + (size_t)q * dn * dn);
}

// src/get_mcs_data.f90:318-351 (Ricker_mcs), FP32.
void orc_ricker_mcs(int nt, float dt, float f0, float t0, float* S0) {
    const float pi = 3.14159265f;
    const float tmp = 10.f / f0;
    for (int i = 1; i <= nt; ++i) {
        const float t = float(i - 1) * dt;
        const float X = (pi * f0) * (t - t0);
        const float X2 = X * X;
        S0[i - 1] = (1.f - 2.f * X2) * expf(-(1.f * X2));
        if (t >= tmp) S0[i - 1] = 0.f;
    }
}

void orc_taper_pad_trace_f(float* tr, int nt_prop, int N_taper, int N_zeros, int nt_new) {
    taper_pad_trace<float>(tr, nt_prop, N_taper, N_zeros, nt_new);
}

void orc_dynamic_window(int NumRec, int nxSou, const int* nxRec, float dd, int nx, float dd_space,
                        int* nx_w, int* x_i, int* x_f) {
    dynamic_window(NumRec, nxSou, nxRec, dd, nx, dd_space, nx_w, x_i, x_f);
}

// Solver level (window coordinates), FP32.
void orc_solver_f(int iprop, int disk_mode, int dPML, int fs, int NumRec,
                  const int* nxSou, const int* nySou, const int* nxRec, const int* nyRec,
                  const float* S, float dmodel, float dt, int ny, int nx, const float* ctmp,
                  int store_snap, int nt_snap, int nt, float* Fields, float* out) {
    solver_ac<float>(iprop, disk_mode, dPML, fs, NumRec, nxSou, nySou, nxRec, nyRec, S, dmodel, dt,
                     ny, nx, ctmp, store_snap, nt_snap, nt, Fields, out);
}

// Solver level, FP32, also returning the padded wavefield p (nyt, nxt) after
// the last step (for locating the first differing cell in a parity failure).
void orc_solver_dump_f(int iprop, int disk_mode, int dPML, int fs, int NumRec,
                       const int* nxSou, const int* nySou, const int* nxRec, const int* nyRec,
                       const float* S, float dmodel, float dt, int ny, int nx, const float* ctmp,
                       int store_snap, int nt_snap, int nt, float* Fields, float* out, float* p_dump) {
    solver_ac<float>(iprop, disk_mode, dPML, fs, NumRec, nxSou, nySou, nxRec, nyRec, S, dmodel, dt,
                     ny, nx, ctmp, store_snap, nt_snap, nt, Fields, out, p_dump);
}

// Solver level, FP64 (inputs widened from float).
void orc_solver_d(int iprop, int disk_mode, int dPML, int fs, int NumRec,
                  const int* nxSou, const int* nySou, const int* nxRec, const int* nyRec,
                  const float* S, int nS, float dmodel, float dt, int ny, int nx, const float* ctmp,
                  int store_snap, int nt_snap, int nt, double* Fields, double* out) {
    auto Sd = widen<double>(S, (size_t)nS);
    auto cd = widen<double>(ctmp, (size_t)ny * nx);
    solver_ac<double>(iprop, disk_mode, dPML, fs, NumRec, nxSou, nySou, nxRec, nyRec, Sd.data(), double(dmodel),
                      double(dt), ny, nx, cd.data(), store_snap, nt_snap, nt, Fields, out);
}

// Per-shot RTM (calculate_PSDM_RTM.f90:395-466), FP32.
void orc_rtm_shot_f(int disk_mode, int dPML, int fs, int NumRec, int nxSou, int nySou,
                    const int* nxRec, const int* nyRec, const float* Data_source, const float* Data_target,
                    float dd, float dt, int ny, int nx, int nx_w, const float* Vp_w, float added_space,
                    int store_snap, int nt_snap, int nt_prop2, int nt_taper, int taper_option,
                    int N_taper, int N_zeros, float* PSDM_w, float* Data_synth) {
    rtm_shot<float>(disk_mode, dPML, fs, NumRec, nxSou, nySou, nxRec, nyRec, Data_source, Data_target, dd, dt,
                    ny, nx, nx_w, Vp_w, added_space, store_snap, nt_snap, nt_prop2, nt_taper, taper_option,
                    N_taper, N_zeros, PSDM_w, Data_synth);
}

// Per-shot RTM, FP64 (float inputs widened).
void orc_rtm_shot_d(int disk_mode, int dPML, int fs, int NumRec, int nxSou, int nySou,
                    const int* nxRec, const int* nyRec, const float* Data_source, const float* Data_target,
                    float dd, float dt, int ny, int nx, int nx_w, const float* Vp_w, float added_space,
                    int store_snap, int nt_snap, int nt_prop2, int nt_taper, int taper_option,
                    int N_taper, int N_zeros, double* PSDM_w, double* Data_synth) {
    auto src = widen<double>(Data_source, (size_t)nt_prop2);
    auto tgt = widen<double>(Data_target, (size_t)nt_taper * NumRec);
    auto vp = widen<double>(Vp_w, (size_t)ny * nx_w);
    rtm_shot<double>(disk_mode, dPML, fs, NumRec, nxSou, nySou, nxRec, nyRec, src.data(), tgt.data(), double(dd),
                     double(dt), ny, nx, nx_w, vp.data(), added_space, store_snap, nt_snap, nt_prop2, nt_taper,
                     taper_option, N_taper, N_zeros, PSDM_w, Data_synth);
}

// Mixed-precision form, float build: emulates the engine's FP16/BF16 form
// bit for bit (q16 = 1 / 2, Kahan image).  Fields_out (ny, nx_w, nsnap) gets
// the snapshots as the backward pass reads them, or null.
void orc_rtm_shot_mixed_f(int q16, int kahan, int disk_mode, int dPML, int fs, int NumRec, int nxSou, int nySou,
                          const int* nxRec, const int* nyRec, const float* Data_source, const float* Data_target,
                          float dd, float dt, int ny, int nx, int nx_w, const float* Vp_w, float added_space,
                          int store_snap, int nt_prop2, int nt_taper, int taper_option, int N_taper, int N_zeros,
                          float* PSDM_w, float* Fields_out) {
    MixedOpts mo;
    mo.pair_mode = 1;
    mo.q16 = q16;
    mo.kahan = kahan;
    mo.coef64 = q16 != 0;  // the engine's 16-bit forms; q16 = 0 keeps the reference's set-up
    rtm_shot_mixed<float>(mo, disk_mode, dPML, fs, NumRec, nxSou, nySou, nxRec, nyRec, Data_source, Data_target, dd,
                          dt, ny, nx, nx_w, Vp_w, added_space, store_snap, nt_prop2, nt_taper, taper_option, N_taper,
                          N_zeros, PSDM_w, Fields_out);
}

// Mixed-precision form, FP64 oracle: the same schedule in double precision
// throughout (no rounding of the snapshots, plain summation).
void orc_rtm_shot_mixed_d(int disk_mode, int dPML, int fs, int NumRec, int nxSou, int nySou, const int* nxRec,
                          const int* nyRec, const float* Data_source, const float* Data_target, float dd, float dt,
                          int ny, int nx, int nx_w, const float* Vp_w, float added_space, int store_snap,
                          int nt_prop2, int nt_taper, int taper_option, int N_taper, int N_zeros, double* PSDM_w,
                          double* Fields_out) {
    MixedOpts mo;
    mo.pair_mode = 1;
    auto src = widen<double>(Data_source, (size_t)nt_prop2);
    auto tgt = widen<double>(Data_target, (size_t)nt_taper * NumRec);
    auto vp = widen<double>(Vp_w, (size_t)ny * nx_w);
    rtm_shot_mixed<double>(mo, disk_mode, dPML, fs, NumRec, nxSou, nySou, nxRec, nyRec, src.data(), tgt.data(),
                           double(dd), double(dt), ny, nx, nx_w, vp.data(), added_space, store_snap, nt_prop2,
                           nt_taper, taper_option, N_taper, N_zeros, PSDM_w, Fields_out);
}

// src/auxiliar_PSDM.f90:1-20.
void orc_normalize_psdm(int nx, int ny, const float* PSDM_sum, const float* Cov_sum, float* PSDM) {
    for (size_t q = 0; q < (size_t)nx * ny; ++q) PSDM[q] = (Cov_sum[q] > 0.f) ? PSDM_sum[q] / Cov_sum[q] : 0.f;
}

}  // extern "C"

// ---- trace conditioning (src/calculate_PSDM_RTM.f90:231-355) ----------------
//
// The per-shot preparation of the observed data before the backward pass:
// travel-time windows from the bathymetry, resampling to the propagation
// time step, the sea-floor cut, the multiple cut and the taper.  The
// frequency filter (freq_filter, auxiliar.f90:498-531) is not restated.

namespace {

// Time-window lengths (calculate_PSDM_RTM.f90:231-291), FP32 as the
// reference: nt_cut / nt_sf per trace, then nt_prop2, nt_taper, N_taper,
// N_zeros.  Batmodel is indexed with the 1-based model column mid_x.
void trace_windows(int cut_multiple, int cut_sf, int taper_option, float T_taper, float T_zeros, int NumRec,
                   int nxSou, int nySou, const int* nxRec, const int* nyRec, const float* Batmodel,
                   float dmodel_prop, float dt_prop, int nt_prop, int* nt_cut, int* nt_sf, int* nt_prop2,
                   int* nt_taper, int* N_taper, int* N_zeros) {
    for (int j = 0; j < NumRec; ++j) {
        nt_cut[j] = nt_prop;  // :123
        nt_sf[j] = 1;         // :124
    }
    for (int pass = 0; pass < 2; ++pass) {
        if ((pass == 0 && cut_multiple <= 0) || (pass == 1 && cut_sf <= 0)) continue;
        for (int j = 0; j < NumRec; ++j) {
            const float offset = std::fabs(float(nxSou) * dmodel_prop - float(nxRec[j]) * dmodel_prop);
            const int mid_x = (int)std::ceil(0.5f * float(nxSou + nxRec[j]));
            const float D_src = Batmodel[mid_x - 1] - float(nySou) * dmodel_prop;
            const float D_rec = Batmodel[mid_x - 1] - float(nyRec[j]) * dmodel_prop;
            const float a = offset * 0.5f, b = 0.5f * (D_src + D_rec);
            const float leg = std::sqrt(a * a + b * b);
            if (pass == 0) {
                const float twt = (4.0f * leg) / 1500.f;
                nt_cut[j] = (int)std::ceil((0.9f * twt) / dt_prop);
            } else {
                const float twt = (2.0f * leg) / 1500.f;
                nt_sf[j] = (int)std::ceil((1.1f * twt) / dt_prop);
            }
        }
    }
    *nt_prop2 = nt_prop;
    *nt_taper = nt_prop;
    *N_taper = 1;
    *N_zeros = 0;
    if (taper_option != 0 || cut_multiple != 0) {
        *N_taper = std::max(1, (int)(T_taper / dt_prop));
        *N_zeros = std::max(0, (int)(T_zeros / dt_prop));
        int mx = nt_cut[0];
        for (int j = 1; j < NumRec; ++j) mx = std::max(mx, nt_cut[j]);
        *nt_prop2 = std::min(nt_prop, mx);
        *nt_taper = *nt_prop2 + *N_zeros;
    }
}

// Akima's (1970) local cubic interpolation of y sampled at x_k = k*dx
// (k = 0..n-1), evaluated at t; the end slopes are extended with
// m[-1] = 2m[0] - m[1], m[-2] = 2m[-1] - m[0] (and mirrored at the far end),
// and points outside the data use the end interval's cubic.  Written from
// the published method; the engine's kernel evaluates the same expressions
// in the same order.
struct AkimaTrace {
    const float* y;
    int n;
    float dx;
    float x(int k) const { return float(k) * dx; }
    float m(int k) const {  // slope of interval k, extended beyond both ends
        if (k < 0) {
            const float m0 = m(0), m1 = m(1);
            const float mm1 = 2.f * m0 - m1;
            return k == -1 ? mm1 : 2.f * mm1 - m0;
        }
        if (k > n - 2) {
            const float a = m(n - 2), b = m(n - 3);
            const float mp = 2.f * a - b;
            return k == n - 1 ? mp : 2.f * mp - a;
        }
        return (y[k + 1] - y[k]) / (x(k + 1) - x(k));
    }
    float slope_at(int k) const {  // derivative at point k
        const float w1 = std::fabs(m(k + 1) - m(k)), w2 = std::fabs(m(k - 1) - m(k - 2));
        if (w1 + w2 == 0.f) return 0.5f * (m(k - 1) + m(k));
        return (w1 * m(k - 1) + w2 * m(k)) / (w1 + w2);
    }
    float at(float t) const {
        if (n == 1) return y[0];
        if (n == 2) return y[0] + (t - x(0)) * ((y[1] - y[0]) / (x(1) - x(0)));
        if (t == x(n - 1)) return y[n - 1];
        int j = (int)(t / dx);
        j = std::min(std::max(j, 0), n - 2);
        while (j > 0 && t < x(j)) --j;
        while (j < n - 2 && t >= x(j + 1)) ++j;
        const float h = x(j + 1) - x(j), d = t - x(j);
        const float tj = slope_at(j), tj1 = slope_at(j + 1), mj = m(j);
        const float p2 = (3.f * mj - 2.f * tj - tj1) / h;
        const float p3 = (tj + tj1 - 2.f * mj) / (h * h);
        return y[j] + d * (tj + d * (p2 + d * p3));
    }
};

}  // namespace

extern "C" {

void orc_trace_windows(int cut_multiple, int cut_sf, int taper_option, float T_taper, float T_zeros, int NumRec,
                       int nxSou, int nySou, const int* nxRec, const int* nyRec, const float* Batmodel,
                       float dmodel_prop, float dt_prop, int nt_prop, int* nt_cut, int* nt_sf, int* out4) {
    trace_windows(cut_multiple, cut_sf, taper_option, T_taper, T_zeros, NumRec, nxSou, nySou, nxRec, nyRec, Batmodel,
                  dmodel_prop, dt_prop, nt_prop, nt_cut, nt_sf, out4, out4 + 1, out4 + 2, out4 + 3);
}

void orc_akima(const float* y, int n, float dx, int m, float dt, float* out) {
    AkimaTrace a{y, n, dx};
    for (int i = 0; i < m; ++i) out[i] = a.at(float(i) * dt);
}

// Data_target (nt_taper, NumRec) from Field_Data (nt_data, NumRec),
// calculate_PSDM_RTM.f90:316-355 without the frequency filter.
void orc_condition_traces(int cut_multiple, int cut_sf, int taper_option, int NumRec, const float* Field_Data,
                          int nt_data, float dt_data, float dt_prop, int nt_prop2, int nt_taper, int N_taper,
                          int N_zeros, const int* nt_cut, const int* nt_sf, float* Data_target) {
    for (int i = 0; i < NumRec; ++i) {
        float* tr = Data_target + (size_t)i * nt_taper;
        const float* f = Field_Data + (size_t)i * nt_data;
        for (int s = 0; s < nt_taper; ++s) tr[s] = 0.f;
        if (dt_data != dt_prop) {
            AkimaTrace a{f, nt_data, dt_data};
            for (int s = 0; s < nt_prop2; ++s) tr[s] = a.at(float(s) * dt_prop);
        } else {
            for (int s = 0; s < nt_prop2 && s < nt_data; ++s) tr[s] = f[s];
        }
        if (cut_sf > 0)
            for (int s = 0; s < nt_sf[i] && s < nt_taper; ++s) tr[s] = 0.f;
        if (cut_multiple == 0) {
            if (taper_option != 0) taper_pad_trace<float>(tr, nt_prop2, N_taper, N_zeros, nt_taper);
        } else {
            // guard: the reference indexes outside the trace if nt_cut > nt_taper or < 1
            const int c = std::max(1, std::min(nt_cut[i], nt_taper));
            for (int s = c - 1; s < nt_taper; ++s) tr[s] = 0.f;
            taper_pad_trace<float>(tr, c, N_taper, N_zeros, nt_taper);
        }
    }
}

}  // extern "C"
