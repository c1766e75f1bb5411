// Internal declarations shared by the host code and the CUDA translation
// units of the RTM engine.  Not part of the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>

namespace psdm {

constexpr int kAcc = 3;  // FD half-width (acc=3, src/solver_ac_forward_ram.f90:95)

void pml_profiles_f32(int acc, int dPML, float dt, float d, int dn, float* fA, float* fB);
void pml_profiles_f64(int acc, int dPML, double dt, double d, int dn, double* fA, double* fB);
float taper_weight(int n, int N_taper);

// Padded propagation grid of one shot (0-based, column-major, z fastest):
//   z in [0, nyt), x in [0, nxt), element (z, x) at x*ldz + z.
// Interior rows [dn, dn+ny), interior columns [dn, dn+nx); dn = dPML+2*acc
// (src/solver_ac_forward_ram.f90:103-127).
struct Grid {
    int ny = 0, nx = 0, dPML = 0, dn = 0, nyt = 0, nxt = 0, ldz = 0;
    size_t cells() const { return (size_t)ldz * (size_t)nxt; }
};

// Arguments of one fused time step.  Pointers are device pointers.
struct StepArgs {
    // wavefield: p = level n (read only); pm = level n-1 in, level n+1 out
    const float* p;
    float* pm;
    const float* c2;
    // C-PML memory variables on the padded grid (only PML cells touched)
    const float* phix_in;
    float* phix_out;
    float* chix;
    const float* phiz_in;
    float* phiz_out;
    float* chiz;
    // strip-private histories of the free-surface row in the x-strip columns
    // (RAM ordering with a free surface): side_p = level n, side_pm = n-1 -> n+1
    const float* side_p;
    float* side_pm;
    // C-PML profiles factorA/B[dn] (index k-1, k = 1 next to the interior)
    const float* fA;
    const float* fB;
    // FD coefficients (finite_difference_coef, acc = 3)
    float cf1[4];
    float cf2[4];
    // grid
    int nyt, nxt, ldz, ny, nx, dn;
    int fs;     // free surface on
    int disk;   // disk solvers' statement order
    // injection (sources / adjoint sources): row_slot[z] = -1 or a row slot;
    // inj_cols[slot*nxt + x] = trace index or -1; value inj_trace[j*inj_ld + inj_t]
    const int* row_slot;
    const int* inj_cols;
    const float* inj_trace;
    int inj_ld, inj_t;
    // forward snapshot (write) or backward snapshot (read); null = none this step
    float* field;
    float dt;
    // backward imaging: image[(x-dn)*ny + (z-dn)] += 0.5*(p3-p1)*field*w*ss
    float* image;
    float field_w;   // taper weight of this snapshot slot
    float ss;        // float(store_snap)
    // deferred receiver gather (forward): rec_out[i*rec_ld + rec_t] = p[rec_cell[i]]
    const int* rec_cell;
    float* rec_out;
    int nrec, rec_ld, rec_t;  // rec_t < 0: no gather this step
};

// Launch one fused forward (mode 0) or backward (mode 1) step on `stream`.
int launch_step(int mode, const StepArgs& a, void* stream);
// Receiver gather after the last forward step (Rec(nt-1) and Rec(nt)).
int launch_rec_final(const int* rec_cell, const float* p, float* rec_out, int nrec, int rec_ld, int nt, void* stream);
// Padded c2 = c^2 dt^2 / d^2 from the window model (edge replication;
// ram_padding = 1 reproduces the RAM solvers' partial top/bottom padding).
int launch_pad_c2(const float* vp, int ny, int nx, int dn, int nyt, int nxt, int ldz, float dt, float dd,
                  int ram_padding, float* c2, void* stream);

}  // namespace psdm
