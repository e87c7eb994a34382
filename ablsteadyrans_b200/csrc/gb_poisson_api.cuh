// Host-side state of the Poisson layer (the C ABI's gb_poisson handle).
#pragma once

#include "gb_poisson.cuh"

#include <vector>

namespace gb {

constexpr int kMaxLevels = 16;

//! The multigrid hierarchy in one arithmetic type.
template <typename T>
struct PoissonLevels {
    gb_grid g[kMaxLevels];
    PBC b[kMaxLevels];
    T* z[kMaxLevels] = {};
    T* J[kMaxLevels] = {};
    T* AX[kMaxLevels] = {};
    T* AY[kMaxLevels] = {};
    T* AZ[kMaxLevels] = {};
    T* x[kMaxLevels] = {};
    T* bv[kMaxLevels] = {};
    T* r[kMaxLevels] = {};
    T* snap[kMaxLevels] = {};
    T* TD[kMaxLevels] = {};   // the smoother's line tridiagonal, per level
    T* TC[kMaxLevels] = {};
    T* TU[kMaxLevels] = {};
    T* RX[kMaxLevels] = {};  // the mesh ratios of the operator (MeshRatios), per level
    T* RY[kMaxLevels] = {};
    T* HZ[kMaxLevels] = {};
    T* SX[kMaxLevels] = {};
    T* SY[kMaxLevels] = {};
    MeshRatios<T> ratios(int l) const { return MeshRatios<T>{RX[l], RY[l], HZ[l], SX[l], SY[l], z[l]}; }
    std::vector<void*> owned;
    void release();
};

}  // namespace gb

struct gb_poisson {
    gb_ctx* ctx{nullptr};
    gb_grid g{};
    int bc[6]{};
    gb_poisson_opts opt{};
    const double* z_fine{nullptr};  // the caller's node heights (kept by reference)
    const double* J_fine{nullptr};
    int nlev{0};
    gb::PoissonLevels<double> dl;  // FP64 hierarchy (geometry and coefficients of every level)
    gb::PoissonLevels<float> fl;   // FP32 copies (precision == 1)
    bool coeffs_set{false};
    // FaceCoeffs::z_cross: d = beta_z - z_cross and a_z d per z-face (owned;
    // null: no split). The Krylov operator and the fluxes carry it, the
    // V-cycle (the preconditioner) does not.
    double* cross_d{nullptr};
    double* cross_ad{nullptr};
    double* cross_store[2]{nullptr, nullptr};
    // Krylov workspace
    int64_t vstride{0};
    double* V{nullptr};
    double* Zv{nullptr};
    unsigned long long* d_err{nullptr};    // set when a TMA tile wait gave up
    double* w{nullptr};
    double* t{nullptr};
    int dot_blocks{0};
    double* d_partial{nullptr};
    double* d_dots{nullptr};
    double* d_coef{nullptr};
    double* h_dots{nullptr};
    // one Arnoldi step's dots on the device and their one read-back:
    // [0, m+2) the first Gram-Schmidt pass, [m+2, 2m+4) the second, [2m+4] |w|^2
    double* d_step{nullptr};
    double* h_step{nullptr};
    double J_sum{0};
    // The V-cycle as a CUDA graph per precision (0 FP64, 1 FP32): captured on
    // the solver's own stream on its second call (the first runs eagerly) and
    // launched on the context's stream; rebuilt when the tuning knobs change.
    cudaStream_t capture_stream{nullptr};
    cudaGraphExec_t vc_exec[2]{nullptr, nullptr};
    int64_t vc_launches[2]{0, 0};
    int vc_calls[2]{0, 0};
    uint64_t vc_tune_key[2]{0, 0};
    std::vector<void*> owned;
    ~gb_poisson();
};

namespace gb {

//! The range checks of solver.poisson_* (messages name the keys).
gb_status check_poisson_options(const gb_poisson_opts& o);
gb_status poisson_build(gb_poisson* P);
gb_status poisson_set_coeffs(gb_poisson* P, const double* ax, const double* ay, const double* az, const double* bx,
                             const double* by, const double* bz);
gb_status poisson_set_z_cross(gb_poisson* P, const double* az, const double* bz, const double* z_cross);
gb_status poisson_apply(gb_poisson* P, const double* phi, double* y);
gb_status poisson_vcycle(gb_poisson* P, const double* r, double* e);
gb_status poisson_fluxes(gb_poisson* P, const double* phi, const double* bx, const double* by, const double* bz,
                         double* fx, double* fy, double* fz);
gb_status poisson_solve(gb_poisson* P, double* rhs, double* phi, gb_poisson_result* res);
gb_status weighted_mean(gb_poisson* P, const double* f, double* host_mean, int slot);
gb_status mesh_metrics(gb_ctx* ctx, const gb_grid& g, const double* z, double* J, double* ax, double* ay, double* az,
                       double* zcc);
gb_status face_divergence(gb_ctx* ctx, const gb_grid& g, const double* ax, const double* ay, const double* az,
                          const double* J, const double* fx, const double* fy, const double* fz, double* div);
void multiply_inplace(gb_ctx* ctx, double* a, const double* b, int64_t n);

}  // namespace gb
