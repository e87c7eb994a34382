// Compile-check stand-ins for the AMReX and GUST declarations the C++ shim
// (ablsteadyrans_b200/shim/gust_b200_shim.cpp) uses: just enough of each
// type's interface for the shim's calls to type-check in a host-only unit
// with no AMReX. In a GUST build the real headers of the same names are used.
#pragma once

#include <array>
#include <cstddef>
#include <string>

namespace amrex {
using Real = double;
using Long = long long;
template <class T, std::size_t N>
using Array = std::array<T, N>;

struct IntVect {
    int v[3]{0, 0, 0};
    int operator[](int d) const { return v[d]; }
};

struct Box {
    IntVect lo, hi;
    int length(int d) const { return hi[d] - lo[d] + 1; }
};

struct Geometry {
    Box dom;
    Real dx[3]{1, 1, 1};
    bool per[3]{false, false, false};
    const Box& Domain() const { return dom; }
    Real CellSize(int d) const { return dx[d]; }
    bool isPeriodic(int d) const { return per[d]; }
};

struct FArrayBox {
    Real* p{nullptr};
    Real* dataPtr(int comp = 0) { return p + comp; }
    const Real* dataPtr(int comp = 0) const { return p + comp; }
};

struct MultiFab {
    FArrayBox fab;
    int ncomp{1};
    FArrayBox& operator[](int) { return fab; }
    const FArrayBox& operator[](int) const { return fab; }
    int nComp() const { return ncomp; }
    bool empty() const { return fab.p == nullptr; }
};

[[noreturn]] void Abort(const std::string& msg);

namespace Gpu {
void* gpuStream();
}
}  // namespace amrex

namespace gust {
using amrex::Real;
enum class Loc : int { cell = 0, xface = 1, yface = 2, zface = 4 };
enum class Equation { u, v, w, theta, tke };
enum class FaceMean { arithmetic, logarithmic };

struct Mesh {
    amrex::MultiFab detJ;
    Real dz{1};
    Real dzeta() const { return dz; }
};

struct State {
    amrex::MultiFab u, v, w, p, theta, tke;
};

struct ResidualFields {
    amrex::MultiFab u, v, w, p, theta, tke;
};

struct PredictorFields {
    amrex::MultiFab ap_u, ap_v, ap_w;
    amrex::MultiFab d_u, d_v, d_w;
};

struct MomentumPredictorResult {
    Real max_du{0}, max_dv{0}, max_dw{0};
    Real last_sweep_du{0}, last_sweep_dv{0}, last_sweep_dw{0};
};

struct PoissonResult {
    int iterations{0};
    Real initial_residual{0}, final_residual{0};
    bool singular{false};
    Real removed_mean{0};
};

struct PressureCorrectionResult {
    PoissonResult poisson;
    Real divergence_before{0}, divergence_after{0}, max_dp{0};
    Real max_du{0}, max_dv{0}, max_dw{0};
};

struct ScalarSweepResult {
    Real max_dq{0};
    Real last_sweep{0};
    amrex::Long clipped{0};
};
}  // namespace gust
