// The pressure-correction Poisson layer on the GPU: mesh metrics, the
// terrain operator (FP64 and FP32), fluxes, divergence, the multigrid
// hierarchy (z-line zebra relaxation, x-y 2:1 coarsening, coarsest-level
// relaxation) and the FP64 flexible GMRES it preconditions.
//
// Reference: gust::PoissonSolver (Source/Poisson.H:135-161, Source/Poisson.cpp:
// 421-623), ERF's TerrainPoisson (extern_erf/ERF_TerrainPoisson.cpp:74-264),
// the metrics (extern_erf/ERF_TerrainMetrics.cpp:680-808). The multigrid is
// this project's own (the reference's default, AMReX MLTerrainPoisson, is not
// in the reference's tree); it is restated by the oracle operation for
// operation, so one V-cycle agrees with the oracle's to rounding.
#include "gb_poisson.cuh"
#include "gb_poisson_api.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <vector>

namespace gb {

namespace {

constexpr int kBlock = 256;

inline int nblocks(int64_t n, int b = kBlock) { return static_cast<int>((n + b - 1) / b); }

// ------------------------------------------------------------- metrics ---

__global__ void k_metrics(gb_grid g, const double* __restrict__ z, double* __restrict__ J, double* __restrict__ ax,
                          double* __restrict__ ay, double* __restrict__ zcc)
{
    // one thread per (i, j, k) in i, j in [-1, n+1], k in [-1, nz]
    const int ni = g.nx + 3, nj = g.ny + 3, nk = g.nz + 2;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= static_cast<int64_t>(ni) * nj * nk) { return; }
    const int i = static_cast<int>(n % ni) - 1;
    const int j = static_cast<int>((n / ni) % nj) - 1;
    const int k = static_cast<int>(n / (static_cast<int64_t>(ni) * nj)) - 1;
    const double dzi = 1.0 / g.dzeta;
#define Z(a, b, c) z[at(g, a, b, c)]
    if (k >= 0 && i <= g.nx && j <= g.ny) {
        J[at(g, i, j, k)] = 0.25 * dzi
            * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i, j, k)
               - Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i + 1, j + 1, k));
    }
    if (k >= 0 && j <= g.ny) {
        ax[at(g, i, j, k)] = 0.5 * dzi * (Z(i, j, k + 1) + Z(i, j + 1, k + 1) - Z(i, j, k) - Z(i, j + 1, k));
    }
    if (k >= 0 && i <= g.nx) {
        ay[at(g, i, j, k)] = 0.5 * dzi * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) - Z(i, j, k) - Z(i + 1, j, k));
    }
    if (i <= g.nx && j <= g.ny) {
        zcc[at(g, i, j, k)] = 0.125 * (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k) + Z(i, j, k + 1)
                                       + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1));
    }
#undef Z
}

__global__ void k_fill(double* __restrict__ a, int64_t n, double v)
{
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t < n) { a[t] = v; }
}

// ------------------------------------------------------- valid-cell maps ---

__device__ __forceinline__ bool cell_of(const gb_grid& g, int64_t n, int& i, int& j, int& k)
{
    if (n >= static_cast<int64_t>(g.nx) * g.ny * g.nz) { return false; }
    i = static_cast<int>(n % g.nx);
    j = static_cast<int>((n / g.nx) % g.ny);
    k = static_cast<int>(n / (static_cast<int64_t>(g.nx) * g.ny));
    return true;
}

// ------------------------------------------------------- operator apply ---

//! y = A x, or with rhs given y = rhs - A x (the residual).
//! At most 72 registers a thread (no spills): 7 blocks of 128 an SM where
//! the 80 the compiler picks fit 6; the operator is bound by its loads'
//! latency, and the added warps took the fine-level apply from 46 to 38 us.
template <typename T>
__global__ void __maxnreg__(72) k_apply(gb_grid g, PBC b, const T* __restrict__ x, const T* __restrict__ AX, const T* __restrict__ AY,
                        const T* __restrict__ AZ, const T* __restrict__ J, MeshRatios<T> m,
                        const T* __restrict__ rhs, T* __restrict__ y)
{
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) { return; }
    const T v = adotx_cell<T>(g, b, i, j, k, x, AX, AY, AZ, J, m);
    const int64_t o = at(g, i, j, k);
    y[o] = rhs ? rhs[o] - v : v;
}

//! The mesh ratios of one level (MeshRatios) in FP64 from the node heights,
//! stored as T, on every valid point of each array's location.
template <typename T>
__global__ void k_mesh_ratios(gb_grid g, const double* __restrict__ zp, T* __restrict__ rx, T* __restrict__ ry,
                              T* __restrict__ hz, T* __restrict__ sx, T* __restrict__ sy)
{
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int ni = g.nx + 1, nj = g.ny + 1, nk = g.nz + 1;
    if (n >= static_cast<int64_t>(ni) * nj * nk) { return; }
    const int i = static_cast<int>(n % ni);
    const int j = static_cast<int>((n / ni) % nj);
    const int k = static_cast<int>(n / (static_cast<int64_t>(ni) * nj));
    const double dxinv = 1.0 / g.dx, dyinv = 1.0 / g.dy, q = 0.25, h = 0.5;
    const int64_t o = at(g, i, j, k);
#define Z(a, bb, c) zp[at(g, a, bb, c)]
    if (j < g.ny) {  // x-z edge at x-node i, z-node k
        const double h_xi = q * (Z(i + 1, j, k) - Z(i - 1, j, k) + Z(i + 1, j + 1, k) - Z(i - 1, j + 1, k)) * dxinv;
        const double h_zeta = q * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1));
        rx[o] = static_cast<T>(h_xi / h_zeta);
    }
    if (i < g.nx) {  // y-z edge at y-node j, z-node k
        const double h_eta = q * (Z(i, j + 1, k) - Z(i, j - 1, k) + Z(i + 1, j + 1, k) - Z(i + 1, j - 1, k)) * dyinv;
        const double h_zeta = q * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1));
        ry[o] = static_cast<T>(h_eta / h_zeta);
    }
    if (i < g.nx && j < g.ny) {  // z-face k
        hz[o] = static_cast<T>(8.0 / ((Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1))
                                      - (Z(i, j, k - 1) + Z(i + 1, j, k - 1) + Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k - 1))));
        sx[o] = static_cast<T>(h * (Z(i + 1, j + 1, k) + Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i, j, k)) * dxinv);
        sy[o] = static_cast<T>(h * (Z(i + 1, j + 1, k) + Z(i, j + 1, k) - Z(i + 1, j, k) - Z(i, j, k)) * dyinv);
    }
#undef Z
}

// ---------------------------------------------------------------- fluxes ---

//! The face fluxes -grad phi of the terrain operator at x-face (i, j, k),
//! y-face and z-face (ERF_TerrainPoisson_3D_K.H:22-275), with the mesh
//! ratios precomputed (MeshRatios) in place of their inline divisions.
template <typename T>
__device__ __forceinline__ T flux_x_r(const gb_grid& g, const PBC& b, int i, int j, int k, const T* x,
                                      const MeshRatios<T>& m)
{
    const T dxinv = static_cast<T>(1.0 / g.dx), h = T(0.5);
    const int64_t o = at(g, i, j, k);
#define X(a, bb, c) ldc<T>(x, x, g, b, a, bb, c)
    T px_lo = (X(i, j, k) - X(i - 1, j, k)) * dxinv;
    T pz_lo_md_hi = h * (X(i, j, k + 1) + X(i - 1, j, k + 1) - X(i, j, k) - X(i - 1, j, k));
    pz_lo_md_hi *= m.rx[o + g.sz];
    T pz_lo_md_lo = h * (X(i, j, k) + X(i - 1, j, k) - X(i, j, k - 1) - X(i - 1, j, k - 1));
    pz_lo_md_lo *= m.rx[o];
    px_lo -= h * (pz_lo_md_hi + pz_lo_md_lo);
    return -px_lo;
#undef X
}

template <typename T>
__device__ __forceinline__ T flux_y_r(const gb_grid& g, const PBC& b, int i, int j, int k, const T* x,
                                      const MeshRatios<T>& m)
{
    const T dyinv = static_cast<T>(1.0 / g.dy), h = T(0.5);
    const int64_t o = at(g, i, j, k);
#define X(a, bb, c) ldc<T>(x, x, g, b, a, bb, c)
    T py_lo = (X(i, j, k) - X(i, j - 1, k)) * dyinv;
    T pz_md_lo_hi = h * (X(i, j, k + 1) + X(i, j - 1, k + 1) - X(i, j, k) - X(i, j - 1, k));
    pz_md_lo_hi *= m.ry[o + g.sz];
    T pz_md_lo_lo = h * (X(i, j, k) + X(i, j - 1, k) - X(i, j, k - 1) - X(i, j - 1, k - 1));
    pz_md_lo_lo *= m.ry[o];
    py_lo -= h * (pz_md_lo_hi + pz_md_lo_lo);
    return -py_lo;
#undef X
}

template <typename T>
__device__ __forceinline__ T flux_z_r(const gb_grid& g, const PBC& b, int i, int j, int k, const T* x,
                                      const MeshRatios<T>& m)
{
    const T dxinv = static_cast<T>(1.0 / g.dx), dyinv = static_cast<T>(1.0 / g.dy), h = T(0.5);
    const int64_t o = at(g, i, j, k);
#define X(a, bb, c) ldc<T>(x, x, g, b, a, bb, c)
    T pz_lo = X(i, j, k) - X(i, j, k - 1);
    pz_lo *= m.hz[o];
    const T px_hi_md_lo = h * (X(i + 1, j, k) - X(i, j, k) + X(i + 1, j, k - 1) - X(i, j, k - 1)) * dxinv;
    const T px_lo_md_lo = h * (X(i, j, k) - X(i - 1, j, k) + X(i, j, k - 1) - X(i - 1, j, k - 1)) * dxinv;
    const T py_md_hi_lo = h * (X(i, j + 1, k) - X(i, j, k) + X(i, j + 1, k - 1) - X(i, j, k - 1)) * dyinv;
    const T py_md_lo_lo = h * (X(i, j, k) - X(i, j - 1, k) + X(i, j, k - 1) - X(i, j - 1, k - 1)) * dyinv;
    T pz_hi_md_lo = h * (X(i + 1, j, k) + X(i, j, k) - X(i + 1, j, k - 1) - X(i, j, k - 1));
    pz_hi_md_lo *= m.rx[o + 1];
    T pz_lo_md_lo = h * (X(i, j, k) + X(i - 1, j, k) - X(i, j, k - 1) - X(i - 1, j, k - 1));
    pz_lo_md_lo *= m.rx[o];
    T pz_md_hi_lo = h * (X(i, j + 1, k) + X(i, j, k) - X(i, j + 1, k - 1) - X(i, j, k - 1));
    pz_md_hi_lo *= m.ry[o + g.sy];
    T pz_md_lo_lo = h * (X(i, j, k) + X(i, j - 1, k) - X(i, j, k - 1) - X(i, j - 1, k - 1));
    pz_md_lo_lo *= m.ry[o];
    pz_lo -= h * m.sx[o] * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo));
    pz_lo -= h * m.sy[o] * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));
    if (k == 0) { pz_lo = T(0); }
    return -pz_lo;
#undef X
}

//! The face fluxes -grad phi with the zero-flux faces masked, times beta
//! (null: 1). One thread per node column (i, j) slot and level k.
__global__ void k_fluxes(gb_grid g, PBC b, const double* __restrict__ phi, MeshRatios<double> m,
                         const double* __restrict__ bx, const double* __restrict__ by, const double* __restrict__ bz,
                         double* __restrict__ fx, double* __restrict__ fy, double* __restrict__ fz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i > g.nx || j > g.ny) { return; }
    if (j < g.ny && k < g.nz) {
        double f = flux_x_r<double>(g, b, i, j, k, phi, m);
        if (((b.zf & TP_XLO) && i == 0) || ((b.zf & TP_XHI) && i == g.nx)) { f = 0; }
        const int64_t o = at(g, i, j, k);
        fx[o] = bx ? f * bx[o] : f;
    }
    if (i < g.nx && k < g.nz) {
        double f = flux_y_r<double>(g, b, i, j, k, phi, m);
        if (((b.zf & TP_YLO) && j == 0) || ((b.zf & TP_YHI) && j == g.ny)) { f = 0; }
        const int64_t o = at(g, i, j, k);
        fy[o] = by ? f * by[o] : f;
    }
    if (i < g.nx && j < g.ny) {
        double f = flux_z_r<double>(g, b, i, j, k, phi, m);
        if ((b.zf & TP_ZHI) && k == g.nz) { f = 0; }
        const int64_t o = at(g, i, j, k);
        fz[o] = bz ? f * bz[o] : f;
    }
}

//! z_face_cross (Source/PoissonCross_K.H:16-58): the terrain cross part
//! h_x dphi/dx + h_y dphi/dy of the gradient at the low z-face of cell (i, j, k),
//! the edge ratios and face slopes taken from MeshRatios.
__device__ __forceinline__ double z_face_cross_r(const gb_grid& g, const PBC& b, int i, int j, int k,
                                                 const double* x, const MeshRatios<double>& m)
{
    const double dxinv = 1.0 / g.dx, dyinv = 1.0 / g.dy, h = 0.5;
    const int64_t o = at(g, i, j, k);
#define X(a, bb, c) ldc<double>(x, x, g, b, a, bb, c)
    const double px_hi_md_lo = h * (X(i + 1, j, k) - X(i, j, k) + X(i + 1, j, k - 1) - X(i, j, k - 1)) * dxinv;
    const double px_lo_md_lo = h * (X(i, j, k) - X(i - 1, j, k) + X(i, j, k - 1) - X(i - 1, j, k - 1)) * dxinv;
    const double py_md_hi_lo = h * (X(i, j + 1, k) - X(i, j, k) + X(i, j + 1, k - 1) - X(i, j, k - 1)) * dyinv;
    const double py_md_lo_lo = h * (X(i, j, k) - X(i, j - 1, k) + X(i, j, k - 1) - X(i, j - 1, k - 1)) * dyinv;
    const double pz_hi_md_lo = h * (X(i + 1, j, k) + X(i, j, k) - X(i + 1, j, k - 1) - X(i, j, k - 1)) * m.rx[o + 1];
    const double pz_lo_md_lo = h * (X(i, j, k) + X(i - 1, j, k) - X(i, j, k - 1) - X(i - 1, j, k - 1)) * m.rx[o];
    const double pz_md_hi_lo = h * (X(i, j + 1, k) + X(i, j, k) - X(i, j + 1, k - 1) - X(i, j, k - 1)) * m.ry[o + g.sy];
    const double pz_md_lo_lo = h * (X(i, j, k) + X(i, j - 1, k) - X(i, j, k - 1) - X(i, j - 1, k - 1)) * m.ry[o];
#undef X
    return h * m.sx[o] * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo))
         + h * m.sy[o] * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));
}

//! The z-faces the split correction touches: not the ground, not a Neumann
//! top (Source/Poisson.cpp:233-235, 246-249).
__device__ __forceinline__ bool cross_face(const gb_grid& g, const PBC& b, int kf)
{
    return kf != 0 && !((b.zf & TP_ZHI) && kf == g.nz);
}

//! PoissonSolver::Op::add_cross (Source/Poisson.cpp:229-253): y += sign (1/J)
//! d_zeta (a_z d cross), a_z d given per z-face. One thread per cell.
__global__ void k_add_cross(gb_grid g, PBC b, const double* __restrict__ x, const double* __restrict__ ad,
                            const double* __restrict__ J, MeshRatios<double> m, double sign, double* __restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) { return; }
    const int64_t o = at(g, i, j, k);
    const double hi = cross_face(g, b, k + 1) ? ad[o + g.sz] * z_face_cross_r(g, b, i, j, k + 1, x, m) : 0.0;
    const double lo = cross_face(g, b, k) ? ad[o] * z_face_cross_r(g, b, i, j, k, x, m) : 0.0;
    y[o] += sign * ((hi - lo) * (1.0 / g.dzeta) / J[o]);
}

//! PoissonSolver::Op::add_cross_flux (Source/Poisson.cpp:255-273):
//! F_z -= d cross on the same faces. One thread per z-face.
__global__ void k_cross_flux(gb_grid g, PBC b, const double* __restrict__ x, const double* __restrict__ d,
                             MeshRatios<double> m, double* __restrict__ fz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || !cross_face(g, b, k)) { return; }
    const int64_t o = at(g, i, j, k);
    fz[o] -= d[o] * z_face_cross_r(g, b, i, j, k, x, m);
}

__global__ void k_face_divergence(gb_grid g, const double* __restrict__ ax, const double* __restrict__ ay,
                                  const double* __restrict__ az, const double* __restrict__ J,
                                  const double* __restrict__ fx, const double* __restrict__ fy,
                                  const double* __restrict__ fz, double* __restrict__ div)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) { return; }
    const double dxinv = 1.0 / g.dx, dyinv = 1.0 / g.dy, dzinv = 1.0 / g.dzeta;
    const int64_t o = at(g, i, j, k);
    const int64_t ox = at(g, i + 1, j, k), oy = at(g, i, j + 1, k), oz = at(g, i, j, k + 1);
    div[o] = ((ax[ox] * fx[ox] - ax[o] * fx[o]) * dxinv + (ay[oy] * fy[oy] - ay[o] * fy[o]) * dyinv
              + (az[oz] * fz[oz] - az[o] * fz[o]) * dzinv)
           / J[o];
}

// ------------------------------------------------------------- multigrid ---

//! Coarse node heights by injection (the fine column under each coarse node
//! column; ghost columns the periodic image or the clamped edge).
__global__ void k_coarse_z(gb_grid gc, double* __restrict__ zc, gb_grid gf, const double* __restrict__ zf)
{
    const int ni = gc.nx + 3, nj = gc.ny + 3, nk = gc.nz + 3;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= static_cast<int64_t>(ni) * nj * nk) { return; }
    int I = static_cast<int>(n % ni) - 1;
    int J2 = static_cast<int>((n / ni) % nj) - 1;
    const int k = static_cast<int>(n / (static_cast<int64_t>(ni) * nj)) - 1;
    int si = I, sj = J2;
    if (si < 0 || si > gc.nx) { si = gc.periodic_x ? ((si < 0) ? si + gc.nx : si - gc.nx) : ((si < 0) ? 0 : gc.nx); }
    if (sj < 0 || sj > gc.ny) { sj = gc.periodic_y ? ((sj < 0) ? sj + gc.ny : sj - gc.ny) : ((sj < 0) ? 0 : gc.ny); }
    zc[at(gc, I, J2, k)] = zf[at(gf, 2 * si, 2 * sj, k)];
}

//! Coarse premultiplied areas: the means of the fine faces a coarse face covers.
__global__ void k_coarse_areas(gb_grid gc, double* __restrict__ AXc, double* __restrict__ AYc,
                               double* __restrict__ AZc, gb_grid gf, const double* __restrict__ AXf,
                               const double* __restrict__ AYf, const double* __restrict__ AZf)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J2 = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (I > gc.nx || J2 > gc.ny) { return; }
    if (J2 < gc.ny && k < gc.nz) {
        AXc[at(gc, I, J2, k)] = 0.5 * (AXf[at(gf, 2 * I, 2 * J2, k)] + AXf[at(gf, 2 * I, 2 * J2 + 1, k)]);
    }
    if (I < gc.nx && k < gc.nz) {
        AYc[at(gc, I, J2, k)] = 0.5 * (AYf[at(gf, 2 * I, 2 * J2, k)] + AYf[at(gf, 2 * I + 1, 2 * J2, k)]);
    }
    if (I < gc.nx && J2 < gc.ny) {
        AZc[at(gc, I, J2, k)] = 0.25 * (AZf[at(gf, 2 * I, 2 * J2, k)] + AZf[at(gf, 2 * I + 1, 2 * J2, k)]
                                        + AZf[at(gf, 2 * I, 2 * J2 + 1, k)] + AZf[at(gf, 2 * I + 1, 2 * J2 + 1, k)]);
    }
}

//! The principal tridiagonal (D, C, U) of every cell of a level, computed
//! once per set of coefficients (the smoother's line operator T).
template <typename T>
__global__ void k_line_tridiag(gb_grid g, PBC b, const T* __restrict__ AX, const T* __restrict__ AY,
                               const T* __restrict__ AZ, const T* __restrict__ J, const T* __restrict__ z,
                               T* __restrict__ TD, T* __restrict__ TC, T* __restrict__ TU)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) { return; }
    T D, C, U;
    line_tridiag<T>(g, b, AX, AY, AZ, J, z, i, j, k, D, C, U);
    const int64_t o = at(g, i, j, k);
    TD[o] = D;
    TC[o] = C;
    TU[o] = U;
}

//! Zebra relaxation, first half of a colour: r = b - A x on every cell of the
//! columns with (i + j) & 1 == color (one thread per cell; every read happens
//! before the colour's updates, so the periodic wrap reads see the old values).
//! Capped at 72 registers as k_apply.
template <typename T>
__global__ void __maxnreg__(72) k_color_residual(gb_grid g, PBC b, int color, const T* __restrict__ x, const T* __restrict__ bv,
                                 const T* __restrict__ AX, const T* __restrict__ AY, const T* __restrict__ AZ,
                                 const T* __restrict__ J, MeshRatios<T> m, T* __restrict__ r)
{
    pdl_entry();
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((j + color) & 1);
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) { return; }
    const int64_t o = at(g, i, j, k);
    r[o] = bv[o] - adotx_cell<T>(g, b, i, j, k, x, AX, AY, AZ, J, m);
}

// ------------------------------------------------ TMA-staged operator tiles ---
//
// The operator on a level as blocks of kTileI x kTileJ columns (COLOR: the
// block's columns of one zebra colour, over 2 kTileI consecutive i) that
// march up kTileK levels. The iterate's planes reach shared memory by bulk
// copies (cp.async.bulk, the TMA unit): one copy per staged row, the rows
// j0 - 1 .. j0 + kTileJ of columns i0 - 1 .. i0 + span, into a ring of
// kTileRing plane slots, each slot's copies completing on its own mbarrier;
// the plane two levels up streams in while a level is evaluated. A row's
// copy starts at the 16-byte boundary at or below column i0 - 1 (a level's
// row stride is an odd number of elements, so rows start on either
// boundary) and the tile records the shift. Entries outside the valid cells
// (the ghost rows, columns and planes a boundary block stages) are then
// overwritten with their ghost-resolved values (ldc: periodic images and
// mirrors with the face's sign), so every cell reads its 15 values from the
// tile by one code path; the mesh ratios, areas and J, each read once or
// twice a cell, stay direct loads.

constexpr int kTileI = 32, kTileJ = 8, kTileK = 8, kTileRing = 4;
constexpr int kTileWaitLimit = 1 << 22;

template <typename T, bool COLOR>
struct TileShape {
    static constexpr int E = 16 / static_cast<int>(sizeof(T));    // elements per 16 bytes
    static constexpr int SPAN = COLOR ? 2 * kTileI : kTileI;         // the block's i-span of cells
    static constexpr int PITCH = ((SPAN + 2 + E - 1 + E - 1) / E) * E;  // staged row: shift + SPAN + 2, rounded
    static constexpr int ROWS = kTileJ + 2;
};

//! y = rhs - A x (or A x with rhs null) on every cell (COLOR false) or on
//! the cells of one colour (COLOR true), from TMA-staged tiles of x. err: a
//! device word set when a wait for a tile gave up (the block then finishes
//! with whatever the tile holds, and the caller reports the failure).
template <typename T, bool COLOR>
__global__ void __launch_bounds__(kTileI* kTileJ)
    k_stencil_tile(gb_grid g, PBC b, int color, const T* __restrict__ x, const T* __restrict__ AX,
                   const T* __restrict__ AY, const T* __restrict__ AZ, const T* __restrict__ J, MeshRatios<T> m,
                   const T* __restrict__ rhs, T* __restrict__ y, unsigned long long* err)
{
    using S = TileShape<T, COLOR>;
    __shared__ __align__(16) T tile[kTileRing][S::ROWS][S::PITCH];
    __shared__ __align__(8) uint64_t bar[kTileRing];
    __shared__ int shift[kTileRing][S::ROWS];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTileI + tx;
    const int i0 = blockIdx.x * S::SPAN, j0 = blockIdx.y * kTileJ;
    const int kb = blockIdx.z * kTileK, ke = min(kb + kTileK, g.nz);
    const int ilast = min(i0 + S::SPAN, g.nx);  // staged columns i0 - 1 .. ilast
    const int jlast = min(j0 + kTileJ, g.ny);   // staged rows j0 - 1 .. jlast
    const bool edge_block = (i0 == 0) || (ilast == g.nx) || (j0 == 0) || (jlast == g.ny);
    const int j = j0 + ty;
    const int i = COLOR ? i0 + 2 * tx + ((j + color) & 1) : i0 + tx;
    const bool active = (i < g.nx) && (j < g.ny);
    if (tid == 0) {
        for (int q = 0; q < kTileRing; ++q) { mbar_init(&bar[q], 1); }
        fence_barrier_init();
    }
    __syncthreads();
    auto slot_of = [&](int kk) { return (kk + 1) & (kTileRing - 1); };
    auto parity_of = [&](int kk) { return static_cast<unsigned>(((kk - (kb - 1)) / kTileRing) & 1); };
    // one thread issues a plane's row copies (kk in -1 .. nz)
    auto issue = [&](int kk) {
        const int q = slot_of(kk);
        unsigned total = 0;
        int64_t ea[S::ROWS];
        unsigned nb[S::ROWS];
        for (int r = 0; r < S::ROWS; ++r) {
            const int jj = j0 - 1 + r;
            nb[r] = 0;
            ea[r] = 0;
            if (jj > jlast) { continue; }
            const int64_t e0 = at(g, i0 - 1, jj, kk);
            const int64_t e1 = at(g, ilast, jj, kk);
            ea[r] = e0 & ~static_cast<int64_t>(S::E - 1);
            const int64_t n = ((e1 - ea[r] + 1 + S::E - 1) / S::E) * S::E;
            nb[r] = static_cast<unsigned>(n * sizeof(T));
            shift[q][r] = static_cast<int>(e0 - ea[r]);
            total += nb[r];
        }
        mbar_arrive_expect_tx(&bar[q], total);
        for (int r = 0; r < S::ROWS; ++r) {
            if (nb[r] != 0) { bulk_copy_g2s(&tile[q][r][0], x + ea[r], nb[r], &bar[q]); }
        }
    };
    // after the copies landed: the entries outside the valid cells take their ghost-resolved values
    auto fixup = [&](int kk) {
        if (!edge_block && kk >= 0 && kk < g.nz) { return; }
        const int q = slot_of(kk);
        const int ncol = ilast - (i0 - 1) + 1;
        const int nrow = jlast - (j0 - 1) + 1;
        for (int e = tid; e < nrow * ncol; e += kTileI * kTileJ) {
            const int r = e / ncol, c = e % ncol;
            const int ii = i0 - 1 + c, jj = j0 - 1 + r;
            if (ii < 0 || ii >= g.nx || jj < 0 || jj >= g.ny || kk < 0 || kk >= g.nz) {
                tile[q][r][shift[q][r] + c] = ldc<T>(x, x, g, b, ii, jj, kk);
            }
        }
    };
    bool ok = true;
    if (tid == 0) {
        issue(kb - 1);
        issue(kb);
        if (kb + 1 <= ke) { issue(kb + 1); }
    }
    for (int kk = kb - 1; kk <= kb; ++kk) {
        ok = mbar_wait_bounded(&bar[slot_of(kk)], parity_of(kk), kTileWaitLimit) && ok;
        fixup(kk);
    }
    for (int k = kb; k < ke; ++k) {
        if (tid == 0 && k + 2 <= ke) {
            fence_proxy_async_shared();
            issue(k + 2);
        }
        ok = mbar_wait_bounded(&bar[slot_of(k + 1)], parity_of(k + 1), kTileWaitLimit) && ok;
        fixup(k + 1);
        __syncthreads();
        if (active) {
            const int qm = slot_of(k - 1), q0 = slot_of(k), qp = slot_of(k + 1);
            const int c = i - i0 + 1;
            const int r = j - j0 + 1;
            auto X = [&](int di, int dj, int dk) {
                const int q = (dk < 0) ? qm : (dk > 0) ? qp : q0;
                return tile[q][r + dj][shift[q][r + dj] + c + di];
            };
            const int64_t o = at(g, i, j, k);
            const T v = adotx_body<T, true>(g, b, i, j, k, o, X, AX, AY, AZ, J, m);
            y[o] = rhs ? rhs[o] - v : v;
        }
        // this thread's reads (and fix-up writes) of the slots before the next bulk copy into one
        fence_proxy_async_shared();
        __syncthreads();
    }
    if (!ok && tid == 0) { atomicOr(err, 1ull); }
}

//! The LU factors of every column's line tridiagonal T, once per coefficient
//! set (T does not change between relaxations): in place of C and U the
//! reciprocal pivots 1/m_k and the eliminated uppers c'_k = U_k / m_k, with
//! m_0 = C_0, m_k = C_k - D_k c'_{k-1} (D, the lower diagonal, is kept). One
//! thread per column; the loads of 8 levels are batched ahead of the chain.
template <typename T>
__device__ __forceinline__ void line_factor_column(const gb_grid& g, T* __restrict__ TD, T* __restrict__ TC,
                                                   T* __restrict__ TU, int i, int j);

template <typename T>
__global__ void k_line_factor(gb_grid g, T* __restrict__ TD, T* __restrict__ TC, T* __restrict__ TU)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) { return; }
    line_factor_column<T>(g, TD, TC, TU, i, j);
}

//! The factorisation of column (i, j): the reciprocal pivots and eliminated
//! uppers in place of C and U (the loads of 8 levels batched ahead of the chain).
template <typename T>
__device__ __forceinline__ void line_factor_column(const gb_grid& g, T* __restrict__ TD, T* __restrict__ TC,
                                                   T* __restrict__ TU, int i, int j)
{
    const int64_t o0 = at(g, i, j, 0);
    T cp = T(0);
    for (int k0 = 0; k0 < g.nz; k0 += 8) {
        T D[8], C[8], U[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (k0 + q < g.nz) {
                const int64_t o = o0 + static_cast<int64_t>(k0 + q) * g.sz;
                D[q] = TD[o];
                C[q] = TC[o];
                U[q] = TU[o];
            }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int k = k0 + q;
            if (k < g.nz) {
                const T m = (k == 0) ? C[q] : C[q] - D[q] * cp;
                const T im = T(1) / m;
                cp = U[q] * im;
                const int64_t o = o0 + static_cast<int64_t>(k) * g.sz;
                TC[o] = im;
                TU[o] = cp;
            }
        }
    }
}

//! Every level's line tridiagonal (k_line_tridiag) in one launch and every
//! level's column factorisation (k_line_factor) in another: the levels are
//! independent, and one launch over all of them replaces two per level (the
//! coarse levels' launches were latency for a few hundred cells).
template <typename T>
struct LineLevels {
    gb_grid g[kMaxLevels];
    PBC b[kMaxLevels];
    const T* AX[kMaxLevels];
    const T* AY[kMaxLevels];
    const T* AZ[kMaxLevels];
    const T* J[kMaxLevels];
    const T* z[kMaxLevels];
    T* TD[kMaxLevels];
    T* TC[kMaxLevels];
    T* TU[kMaxLevels];
    int64_t cells[kMaxLevels + 1];  // prefix sums of the levels' cells
    int64_t cols[kMaxLevels + 1];   // prefix sums of the levels' columns
    int n;
};

template <typename T>
__global__ void k_line_tridiag_all(const __grid_constant__ LineLevels<T> L)
{
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= L.cells[L.n]) { return; }
    int l = 0;
    while (n >= L.cells[l + 1]) { ++l; }
    const gb_grid& g = L.g[l];
    const int64_t m = n - L.cells[l];
    const int i = static_cast<int>(m % g.nx), j = static_cast<int>((m / g.nx) % g.ny);
    const int k = static_cast<int>(m / (static_cast<int64_t>(g.nx) * g.ny));
    T D, C, U;
    line_tridiag<T>(g, L.b[l], L.AX[l], L.AY[l], L.AZ[l], L.J[l], L.z[l], i, j, k, D, C, U);
    const int64_t o = at(g, i, j, k);
    L.TD[l][o] = D;
    L.TC[l][o] = C;
    L.TU[l][o] = U;
}

template <typename T>
__global__ void k_line_factor_all(const __grid_constant__ LineLevels<T> L)
{
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= L.cols[L.n]) { return; }
    int l = 0;
    while (n >= L.cols[l + 1]) { ++l; }
    const gb_grid& g = L.g[l];
    const int64_t m = n - L.cols[l];
    line_factor_column<T>(g, L.TD[l], L.TC[l], L.TU[l], static_cast<int>(m % g.nx), static_cast<int>(m / g.nx));
}

//! Zebra relaxation, second half: on every column of the colour x += T^{-1} r
//! with the factors of k_line_factor (e_k = (r_k - D_k e_{k-1}) / m_k, then
//! x_k = e_k - c'_k x_{k+1}), the column's r, D, 1/m, c' staged R levels ahead
//! into shared memory with asynchronous copies (c', e' kept in shared memory).
//! Used when a whole column does not fit the staged kernel below.
template <typename T, int R>
__global__ void __launch_bounds__(64) k_color_solve(gb_grid g, int color, const T* __restrict__ r,
                                                    const T* __restrict__ TD, const T* __restrict__ TC,
                                                    const T* __restrict__ TU, T* __restrict__ x)
{
    pdl_entry();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    const int j = blockIdx.y;
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((j + color) & 1);
    const bool active = i < g.nx;
    T* ring = reinterpret_cast<T*>(smem_raw);
    T* cs = ring + R * 4 * nthr;
    T* es = cs + static_cast<int64_t>(g.nz) * nthr;
    const int64_t o0 = active ? at(g, i, j, 0) : 0;
    auto issue = [&](int k) {
        if (active && k < g.nz) {
            const int64_t o = o0 + static_cast<int64_t>(k) * g.sz;
            T* s = ring + (k % R) * 4 * nthr + tid;
            cp_async_elem(s, r + o);
            cp_async_elem(s + nthr, TD + o);
            cp_async_elem(s + 2 * nthr, TC + o);
            cp_async_elem(s + 3 * nthr, TU + o);
        }
        cp_async_commit();
    };
#pragma unroll
    for (int k = 0; k < R - 1; ++k) { issue(k); }
    T ep = T(0);
    for (int k = 0; k < g.nz; ++k) {
        issue(k + R - 1);
        cp_async_wait<R - 1>();
        if (active) {
            const T* s = ring + (k % R) * 4 * nthr + tid;
            const T rk = s[0], D = s[nthr], im = s[2 * nthr];
            ep = ((k == 0) ? rk : rk - D * ep) * im;
            cs[k * nthr + tid] = s[3 * nthr];
            es[k * nthr + tid] = ep;
        }
    }
    cp_async_wait<0>();
    if (!active) { return; }
    T xk = ep;
    int64_t o = o0 + static_cast<int64_t>(g.nz - 1) * g.sz;
    x[o] += xk;
    for (int k = g.nz - 2; k >= 0; --k) {
        o -= g.sz;
        xk = es[k * nthr + tid] - cs[k * nthr + tid] * xk;
        x[o] += xk;
    }
}

//! The same relaxation with the whole column staged at once: every level's r,
//! D, 1/m, c' and x goes into shared memory ([array][k][thread]) in one burst
//! of asynchronous copies, so the column's memory latency is paid once and the
//! two recurrences then run from shared memory without a division; e
//! overwrites r in place and x is written back once per level.
template <typename T>
__global__ void __launch_bounds__(32) k_color_solve_staged(gb_grid g, int color, const T* __restrict__ r,
                                                           const T* __restrict__ TD, const T* __restrict__ TC,
                                                           const T* __restrict__ TU, T* __restrict__ x)
{
    pdl_entry();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    const int j = blockIdx.y;
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((j + color) & 1);
    if (i >= g.nx) { return; }  // no block barrier below: each thread owns its column
    const int nz = g.nz;
    const int64_t plane = static_cast<int64_t>(nz) * nthr;
    T* sr = reinterpret_cast<T*>(smem_raw) + tid;
    T* sd = sr + plane;
    T* sm = sd + plane;
    T* sc = sm + plane;
    T* sx = sc + plane;
    const int64_t o0 = at(g, i, j, 0);
    for (int k = 0; k < nz; ++k) {
        const int64_t o = o0 + static_cast<int64_t>(k) * g.sz;
        const int s = k * nthr;
        cp_async_elem(sr + s, r + o);
        cp_async_elem(sd + s, TD + o);
        cp_async_elem(sm + s, TC + o);
        cp_async_elem(sc + s, TU + o);
        cp_async_elem(sx + s, x + o);
    }
    cp_async_commit();
    cp_async_wait<0>();
    T ep = sr[0] * sm[0];
    sr[0] = ep;
    for (int k = 1; k < nz; ++k) {
        const int s = k * nthr;
        ep = (sr[s] - sd[s] * ep) * sm[s];
        sr[s] = ep;
    }
    T xk = ep;
    int64_t o = o0 + static_cast<int64_t>(nz - 1) * g.sz;
    x[o] = sx[(nz - 1) * nthr] + xk;
    for (int k = nz - 2; k >= 0; --k) {
        const int s = k * nthr;
        o -= g.sz;
        xk = sr[s] - sc[s] * xk;
        x[o] = sx[s] + xk;
    }
}

//! One colour's relaxation in ONE launch: a block owns up to kFusedCols
//! columns of the colour along one row; its threads compute the residual
//! r = b - A x of every cell of those columns into shared memory (with the
//! columns' x and line factors), a block barrier, then one thread per column
//! runs the factored Thomas solve of k_color_solve_staged and writes x. The
//! arithmetic and its order are those of k_color_residual followed by
//! k_color_solve_staged; r never goes to global memory and the colour costs
//! one launch. The lateral neighbours of a column are of the other colour,
//! and only this block updates its own columns, so every read sees the
//! values from before the colour's update (a periodic direction of odd
//! extent pairs a column with a same-colour image: the caller then uses the
//! two-launch form). Shared memory: [array][k][column] for r, D, 1/m, c', x.
constexpr int kFusedCols = 32;

template <typename T>
__global__ void __launch_bounds__(256) k_color_relax_fused(gb_grid g, PBC b, int color, T* x, const T* __restrict__ bv,
                                                           const T* __restrict__ AX, const T* __restrict__ AY,
                                                           const T* __restrict__ AZ, const T* __restrict__ J,
                                                           MeshRatios<T> m, const T* __restrict__ TD,
                                                           const T* __restrict__ TC, const T* __restrict__ TU)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int C = kFusedCols;
    const int nz = g.nz;
    const int plane = nz * C;
    T* sr = reinterpret_cast<T*>(smem_raw);
    T* sd = sr + plane;
    T* sm = sd + plane;
    T* sc = sm + plane;
    T* sx = sc + plane;
    const int j = blockIdx.y;
    const int c0 = blockIdx.x * C;
    for (int n = threadIdx.x; n < plane; n += blockDim.x) {
        const int col = n % C, k = n / C;
        const int i = 2 * (c0 + col) + ((j + color) & 1);
        if (i >= g.nx) { continue; }
        const int64_t o = at(g, i, j, k);
        sx[n] = x[o];
        sd[n] = TD[o];
        sm[n] = TC[o];
        sc[n] = TU[o];
        sr[n] = bv[o] - adotx_cell<T>(g, b, i, j, k, x, AX, AY, AZ, J, m);
    }
    __syncthreads();
    const int col = threadIdx.x;
    if (col >= C) { return; }
    const int i = 2 * (c0 + col) + ((j + color) & 1);
    if (i >= g.nx) { return; }
    T ep = sr[col] * sm[col];
    sr[col] = ep;
    for (int k = 1; k < nz; ++k) {
        const int s = k * C + col;
        ep = (sr[s] - sd[s] * ep) * sm[s];
        sr[s] = ep;
    }
    T xk = ep;
    int64_t o = at(g, i, j, nz - 1);
    x[o] = sx[(nz - 1) * C + col] + xk;
    for (int k = nz - 2; k >= 0; --k) {
        const int s = k * C + col;
        o -= g.sz;
        xk = sr[s] - sc[s] * xk;
        x[o] = sx[s] + xk;
    }
}

//! Zebra relaxation, second half, with the column's levels split among the
//! warps of a block: x += T^{-1} r on every column of the colour with the
//! factors of k_line_factor (e_k = (r_k - D_k e_{k-1}) / m_k, then x_k = e_k
//! - c'_k x_{k+1}). A block holds 32 columns of the colour along one row and
//! ceil(nz / L) warps; each thread loads its L levels' r, D, 1/m, c' and x at
//! once (in-range clamped indices: no load behind a branch), runs the
//! recurrences over them in their sequential order and carries e' upwards and
//! the correction downwards through shared memory as each segment's affine
//! map (the segmented z-line sweep's carries). A coarse level's few columns
//! then keep many warps busy, where one thread per column walks every level.
template <typename T, int L>
__global__ void __launch_bounds__(512) k_color_solve_seg(gb_grid g, int color, const T* __restrict__ r,
                                                         const T* __restrict__ TD, const T* __restrict__ TC,
                                                         const T* __restrict__ TU, T* __restrict__ x)
{
    pdl_entry();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x;
    const int w = threadIdx.y;
    const int W = blockDim.y;
    const int j = blockIdx.y;
    const int half = (g.nx + 1) / 2;
    const int c = blockIdx.x * 32 + lane;
    const bool col = c < half && 2 * c + ((j + color) & 1) < g.nx;
    const int i = col ? 2 * c + ((j + color) & 1) : ((j + color) & 1);   // an in-range column for every lane
    const int nz = g.nz;
    const int k0 = w * L;
    const int cs = W * 32;
    const int me = w * 32 + lane;
    T* carry_e = reinterpret_cast<T*>(smem_raw);  // [2][W][32]
    T* carry_x = carry_e + 2 * cs;                // [2][W][32]
    const int64_t o0 = at(g, min(i, g.nx - 1), j, 0);
    T R[L], D[L], IM[L], CP[L], X0[L];
#pragma unroll
    for (int q = 0; q < L; ++q) {
        const int64_t o = o0 + static_cast<int64_t>(min(k0 + q, nz - 1)) * g.sz;
        R[q] = r[o];
        D[q] = TD[o];
        IM[q] = TC[o];
        CP[q] = TU[o];
        X0[q] = x[o];
    }
    {
        T al = T(0), be = T(1);
#pragma unroll
        for (int q = 0; q < L; ++q) {
            const int k = k0 + q;
            if (k < nz) {
                if (k == 0) {
                    al = R[q] * IM[q];
                    be = T(0);
                } else {
                    al = (R[q] - D[q] * al) * IM[q];
                    be = (-D[q] * be) * IM[q];
                }
            }
        }
        carry_e[me] = al;
        carry_e[cs + me] = be;
    }
    __syncthreads();
    {
        T ep = T(0);
        for (int s = 0; s < w; ++s) { ep = carry_e[s * 32 + lane] + carry_e[cs + s * 32 + lane] * ep; }
#pragma unroll
        for (int q = 0; q < L; ++q) {
            const int k = k0 + q;
            if (k < nz) {
                ep = (k == 0) ? R[q] * IM[q] : (R[q] - D[q] * ep) * IM[q];
                R[q] = ep;
            }
        }
    }
    {
        T ga = T(0), de = T(1);
#pragma unroll
        for (int q = L - 1; q >= 0; --q) {
            const int k = k0 + q;
            if (k < nz) {
                if (k == nz - 1) {
                    ga = R[q];
                    de = T(0);
                } else {
                    ga = R[q] - CP[q] * ga;
                    de = -CP[q] * de;
                }
            }
        }
        carry_x[me] = ga;
        carry_x[cs + me] = de;
    }
    __syncthreads();
    T xk = T(0);
    for (int s = W - 1; s > w; --s) { xk = carry_x[s * 32 + lane] + carry_x[cs + s * 32 + lane] * xk; }
#pragma unroll
    for (int q = L - 1; q >= 0; --q) {
        const int k = k0 + q;
        if (k < nz) {
            xk = (k == nz - 1) ? R[q] : R[q] - CP[q] * xk;
            if (col) { x[o0 + static_cast<int64_t>(k) * g.sz] = X0[q] + xk; }
        }
    }
}

//! One colour's relaxation in ONE launch with every level of a column in
//! flight: a block holds 32 columns of the colour along one row and
//! ceil(nz / L) warps; warp w owns levels [w L, w L + L) of every column. Each
//! thread evaluates r = b - A x at its levels (adotx_cell, as
//! k_color_residual) and loads the columns' line factors (D, 1/m, c') and x;
//! then the factored Thomas solve of k_color_solve_staged runs over the
//! segment with its sequential recurrences, and what crosses a segment
//! boundary (e' upwards, the correction downwards) goes through shared memory
//! as each segment's affine map, applied by the segments above (below) it. The
//! results agree with the two-launch form to rounding (the values carried
//! across a boundary are evaluated through the composed maps). All reads of x
//! precede the block's first barrier and all writes follow its last; the
//! lateral neighbours of a column are of the other colour and only this block
//! writes its columns, so every read sees the values from before the
//! colour's update (a periodic direction of odd extent pairs a column with a
//! same-colour image: the caller then uses the two-launch form).
template <typename T, int L>
__global__ void __launch_bounds__(512) k_color_relax_seg(gb_grid g, PBC b, int color, T* x, const T* __restrict__ bv,
                                                         const T* __restrict__ AX, const T* __restrict__ AY,
                                                         const T* __restrict__ AZ, const T* __restrict__ J,
                                                         MeshRatios<T> m, const T* __restrict__ TD,
                                                         const T* __restrict__ TC, const T* __restrict__ TU)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x;
    const int w = threadIdx.y;
    const int W = blockDim.y;
    const int j = blockIdx.y;
    const int i = 2 * (blockIdx.x * 32 + lane) + ((j + color) & 1);
    const bool col = i < g.nx;
    const int nz = g.nz;
    const int k0 = w * L;
    const int cs = W * 32;
    const int me = w * 32 + lane;
    T* carry_e = reinterpret_cast<T*>(smem_raw);  // [2][W][32]
    T* carry_x = carry_e + 2 * cs;                // [2][W][32]
    T r[L], D[L], im[L], cp[L], x0[L];
#pragma unroll
    for (int q = 0; q < L; ++q) {
        const int k = k0 + q;
        r[q] = T(0);
        D[q] = T(0);
        im[q] = T(0);
        cp[q] = T(0);
        x0[q] = T(0);
        if (col && k < nz) {
            const int64_t o = at(g, i, j, k);
            r[q] = bv[o] - adotx_cell<T>(g, b, i, j, k, x, AX, AY, AZ, J, m);
            D[q] = TD[o];
            im[q] = TC[o];
            cp[q] = TU[o];
            x0[q] = x[o];
        }
    }
    // forward: e_k = (r_k - D_k e_{k-1}) / m_k, the segment's affine map of e'
    {
        T al = T(0), be = T(1);
#pragma unroll
        for (int q = 0; q < L; ++q) {
            const int k = k0 + q;
            if (k < nz) {
                if (k == 0) {
                    al = r[q] * im[q];
                    be = T(0);
                } else {
                    al = (r[q] - D[q] * al) * im[q];
                    be = (-D[q] * be) * im[q];
                }
            }
        }
        carry_e[me] = al;
        carry_e[cs + me] = be;
    }
    __syncthreads();
    {
        T ep = T(0);
        for (int s = 0; s < w; ++s) {
            const int n = s * 32 + lane;
            ep = carry_e[n] + carry_e[cs + n] * ep;
        }
#pragma unroll
        for (int q = 0; q < L; ++q) {
            const int k = k0 + q;
            if (k < nz) {
                ep = (k == 0) ? r[q] * im[q] : (r[q] - D[q] * ep) * im[q];
                r[q] = ep;
            }
        }
    }
    // back: x_k = e_k - c'_k x_{k+1} (x_{nz-1} = e_{nz-1}), the segment's affine map
    {
        T ga = T(0), de = T(1);
#pragma unroll
        for (int q = L - 1; q >= 0; --q) {
            const int k = k0 + q;
            if (k < nz) {
                if (k == nz - 1) {
                    ga = r[q];
                    de = T(0);
                } else {
                    ga = r[q] - cp[q] * ga;
                    de = -cp[q] * de;
                }
            }
        }
        carry_x[me] = ga;
        carry_x[cs + me] = de;
    }
    __syncthreads();
    T xk = T(0);
    for (int s = W - 1; s > w; --s) {
        const int n = s * 32 + lane;
        xk = carry_x[n] + carry_x[cs + n] * xk;
    }
#pragma unroll
    for (int q = L - 1; q >= 0; --q) {
        const int k = k0 + q;
        if (k < nz) {
            xk = (k == nz - 1) ? r[q] : r[q] - cp[q] * xk;
            if (col) { x[at(g, i, j, k)] = x0[q] + xk; }
        }
    }
}

//! Coarse right-hand side at coarse cell (I, J2, k): the J-weighted sum of
//! the four fine residuals over 4 J_c (a coarse cell's flux balance is the sum
//! of its fine cells').
template <typename T>
__device__ __forceinline__ void restrict_cell(const gb_grid& gf, const T* Jf, const T* rf, const gb_grid& gc,
                                              const T* Jc, T* bc, int I, int J2, int k)
{
    const int i = 2 * I, j = 2 * J2;
    const T s = (Jf[at(gf, i, j, k)] * rf[at(gf, i, j, k)] + Jf[at(gf, i + 1, j, k)] * rf[at(gf, i + 1, j, k)])
              + (Jf[at(gf, i, j + 1, k)] * rf[at(gf, i, j + 1, k)] + Jf[at(gf, i + 1, j + 1, k)] * rf[at(gf, i + 1, j + 1, k)]);
    bc[at(gc, I, J2, k)] = s / (T(4) * Jc[at(gc, I, J2, k)]);
}

//! Fine correction at fine cell (i, j, k): bilinear in x-y from the coarse
//! cell centres (weights 9, 3, 3, 1 over 16), coarse ghosts from the BC.
template <typename T>
__device__ __forceinline__ void prolong_cell(const gb_grid& gc, const PBC& bcb, const T* xc, const gb_grid& gf,
                                             T* xf, int i, int j, int k)
{
    const int I = i >> 1, J2 = j >> 1;
    const int si = (i & 1) ? 1 : -1, sj = (j & 1) ? 1 : -1;
    const T v = (T(9) * ldc<T>(xc, xc, gc, bcb, I, J2, k) + T(3) * ldc<T>(xc, xc, gc, bcb, I + si, J2, k))
              + (T(3) * ldc<T>(xc, xc, gc, bcb, I, J2 + sj, k) + T(1) * ldc<T>(xc, xc, gc, bcb, I + si, J2 + sj, k));
    xf[at(gf, i, j, k)] += v * T(0.0625);
}

template <typename T>
__global__ void k_restrict(gb_grid gf, const T* __restrict__ Jf, const T* __restrict__ rf, gb_grid gc,
                           const T* __restrict__ Jc, T* __restrict__ bc, T* __restrict__ xc)
{
    pdl_entry();
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J2 = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (I >= gc.nx || J2 >= gc.ny) { return; }
    restrict_cell<T>(gf, Jf, rf, gc, Jc, bc, I, J2, k);
    // the coarse correction starts from zero (its ghosts are never read: every
    // kernel resolves a level's ghosts by index)
    if (xc != nullptr) { xc[at(gc, I, J2, k)] = T(0); }
}

template <typename T>
__global__ void k_prolong_add(gb_grid gc, PBC bcb, const T* __restrict__ xc, gb_grid gf, T* __restrict__ xf)
{
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= gf.nx || j >= gf.ny) { return; }
    prolong_cell<T>(gc, bcb, xc, gf, xf, i, j, k);
}

//! All relaxations of the coarsest level in ONE block. On a level of a few
//! columns every launch is latency, and the coarsest level takes nu_coarse
//! relaxations: here the level's iterate and its columns' line factors stay
//! in shared memory for the whole kernel. A colour's relaxation is one
//! phase between block barriers: each warp takes whole columns of the
//! colour, each lane evaluates r = b - A x at its P = ceil(nz / 32) levels
//! (adotx_body with the neighbours read from the shared iterate through
//! adotx_cell's resolved indices and mirror signs), and the factored Thomas
//! solve runs as two warp scans of the recurrences' affine maps (forward
//! e', backward x). The iterate returns to global memory at the end.
//! Shared memory: the iterate and D, 1/m, c' ([k][j][i], 4 * nx ny nz).
template <typename T, int P>
__global__ void __launch_bounds__(256) k_coarse_relax(gb_grid g, PBC b, int nrelax, T* x, const T* __restrict__ bv,
                                                      const T* __restrict__ AX, const T* __restrict__ AY,
                                                      const T* __restrict__ AZ, const T* __restrict__ J,
                                                      MeshRatios<T> m, const T* __restrict__ TD,
                                                      const T* __restrict__ TC, const T* __restrict__ TU)
{
    pdl_entry();
    constexpr unsigned kAll = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int plane = nx * ny * nz;
    T* xs = reinterpret_cast<T*>(smem_raw);
    T* sd = xs + plane;
    T* sm = sd + plane;
    T* sc = sm + plane;
    for (int n = threadIdx.x; n < plane; n += blockDim.x) {
        const int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
        const int64_t o = at(g, i, j, k);
        xs[n] = x[o];
        sd[n] = TD[o];
        sm[n] = TC[o];
        sc[n] = TU[o];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int half = (nx + 1) / 2;
    const int ncc = half * ny;
    for (int s = 0; s < nrelax; ++s) {
        for (int color = 0; color < 2; ++color) {
            for (int cc = warp; cc < ncc; cc += nwarps) {
                const int j = cc / half;
                const int i = 2 * (cc % half) + ((j + color) & 1);
                if (i >= nx) { continue; }
                int im, ip, sim, sip, jm, jp, sjm, sjp;
                resolve_neighbours(i, nx, b.per_x, b.sxl, b.sxh, im, ip, sim, sip);
                resolve_neighbours(j, ny, b.per_y, b.syl, b.syh, jm, jp, sjm, sjp);
                const int cx[3] = {im, i, ip}, cy[3] = {jm * nx, j * nx, jp * nx};
                const int sx3[3] = {sim, 1, sip}, sy3[3] = {sjm, 1, sjp};
                T R[P], D[P], IM[P], CP[P], X0[P];
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    const int k = min(lane * P + q, nz - 1);
                    const int km = (k == 0) ? 0 : k - 1, kp = (k == nz - 1) ? k : k + 1;
                    const int skm = (k == 0) ? b.szl : 1, skp = (k == nz - 1) ? b.szh : 1;
                    const int cz[3] = {km * nx * ny, k * nx * ny, kp * nx * ny};
                    const int sz3[3] = {skm, 1, skp};
                    auto X = [&](int di, int dj, int dk) {
                        const T v = xs[cx[di + 1] + cy[dj + 1] + cz[dk + 1]];
                        return (sx3[di + 1] * sy3[dj + 1] * sz3[dk + 1] < 0) ? -v : v;
                    };
                    const int64_t o = at(g, i, j, k);
                    const int n = cx[1] + cy[1] + cz[1];
                    R[q] = bv[o] - adotx_body<T, true>(g, b, i, j, k, o, X, AX, AY, AZ, J, m);
                    D[q] = sd[n];
                    IM[q] = sm[n];
                    CP[q] = sc[n];
                    X0[q] = xs[n];
                }
                __syncwarp();
                // e_k = (r_k - D_k e_{k-1}) / m_k over this lane's levels as e = al + be e_in, scanned over the lanes
                T al = T(0), be = T(1);
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    const int k = lane * P + q;
                    if (k < nz) {
                        if (k == 0) {
                            al = R[q] * IM[q];
                            be = T(0);
                        } else {
                            al = (R[q] - D[q] * al) * IM[q];
                            be = (-D[q] * be) * IM[q];
                        }
                    }
                }
                for (int d = 1; d < 32; d <<= 1) {
                    const T al2 = __shfl_up_sync(kAll, al, d), be2 = __shfl_up_sync(kAll, be, d);
                    if (lane >= d) {
                        al = al + be * al2;
                        be = be * be2;
                    }
                }
                T ep = __shfl_up_sync(kAll, al, 1);
                if (lane == 0) { ep = T(0); }
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    const int k = lane * P + q;
                    if (k < nz) {
                        ep = (k == 0) ? R[q] * IM[q] : (R[q] - D[q] * ep) * IM[q];
                        R[q] = ep;
                    }
                }
                // x_k = e_k - c'_k x_{k+1} over this lane's levels as x = ga + de x_in
                T ga = T(0), de = T(1);
#pragma unroll
                for (int q = P - 1; q >= 0; --q) {
                    const int k = lane * P + q;
                    if (k < nz) {
                        if (k == nz - 1) {
                            ga = R[q];
                            de = T(0);
                        } else {
                            ga = R[q] - CP[q] * ga;
                            de = -CP[q] * de;
                        }
                    }
                }
                for (int d = 1; d < 32; d <<= 1) {
                    const T ga2 = __shfl_down_sync(kAll, ga, d), de2 = __shfl_down_sync(kAll, de, d);
                    if (lane + d < 32) {
                        ga = ga + de * ga2;
                        de = de * de2;
                    }
                }
                T xk = __shfl_down_sync(kAll, ga, 1);
                if (lane == 31) { xk = T(0); }
#pragma unroll
                for (int q = P - 1; q >= 0; --q) {
                    const int k = lane * P + q;
                    if (k < nz) {
                        xk = (k == nz - 1) ? R[q] : R[q] - CP[q] * xk;
                        xs[cx[1] + cy[1] + k * nx * ny] = X0[q] + xk;
                    }
                }
                __syncwarp();
            }
            __syncthreads();
        }
    }
    for (int n = threadIdx.x; n < plane; n += blockDim.x) {
        const int i = n % nx, j = (n / nx) % ny, k = n / (nx * ny);
        x[at(g, i, j, k)] = xs[n];
    }
}

// ------------------------------------------------------ coarse-level tail ---
//
// The V-cycle below a level of at most GB_TUNE_MG_TAIL columns in ONE launch
// of one thread-block cluster (selectable; off by default, see tail_start).
// Every level there costs a handful of launches of a few microseconds each
// for little work, so the tail's levels run as
// phases of one kernel separated by cluster barriers (hardware, no spin):
// per level the pre-smoothing colours, the residual restricted to the next
// level (with its correction zeroed), the level below, the prolongation and
// the post-smoothing colours; on the coarsest level its nu_coarse
// relaxations. A colour's relaxation is one phase: each warp takes whole
// columns of the colour, each lane evaluates r = b - A x at its ceil(nz / 32)
// levels (adotx_cell, the per-level kernels' residual) and the column's
// factored Thomas solve runs as two warp scans of the recurrences' affine
// maps (forward e', backward x), so a column costs a few shuffle steps
// instead of nz dependent steps. A column's lateral neighbours are of the
// other colour, which this phase does not write (levels with a periodic
// direction of odd extent, where a column is its own colour's neighbour,
// keep the per-level launches). The restriction evaluates the four fine
// residuals of each coarse cell itself, so the residual never goes to memory.

namespace cg = cooperative_groups;

constexpr int kTailMaxLevels = 8;
constexpr int kTailThreads = 512;

template <typename T>
struct TailLevel {
    gb_grid g;
    PBC b;
    T* x;
    T* bv;
    const T* AX;
    const T* AY;
    const T* AZ;
    const T* J;
    MeshRatios<T> m;
    const T* TD;
    const T* TC;
    const T* TU;
};

template <typename T>
struct TailArgs {
    TailLevel<T> lv[kTailMaxLevels];
    int n;  // levels in the tail (the last is the coarsest)
    int nu1, nu2, nu_coarse;
};

//! One colour's zebra relaxation of a tail level: a warp per column.
template <typename T, int P>
__device__ __forceinline__ void tail_relax(const TailLevel<T>& v, int color, int warp, int nwarps, int lane)
{
    constexpr unsigned kAll = 0xffffffffu;
    const gb_grid& g = v.g;
    const int half = (g.nx + 1) / 2;
    const int ncc = half * g.ny;
    const int nz = g.nz;
    for (int cc = warp; cc < ncc; cc += nwarps) {
        const int j = cc / half;
        const int i = 2 * (cc % half) + ((j + color) & 1);
        if (i >= g.nx) { continue; }
        T R[P], D[P], IM[P], CP[P], X0[P];
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const int k = min(lane * P + q, nz - 1);
            const int64_t o = at(g, i, j, k);
            R[q] = v.bv[o] - adotx_cell<T>(g, v.b, i, j, k, v.x, v.AX, v.AY, v.AZ, v.J, v.m);
            D[q] = v.TD[o];
            IM[q] = v.TC[o];
            CP[q] = v.TU[o];
            X0[q] = v.x[o];
        }
        __syncwarp();
        // e_k = (r_k - D_k e_{k-1}) / m_k over this lane's levels as e = al + be e_in
        T al = T(0), be = T(1);
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const int k = lane * P + q;
            if (k < nz) {
                if (k == 0) {
                    al = R[q] * IM[q];
                    be = T(0);
                } else {
                    al = (R[q] - D[q] * al) * IM[q];
                    be = (-D[q] * be) * IM[q];
                }
            }
        }
        for (int d = 1; d < 32; d <<= 1) {
            const T al2 = __shfl_up_sync(kAll, al, d), be2 = __shfl_up_sync(kAll, be, d);
            if (lane >= d) {
                al = al + be * al2;
                be = be * be2;
            }
        }
        T ep = __shfl_up_sync(kAll, al, 1);
        if (lane == 0) { ep = T(0); }
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const int k = lane * P + q;
            if (k < nz) {
                ep = (k == 0) ? R[q] * IM[q] : (R[q] - D[q] * ep) * IM[q];
                R[q] = ep;
            }
        }
        // x_k = e_k - c'_k x_{k+1} over this lane's levels as x = ga + de x_in
        T ga = T(0), de = T(1);
#pragma unroll
        for (int q = P - 1; q >= 0; --q) {
            const int k = lane * P + q;
            if (k < nz) {
                if (k == nz - 1) {
                    ga = R[q];
                    de = T(0);
                } else {
                    ga = R[q] - CP[q] * ga;
                    de = -CP[q] * de;
                }
            }
        }
        for (int d = 1; d < 32; d <<= 1) {
            const T ga2 = __shfl_down_sync(kAll, ga, d), de2 = __shfl_down_sync(kAll, de, d);
            if (lane + d < 32) {
                ga = ga + de * ga2;
                de = de * de2;
            }
        }
        T xk = __shfl_down_sync(kAll, ga, 1);
        if (lane == 31) { xk = T(0); }
#pragma unroll
        for (int q = P - 1; q >= 0; --q) {
            const int k = lane * P + q;
            if (k < nz) {
                xk = (k == nz - 1) ? R[q] : R[q] - CP[q] * xk;
                v.x[at(g, i, j, k)] = X0[q] + xk;
            }
        }
        __syncwarp();
    }
}

//! The coarse right-hand side from the fine residual (restrict_cell with the
//! four fine residuals evaluated in place, as k_apply does) and the coarse
//! correction zeroed.
template <typename T>
__device__ __forceinline__ void tail_restrict(const TailLevel<T>& f, const TailLevel<T>& c, int t, int nt)
{
    const gb_grid& gf = f.g;
    const gb_grid& gc = c.g;
    const int n = gc.nx * gc.ny * gc.nz;
    for (int e = t; e < n; e += nt) {
        const int I = e % gc.nx, J2 = (e / gc.nx) % gc.ny, k = e / (gc.nx * gc.ny);
        const int i = 2 * I, j = 2 * J2;
        T r[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int ii = i + (q & 1), jj = j + (q >> 1);
            r[q] = f.bv[at(gf, ii, jj, k)] - adotx_cell<T>(gf, f.b, ii, jj, k, f.x, f.AX, f.AY, f.AZ, f.J, f.m);
        }
        const T s = (f.J[at(gf, i, j, k)] * r[0] + f.J[at(gf, i + 1, j, k)] * r[1])
                  + (f.J[at(gf, i, j + 1, k)] * r[2] + f.J[at(gf, i + 1, j + 1, k)] * r[3]);
        c.bv[at(gc, I, J2, k)] = s / (T(4) * c.J[at(gc, I, J2, k)]);
    }
    const int vol = static_cast<int>(volume(gc));
    for (int e = t; e < vol; e += nt) { c.x[e] = T(0); }
}

template <typename T>
__device__ __forceinline__ void tail_prolong(const TailLevel<T>& c, const TailLevel<T>& f, int t, int nt)
{
    const gb_grid& gf = f.g;
    const int n = gf.nx * gf.ny * gf.nz;
    for (int e = t; e < n; e += nt) {
        const int i = e % gf.nx, j = (e / gf.nx) % gf.ny, k = e / (gf.nx * gf.ny);
        prolong_cell<T>(c.g, c.b, c.x, gf, f.x, i, j, k);
    }
}

//! The tail of a V-cycle (TailArgs) as one cluster; P levels per lane.
template <typename T, int P>
__global__ void __launch_bounds__(kTailThreads) k_mg_tail(const __grid_constant__ TailArgs<T> a)
{
    cg::cluster_group cl = cg::this_cluster();
    const int nb = static_cast<int>(cl.num_blocks());
    const int rank = static_cast<int>(cl.block_rank());
    const int wpb = static_cast<int>(blockDim.x) / 32;
    const int warp = rank * wpb + static_cast<int>(threadIdx.x) / 32, nwarps = nb * wpb;
    const int lane = static_cast<int>(threadIdx.x) & 31;
    const int t = rank * static_cast<int>(blockDim.x) + static_cast<int>(threadIdx.x);
    const int nt = nb * static_cast<int>(blockDim.x);
    for (int l = 0; l < a.n - 1; ++l) {
        for (int s = 0; s < a.nu1; ++s) {
            for (int c = 0; c < 2; ++c) {
                tail_relax<T, P>(a.lv[l], c, warp, nwarps, lane);
                cl.sync();
            }
        }
        tail_restrict<T>(a.lv[l], a.lv[l + 1], t, nt);
        cl.sync();
    }
    for (int s = 0; s < a.nu_coarse; ++s) {
        for (int c = 0; c < 2; ++c) {
            tail_relax<T, P>(a.lv[a.n - 1], c, warp, nwarps, lane);
            cl.sync();
        }
    }
    for (int l = a.n - 2; l >= 0; --l) {
        tail_prolong<T>(a.lv[l + 1], a.lv[l], t, nt);
        cl.sync();
        for (int s = 0; s < a.nu2; ++s) {
            for (int c = 0; c < 2; ++c) {
                tail_relax<T, P>(a.lv[l], c, warp, nwarps, lane);
                cl.sync();
            }
        }
    }
}

// --------------------------------------------------------- vector ops ---

template <typename TD, typename TS>
__global__ void k_copy_valid(gb_grid g, TD* __restrict__ dst, const TS* __restrict__ src)
{
    int i, j, k;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (!cell_of(g, n, i, j, k)) { return; }
    const int64_t o = at(g, i, j, k);
    dst[o] = static_cast<TD>(src[o]);
}

template <typename T>
__global__ void k_convert_all(T* __restrict__ dst, const double* __restrict__ src, int64_t n)
{
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t < n) { dst[t] = static_cast<T>(src[t]); }
}

//! Partial sums of sum_q over rows... : per block, sum of a*b over the valid
//! cells (deterministic tree), one partial per (block, vector q).
__global__ void k_multidot(gb_grid g, const double* __restrict__ w, const double* __restrict__ V, int64_t vstride,
                           int nq, double* __restrict__ partial)
{
    __shared__ double red[kBlock / 32];
    const int q = blockIdx.y;
    const double* v = (q < 0) ? w : V + vstride * q;
    double s = 0;
    const int64_t ncell = static_cast<int64_t>(g.nx) * g.ny * g.nz;
    for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < ncell;
         n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        int i, j, k;
        cell_of(g, n, i, j, k);
        const int64_t o = at(g, i, j, k);
        s += w[o] * v[o];
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = s; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < kBlock / 32) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) { partial[static_cast<int64_t>(q) * gridDim.x + blockIdx.x] = t; }
    }
}

__global__ void k_reduce_partials(const double* __restrict__ partial, int nblk, int nq, double* __restrict__ out)
{
    const int q = blockIdx.x;
    __shared__ double red[32];
    double s = 0;
    for (int n = threadIdx.x; n < nblk; n += blockDim.x) { s += partial[static_cast<int64_t>(q) * nblk + n]; }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = s; }
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = (threadIdx.x < static_cast<int>(blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) { out[q] = t; }
    }
}

//! w -= sum_q h[q] V_q (valid cells).
__global__ void k_subtract_projection(gb_grid g, double* __restrict__ w, const double* __restrict__ V, int64_t vstride,
                                      int nq, const double* __restrict__ h)
{
    int i, j, k;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (!cell_of(g, n, i, j, k)) { return; }
    const int64_t o = at(g, i, j, k);
    double s = w[o];
    for (int q = 0; q < nq; ++q) { s -= h[q] * V[vstride * q + o]; }
    w[o] = s;
}

//! y = a x + b y (valid cells); with x null y = b y.
__global__ void k_axpby(gb_grid g, double a, const double* __restrict__ x, double b, double* __restrict__ y)
{
    int i, j, k;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (!cell_of(g, n, i, j, k)) { return; }
    const int64_t o = at(g, i, j, k);
    y[o] = (x ? a * x[o] : 0.0) + b * y[o];
}

//! phi += sum_q y[q] Z_q
__global__ void k_add_combination(gb_grid g, double* __restrict__ phi, const double* __restrict__ Z, int64_t vstride,
                                  int nq, const double* __restrict__ y)
{
    int i, j, k;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (!cell_of(g, n, i, j, k)) { return; }
    const int64_t o = at(g, i, j, k);
    double s = phi[o];
    for (int q = 0; q < nq; ++q) { s += y[q] * Z[vstride * q + o]; }
    phi[o] = s;
}

__global__ void k_add_const(gb_grid g, double* __restrict__ f, const double* __restrict__ c, double sign)
{
    int i, j, k;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (!cell_of(g, n, i, j, k)) { return; }
    f[at(g, i, j, k)] += sign * c[0];
}

}  // namespace

// ================================================================ host ===

namespace {

dim3 cols_grid(const gb_grid& g, int nk, int extra = 0)
{
    return dim3((g.nx + extra + 31) / 32, (g.ny + extra + 3) / 4, nk);
}
const dim3 kColsBlock(32, 4, 1);

template <typename T>
T* dalloc(cudaStream_t stream, std::vector<void*>& owned, int64_t n)
{
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * std::max<int64_t>(n, 1)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    // zeroed on the solver's stream: ordered before every later kernel of the
    // solver (a plain cudaMemset is not ordered against non-blocking streams)
    cudaMemsetAsync(p, 0, sizeof(T) * std::max<int64_t>(n, 1), stream);
    owned.push_back(p);
    return static_cast<T*>(p);
}

gb_grid coarse_grid(const gb_grid& f)
{
    gb_grid c = f;
    c.nx = f.nx / 2;
    c.ny = f.ny / 2;
    c.dx = 2 * f.dx;
    c.dy = 2 * f.dy;
    c.sy = c.nx + 1 + 2 * c.ng;
    c.sz = c.sy * (c.ny + 1 + 2 * c.ng);
    return c;
}

}  // namespace

template <typename T>
void PoissonLevels<T>::release()
{
    for (void* p : owned) { cudaFree(p); }
    owned.clear();
}

}  // namespace gb

gb_poisson::~gb_poisson()
{
    for (int n = 0; n < 2; ++n) {
        if (vc_exec[n] != nullptr) { cudaGraphExecDestroy(vc_exec[n]); }
    }
    if (capture_stream != nullptr) { cudaStreamDestroy(capture_stream); }
    for (void* p : owned) { cudaFree(p); }
    dl.release();
    fl.release();
    if (h_dots) { cudaFreeHost(h_dots); }
    if (h_step) { cudaFreeHost(h_step); }
}

namespace gb {

namespace {

//! Whether the operator over the array x takes the TMA-staged tiles
//! (GB_TUNE_MG_STENCIL = 2; never when x's base is not 16-byte aligned, as
//! the bulk copies need). Not the default: on config 1's fine level the
//! tiles measured 83 us per apply and 54 us per colour residual against 35
//! and 24 us for one thread per cell (ncu, cold): staging the iterate
//! leaves the other ten words of a cell as direct loads, whose latency is
//! what bounds the operator, and adds two block barriers per level.
template <typename T>
bool use_tiles(const gb_poisson* P, const gb_grid& g, const T* x)
{
    (void)g;
    if (P->ctx->tune[GB_TUNE_MG_STENCIL] != 2 || P->d_err == nullptr) { return false; }
    return (reinterpret_cast<uintptr_t>(x) & 15u) == 0;
}

template <typename T, bool COLOR>
void launch_tiles(gb_poisson* P, const gb_grid& g, const PBC& b, int color, const T* x, const T* AX, const T* AY,
                  const T* AZ, const T* J, const MeshRatios<T>& m, const T* rhs, T* y)
{
    using S = TileShape<T, COLOR>;
    const dim3 grid((g.nx + S::SPAN - 1) / S::SPAN, (g.ny + kTileJ - 1) / kTileJ, (g.nz + kTileK - 1) / kTileK);
    k_stencil_tile<T, COLOR><<<grid, dim3(kTileI, kTileJ), 0, P->ctx->stream>>>(g, b, color, x, AX, AY, AZ, J, m, rhs,
                                                                               y, P->d_err);
    ++P->ctx->launches;
}

//! Largest dynamic shared memory a relaxation kernel asks for.
constexpr size_t kSmoothSmemMax = 200 * 1024;

template <typename T>
void mg_smooth(gb_poisson* P, PoissonLevels<T>& L, int l)
{
    gb_ctx* ctx = P->ctx;
    const bool pdl = ctx->tune[GB_TUNE_PDL] != 1;
    const gb_grid& g = L.g[l];
    const PBC& b = L.b[l];
    constexpr int R = 4;
    const int nthr = 32;
    const size_t smem_ring = static_cast<size_t>(R * 4 + 2 * g.nz) * nthr * sizeof(T);
    const size_t smem_staged = static_cast<size_t>(5) * g.nz * nthr * sizeof(T);
    const bool staged = smem_staged <= kSmoothSmemMax;
    static std::atomic<bool> attr_done[2];  // set once per process (one device per process)
    const int ti = sizeof(T) == 8 ? 1 : 0;
    if (!attr_done[ti].load()) {
        cudaFuncSetAttribute(k_color_solve<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmoothSmemMax);
        cudaFuncSetAttribute(k_color_solve_staged<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmoothSmemMax);
        attr_done[ti].store(true);
    }
    const int half = (g.nx + 1) / 2;
    // one launch per colour (k_color_relax_fused) only on request
    // (GB_TUNE_MG_FUSED_RELAX 2: every level, 3: levels of at most
    // kFusedMaxColumns columns): on config 1 it measured slower than the two
    // launches on every level (the residual of the two-launch form runs one
    // thread per cell; the fused block serialises its columns' solves)
    constexpr int kFusedMaxColumns = 1024;
    const size_t smem_fused = static_cast<size_t>(5) * g.nz * kFusedCols * sizeof(T);
    const int fknob = ctx->tune[GB_TUNE_MG_FUSED_RELAX];
    // the segmented one-launch relaxation (GB_TUNE_MG_FUSED_RELAX 4): every
    // level of a column in flight, at most 16 segments of 4 levels (8 for
    // taller columns, or as GB_TUNE_LINE_SEGMENT asks). Measured slower than
    // the two launches on config 1 and on every tile shape the autotuner
    // timed (a coarse level's few blocks each walk 4 cells' stencils per
    // thread), so it is not the default.
    const int sknob = ctx->tune[GB_TUNE_LINE_SEGMENT];
    const int segL = (sknob == 4 || sknob == 8) ? sknob : ((g.nz + 3) / 4 <= 16 ? 4 : 8);
    const int segW = (g.nz + segL - 1) / segL;
    // (GB_TUNE_MG_FUSED_RELAX 5: the segmented one-launch form on the levels
    // of at least 4096 columns only, the two launches below)
    const bool seg = (fknob == 4 || (fknob == 5 && g.nx * g.ny >= 4096)) && segW <= 16
                     && !(g.periodic_x && (g.nx & 1)) && !(g.periodic_y && (g.ny & 1));
    if (seg) {
        const dim3 block(32, segW);
        const dim3 grid((half + 31) / 32, g.ny);
        const size_t sm = static_cast<size_t>(4) * segW * 32 * sizeof(T);
        for (int color = 0; color < 2; ++color) {
            Span span(ctx, GB_KERNEL_MG_SMOOTH);
            if (segL == 4) {
                k_color_relax_seg<T, 4><<<grid, block, sm, ctx->stream>>>(g, b, color, L.x[l], L.bv[l], L.AX[l], L.AY[l],
                                                                         L.AZ[l], L.J[l], L.ratios(l), L.TD[l],
                                                                         L.TC[l], L.TU[l]);
            } else {
                k_color_relax_seg<T, 8><<<grid, block, sm, ctx->stream>>>(g, b, color, L.x[l], L.bv[l], L.AX[l], L.AY[l],
                                                                         L.AZ[l], L.J[l], L.ratios(l), L.TD[l],
                                                                         L.TC[l], L.TU[l]);
            }
            ++ctx->launches;
        }
        return;
    }
    const bool fused = (fknob == 2 || (fknob == 3 && g.nx * g.ny <= kFusedMaxColumns)) && smem_fused <= kSmoothSmemMax
                       && !(g.periodic_x && (g.nx & 1)) && !(g.periodic_y && (g.ny & 1));
    if (fused) {
        static std::atomic<bool> fused_attr[2];
        if (!fused_attr[ti].load()) {
            cudaFuncSetAttribute(k_color_relax_fused<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmoothSmemMax);
            fused_attr[ti].store(true);
        }
        const dim3 fgrid((half + kFusedCols - 1) / kFusedCols, g.ny);
        for (int color = 0; color < 2; ++color) {
            Span span(ctx, GB_KERNEL_MG_SMOOTH);
            k_color_relax_fused<T><<<fgrid, 256, smem_fused, ctx->stream>>>(g, b, color, L.x[l], L.bv[l], L.AX[l], L.AY[l],
                                                                           L.AZ[l], L.J[l], L.ratios(l), L.TD[l],
                                                                           L.TC[l], L.TU[l]);
            ++ctx->launches;
        }
        return;
    }
    for (int color = 0; color < 2; ++color) {
        Span span(ctx, GB_KERNEL_MG_SMOOTH);
        if (use_tiles(P, g, L.x[l])) {
            launch_tiles<T, true>(P, g, b, color, L.x[l], L.AX[l], L.AY[l], L.AZ[l], L.J[l], L.ratios(l), L.bv[l],
                                  L.r[l]);
            --ctx->launches;  // counted with the solve below
        } else {
            const dim3 rgrid((half + 31) / 32, (g.ny + 3) / 4, g.nz);
            launch_pdl(pdl, k_color_residual<T>, rgrid, dim3(32, 4), 0, ctx->stream, g, b, color, L.x[l], L.bv[l],
                       L.AX[l], L.AY[l], L.AZ[l], L.J[l], L.ratios(l), L.r[l]);
        }
        const dim3 sgrid((half + nthr - 1) / nthr, g.ny);
        const int sL = (g.nz + 7) / 8 <= 16 ? 8 : 16;
        const int sW = (g.nz + sL - 1) / sL;
        if (ctx->tune[GB_TUNE_MG_SOLVE] != 1 && sW <= 16) {
            // the segmented column solves (the default; GB_TUNE_MG_SOLVE = 1: one thread per column)
            const size_t sm = static_cast<size_t>(4) * sW * 32 * sizeof(T);
            if (sL == 8) {
                launch_pdl(pdl, k_color_solve_seg<T, 8>, dim3((half + 31) / 32, g.ny), dim3(32, sW), sm, ctx->stream, g,
                           color, static_cast<const T*>(L.r[l]), static_cast<const T*>(L.TD[l]),
                           static_cast<const T*>(L.TC[l]), static_cast<const T*>(L.TU[l]), L.x[l]);
            } else {
                launch_pdl(pdl, k_color_solve_seg<T, 16>, dim3((half + 31) / 32, g.ny), dim3(32, sW), sm, ctx->stream,
                           g, color, static_cast<const T*>(L.r[l]), static_cast<const T*>(L.TD[l]),
                           static_cast<const T*>(L.TC[l]), static_cast<const T*>(L.TU[l]), L.x[l]);
            }
        } else if (staged) {
            launch_pdl(pdl, k_color_solve_staged<T>, sgrid, dim3(nthr), smem_staged, ctx->stream, g, color,
                       static_cast<const T*>(L.r[l]), static_cast<const T*>(L.TD[l]), static_cast<const T*>(L.TC[l]),
                       static_cast<const T*>(L.TU[l]), L.x[l]);
        } else {
            launch_pdl(pdl, k_color_solve<T, R>, sgrid, dim3(nthr), smem_ring, ctx->stream, g, color,
                       static_cast<const T*>(L.r[l]), static_cast<const T*>(L.TD[l]), static_cast<const T*>(L.TC[l]),
                       static_cast<const T*>(L.TU[l]), L.x[l]);
        }
        ctx->launches += 2;
    }
}

template <typename T>
void build_line_tridiag(gb_poisson* P, PoissonLevels<T>& L)
{
    gb_ctx* ctx = P->ctx;
    LineLevels<T> A{};
    A.n = P->nlev;
    A.cells[0] = 0;
    A.cols[0] = 0;
    for (int l = 0; l < P->nlev; ++l) {
        const gb_grid& g = L.g[l];
        A.g[l] = g;
        A.b[l] = L.b[l];
        A.AX[l] = L.AX[l];
        A.AY[l] = L.AY[l];
        A.AZ[l] = L.AZ[l];
        A.J[l] = L.J[l];
        A.z[l] = L.z[l];
        A.TD[l] = L.TD[l];
        A.TC[l] = L.TC[l];
        A.TU[l] = L.TU[l];
        A.cells[l + 1] = A.cells[l] + static_cast<int64_t>(g.nx) * g.ny * g.nz;
        A.cols[l + 1] = A.cols[l] + static_cast<int64_t>(g.nx) * g.ny;
    }
    k_line_tridiag_all<T><<<static_cast<unsigned>((A.cells[A.n] + 255) / 256), 256, 0, ctx->stream>>>(A);
    k_line_factor_all<T><<<static_cast<unsigned>((A.cols[A.n] + 127) / 128), 128, 0, ctx->stream>>>(A);
    ctx->launches += 2;
}

template <typename T>
void mg_residual(gb_poisson* P, PoissonLevels<T>& L, int l)
{
    gb_ctx* ctx = P->ctx;
    const gb_grid& g = L.g[l];
    Span span(ctx, GB_KERNEL_POISSON_APPLY);
    if (use_tiles(P, g, L.x[l])) {
        launch_tiles<T, false>(P, g, L.b[l], -1, L.x[l], L.AX[l], L.AY[l], L.AZ[l], L.J[l], L.ratios(l), L.bv[l],
                               L.r[l]);
        return;
    }
    launch_pdl(ctx->tune[GB_TUNE_PDL] != 1, k_apply<T>, cols_grid(g, g.nz), kColsBlock, 0, ctx->stream, g, L.b[l],
               static_cast<const T*>(L.x[l]), static_cast<const T*>(L.AX[l]), static_cast<const T*>(L.AY[l]),
               static_cast<const T*>(L.AZ[l]), static_cast<const T*>(L.J[l]), L.ratios(l),
               static_cast<const T*>(L.bv[l]), L.r[l]);
    ++ctx->launches;
}

//! The first level of the V-cycle's coarse tail (k_mg_tail), or -1: the
//! levels from it down have at most GB_TUNE_MG_TAIL's columns, at most 128
//! z-levels and no periodic direction of odd extent. Off by default: on
//! config 1 the per-level launches measured as fast with the tail on the
//! coarsest level alone and faster than any larger tail (0.464 ms per FP64
//! V-cycle with the per-level launches or a tail of the 2 x 2 level, 0.488
//! with the levels of at most 16 columns, 0.645 with those of at most 1024):
//! the cluster's 16 SMs take longer over the levels' work than all SMs take
//! over it plus the launches.
template <typename T>
int tail_start(const gb_poisson* P, const PoissonLevels<T>& L)
{
    const int knob = P->ctx->tune[GB_TUNE_MG_TAIL];
    if (knob < 2) { return -1; }
    const int maxcols = knob;
    int start = -1;
    for (int l = P->nlev - 1; l >= 0 && P->nlev - l <= kTailMaxLevels; --l) {
        const gb_grid& g = L.g[l];
        const bool ok = g.nx * g.ny <= maxcols && g.nz <= 128 && !(g.periodic_x && (g.nx & 1))
                        && !(g.periodic_y && (g.ny & 1));
        if (!ok) { break; }
        start = l;
    }
    return start;
}

//! One launch of the tail kernel as a cluster of 16 blocks where the device
//! schedules one (a non-portable size), else 8.
template <typename T, int PL>
cudaError_t launch_tail(gb_ctx* ctx, const TailArgs<T>& a)
{
    static std::atomic<int> csize{0};  // per instantiation, once per process (one device per process)
    int nc = csize.load();
    if (nc == 0) {
        nc = 8;
        if (cudaFuncSetAttribute(k_mg_tail<T, PL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
            cudaLaunchConfig_t q{};
            q.gridDim = dim3(16);
            q.blockDim = dim3(kTailThreads);
            cudaLaunchAttribute qa[1];
            qa[0].id = cudaLaunchAttributeClusterDimension;
            qa[0].val.clusterDim.x = 16;
            qa[0].val.clusterDim.y = 1;
            qa[0].val.clusterDim.z = 1;
            q.attrs = qa;
            q.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, k_mg_tail<T, PL>, &q) == cudaSuccess && nclusters > 0) {
                nc = 16;
            }
        }
        cudaGetLastError();
        csize.store(nc);
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(nc);
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = nc;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_mg_tail<T, PL>, a);
}

//! The V-cycle from level l down (l = tail_start) in one cluster launch.
template <typename T>
bool mg_tail(gb_poisson* P, PoissonLevels<T>& L, int l)
{
    gb_ctx* ctx = P->ctx;
    TailArgs<T> a{};
    a.n = P->nlev - l;
    a.nu1 = P->opt.nu1;
    a.nu2 = P->opt.nu2;
    a.nu_coarse = P->opt.nu_coarse;
    for (int q = 0; q < a.n; ++q) {
        const int m = l + q;
        TailLevel<T>& v = a.lv[q];
        v.g = L.g[m];
        v.b = L.b[m];
        v.x = L.x[m];
        v.bv = L.bv[m];
        v.AX = L.AX[m];
        v.AY = L.AY[m];
        v.AZ = L.AZ[m];
        v.J = L.J[m];
        v.m = L.ratios(m);
        v.TD = L.TD[m];
        v.TC = L.TC[m];
        v.TU = L.TU[m];
    }
    const int pl = (L.g[l].nz + 31) / 32;
    Span span(ctx, GB_KERNEL_MG_SMOOTH);
    cudaError_t e = cudaErrorInvalidValue;
    switch (pl) {
    case 1: e = launch_tail<T, 1>(ctx, a); break;
    case 2: e = launch_tail<T, 2>(ctx, a); break;
    case 3: e = launch_tail<T, 3>(ctx, a); break;
    case 4: e = launch_tail<T, 4>(ctx, a); break;
    default: break;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    ++ctx->launches;
    return true;
}

template <typename T>
void vcycle(gb_poisson* P, PoissonLevels<T>& L, int l)
{
    gb_ctx* ctx = P->ctx;
    const bool pdl = ctx->tune[GB_TUNE_PDL] != 1;
    if (l == tail_start(P, L) && mg_tail(P, L, l)) { return; }
    if (l == P->nlev - 1) {
        const gb_grid& g = L.g[l];
        const size_t smem = static_cast<size_t>(4) * g.nx * g.ny * g.nz * sizeof(T);
        const int pl = (g.nz + 31) / 32;
        const bool one_block = ctx->tune[GB_TUNE_MG_COARSE_KERNEL] != 1 && g.nx * g.ny <= 64 && smem <= kSmoothSmemMax
                               && pl <= 4 && !(g.periodic_x && (g.nx & 1)) && !(g.periodic_y && (g.ny & 1));
        if (one_block && P->opt.nu_coarse > 0) {
            static std::atomic<bool> attr_done[2];  // set once per process (one device per process)
            const int ti = sizeof(T) == 8 ? 1 : 0;
            if (!attr_done[ti].load()) {
                cudaFuncSetAttribute(k_coarse_relax<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmoothSmemMax);
                cudaFuncSetAttribute(k_coarse_relax<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmoothSmemMax);
                cudaFuncSetAttribute(k_coarse_relax<T, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmoothSmemMax);
                cudaFuncSetAttribute(k_coarse_relax<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmoothSmemMax);
                attr_done[ti].store(true);
            }
            Span span(ctx, GB_KERNEL_MG_SMOOTH);
#define GB_COARSE_ARGS g, L.b[l], P->opt.nu_coarse, L.x[l], static_cast<const T*>(L.bv[l]), \
                       static_cast<const T*>(L.AX[l]), static_cast<const T*>(L.AY[l]), static_cast<const T*>(L.AZ[l]), \
                       static_cast<const T*>(L.J[l]), L.ratios(l), static_cast<const T*>(L.TD[l]), \
                       static_cast<const T*>(L.TC[l]), static_cast<const T*>(L.TU[l])
            switch (pl) {
            case 1: launch_pdl(pdl, k_coarse_relax<T, 1>, dim3(1), dim3(256), smem, ctx->stream, GB_COARSE_ARGS); break;
            case 2: launch_pdl(pdl, k_coarse_relax<T, 2>, dim3(1), dim3(256), smem, ctx->stream, GB_COARSE_ARGS); break;
            case 3: launch_pdl(pdl, k_coarse_relax<T, 3>, dim3(1), dim3(256), smem, ctx->stream, GB_COARSE_ARGS); break;
            default: launch_pdl(pdl, k_coarse_relax<T, 4>, dim3(1), dim3(256), smem, ctx->stream, GB_COARSE_ARGS); break;
            }
#undef GB_COARSE_ARGS
            ++ctx->launches;
            return;
        }
        for (int s = 0; s < P->opt.nu_coarse; ++s) { mg_smooth(P, L, l); }
        return;
    }
    for (int s = 0; s < P->opt.nu1; ++s) { mg_smooth(P, L, l); }
    mg_residual(P, L, l);
    const gb_grid& gf = L.g[l];
    const gb_grid& gc = L.g[l + 1];
    {
        Span span(ctx, GB_KERNEL_MG_TRANSFER);
        launch_pdl(pdl, k_restrict<T>, cols_grid(gc, gc.nz), kColsBlock, 0, ctx->stream, gf,
                   static_cast<const T*>(L.J[l]), static_cast<const T*>(L.r[l]), gc, static_cast<const T*>(L.J[l + 1]),
                   L.bv[l + 1], L.x[l + 1]);
        ++ctx->launches;
    }
    vcycle(P, L, l + 1);
    {
        Span span(ctx, GB_KERNEL_MG_TRANSFER);
        launch_pdl(pdl, k_prolong_add<T>, cols_grid(gf, gf.nz), kColsBlock, 0, ctx->stream, gc, L.b[l + 1],
                   static_cast<const T*>(L.x[l + 1]), gf, L.x[l]);
        ++ctx->launches;
    }
    for (int s = 0; s < P->opt.nu2; ++s) { mg_smooth(P, L, l); }
}

//! A key of the tuning knobs that choose the V-cycle's kernels.
uint64_t tune_key(const gb_ctx* ctx)
{
    uint64_t k = 1469598103934665603ull;
    for (int n = 0; n < GB_N_TUNE; ++n) { k = (k ^ static_cast<uint64_t>(static_cast<uint32_t>(ctx->tune[n]))) * 1099511628211ull; }
    return k;
}

//! One V-cycle of the level hierarchy L from L.bv[0] into L.x[0]. The V-cycle
//! has no host synchronisation and its arguments are fixed per solver, so
//! from its second call on it runs as a CUDA graph, captured once on the
//! solver's own stream and launched on the context's: one launch in place of
//! the ~8 per level (the coarse levels' kernels last a few microseconds, so
//! launch overhead, not their work, set their cost). Profiling (per-family
//! events) and GB_TUNE_GRAPHS = 1 run it eagerly; the kernels and their
//! order are the same either way.
template <typename T>
void run_vcycle(gb_poisson* P, PoissonLevels<T>& L, int ti)
{
    gb_ctx* ctx = P->ctx;
    const bool graph = ctx->tune[GB_TUNE_GRAPHS] != 1 && !ctx->profiling;
    if (!graph || P->vc_calls[ti]++ == 0) {
        vcycle(P, L, 0);
        return;
    }
    const uint64_t key = tune_key(ctx);
    if (P->vc_exec[ti] != nullptr && P->vc_tune_key[ti] != key) {
        cudaGraphExecDestroy(P->vc_exec[ti]);
        P->vc_exec[ti] = nullptr;
    }
    if (P->vc_exec[ti] == nullptr) {
        if (P->capture_stream == nullptr
            && cudaStreamCreateWithFlags(&P->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            P->capture_stream = nullptr;
            vcycle(P, L, 0);
            return;
        }
        // the capture stream starts after the work queued so far on the context's
        cudaStream_t own = ctx->stream;
        const int64_t launches0 = ctx->launches;
        cudaGraph_t g = nullptr;
        ctx->stream = P->capture_stream;
        bool ok = cudaStreamBeginCapture(P->capture_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            vcycle(P, L, 0);
            ok = cudaStreamEndCapture(P->capture_stream, &g) == cudaSuccess && g != nullptr;
        }
        ctx->stream = own;
        const int64_t n = ctx->launches - launches0;
        ctx->launches = launches0;
        if (ok) { ok = cudaGraphInstantiate(&P->vc_exec[ti], g, 0) == cudaSuccess; }
        if (g != nullptr) { cudaGraphDestroy(g); }
        if (!ok) {
            cudaGetLastError();
            P->vc_exec[ti] = nullptr;
            vcycle(P, L, 0);
            return;
        }
        P->vc_launches[ti] = n;
        P->vc_tune_key[ti] = key;
    }
    cudaGraphLaunch(P->vc_exec[ti], ctx->stream);
    ctx->launches += P->vc_launches[ti];
}

//! e = one V-cycle for A e = r (FP64 vectors at the fine level).
void precondition(gb_poisson* P, const double* r, double* e)
{
    gb_ctx* ctx = P->ctx;
    const gb_grid& g = P->g;
    const int64_t ncell = static_cast<int64_t>(g.nx) * g.ny * g.nz;
    if (P->opt.precision == 1) {
        auto& L = P->fl;
        k_copy_valid<float, double><<<nblocks(ncell), kBlock, 0, ctx->stream>>>(g, L.bv[0], r);
        cudaMemsetAsync(L.x[0], 0, sizeof(float) * volume(g), ctx->stream);
        ctx->launches += 1;
        run_vcycle(P, L, 1);
        cudaMemsetAsync(e, 0, sizeof(double) * volume(g), ctx->stream);
        k_copy_valid<double, float><<<nblocks(ncell), kBlock, 0, ctx->stream>>>(g, e, L.x[0]);
        ctx->launches += 1;
    } else {
        auto& L = P->dl;
        cudaMemcpyAsync(L.bv[0], r, sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
        cudaMemsetAsync(L.x[0], 0, sizeof(double) * volume(g), ctx->stream);
        run_vcycle(P, L, 0);
        cudaMemcpyAsync(e, L.x[0], sizeof(double) * volume(g), cudaMemcpyDeviceToDevice, ctx->stream);
    }
}

void apply_fine(gb_poisson* P, const double* x, const double* rhs, double* y)
{
    gb_ctx* ctx = P->ctx;
    const gb_grid& g = P->g;
    Span span(ctx, GB_KERNEL_POISSON_APPLY);
    if (use_tiles(P, g, x)) {
        launch_tiles<double, false>(P, g, P->dl.b[0], -1, x, P->dl.AX[0], P->dl.AY[0], P->dl.AZ[0], P->dl.J[0],
                                    P->dl.ratios(0), rhs, y);
    } else {
        launch_pdl(ctx->tune[GB_TUNE_PDL] != 1, k_apply<double>, cols_grid(g, g.nz), kColsBlock, 0, ctx->stream, g,
                   P->dl.b[0], x, static_cast<const double*>(P->dl.AX[0]), static_cast<const double*>(P->dl.AY[0]),
                   static_cast<const double*>(P->dl.AZ[0]), static_cast<const double*>(P->dl.J[0]), P->dl.ratios(0),
                   rhs, y);
        ++ctx->launches;
    }
    if (P->cross_ad != nullptr) {
        // PoissonSolver::Op::apply (Source/Poisson.cpp:148-156): the split
        // correction on top (subtracted when y is the residual rhs - A x)
        k_add_cross<<<cols_grid(g, g.nz), kColsBlock, 0, ctx->stream>>>(g, P->dl.b[0], x, P->cross_ad, P->dl.J[0],
                                                                          P->dl.ratios(0), rhs ? -1.0 : 1.0, y);
        ++ctx->launches;
    }
}

//! Dots <w, V_q> for q < nq into out[0, nq) on the device (deterministic
//! two-stage block sums; no host synchronisation).
void multidot_device(gb_poisson* P, const double* w, const double* V, int64_t vstride, int nq, double* out)
{
    gb_ctx* ctx = P->ctx;
    const int nblk = P->dot_blocks;
    Span span(ctx, GB_KERNEL_VECTOR);
    k_multidot<<<dim3(nblk, nq), kBlock, 0, ctx->stream>>>(P->g, w, V, vstride, nq, P->d_partial);
    k_reduce_partials<<<nq, 256, 0, ctx->stream>>>(P->d_partial, nblk, nq, out);
    ctx->launches += 2;
}

//! The next Arnoldi vector v = w / |w| (0 where |w| is not > 0), |w|^2 read
//! from the device (the host's 1/sqrt in the same IEEE operations).
__global__ void k_scale_by_norm(gb_grid g, const double* __restrict__ w, const double* __restrict__ n2,
                                double* __restrict__ v)
{
    int i, j, k;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (!cell_of(g, n, i, j, k)) { return; }
    const double hn = sqrt(*n2);
    if (!(hn > 0)) { return; }
    const int64_t o = at(g, i, j, k);
    v[o] = (1.0 / hn) * w[o];
}

//! Dots <w, V_q> for q < nq (or <a, b> with V = b, nq = 1) into P->h_dots (host), deterministic.
gb_status multidot(gb_poisson* P, const double* w, const double* V, int64_t vstride, int nq, double* host_out)
{
    gb_ctx* ctx = P->ctx;
    const gb_grid& g = P->g;
    const int nblk = P->dot_blocks;
    {
        Span span(ctx, GB_KERNEL_VECTOR);
        k_multidot<<<dim3(nblk, nq), kBlock, 0, ctx->stream>>>(g, w, V, vstride, nq, P->d_partial);
        k_reduce_partials<<<nq, 256, 0, ctx->stream>>>(P->d_partial, nblk, nq, P->d_dots);
        ctx->launches += 2;
    }
    cudaMemcpyAsync(P->h_dots, P->d_dots, sizeof(double) * nq, cudaMemcpyDeviceToHost, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("poisson dot"); }
    std::copy(P->h_dots, P->h_dots + nq, host_out);
    return GB_OK;
}

}  // namespace

// ------------------------------------------------------------ creation ---

gb_status poisson_build(gb_poisson* P)
{
    gb_ctx* ctx = P->ctx;
    // levels (FP64 geometry for every level, the FP32 copies when asked)
    std::vector<gb_grid> grids{P->g};
    while (static_cast<int>(grids.size()) < P->opt.max_levels) {
        const gb_grid& c = grids.back();
        const bool can = (c.nx % 2 == 0) && (c.ny % 2 == 0) && (c.nx / 2 >= P->opt.min_coarse) && (c.ny / 2 >= P->opt.min_coarse);
        if (!can) { break; }
        grids.push_back(coarse_grid(c));
    }
    P->nlev = static_cast<int>(grids.size());
    auto& D = P->dl;
    for (int l = 0; l < P->nlev; ++l) {
        const gb_grid& g = grids[l];
        D.g[l] = g;
        D.b[l] = make_pbc(g, P->bc, P->bc[2] != PF_DIRICHLET);
        const int64_t vol = volume(g);
        if (l == 0) {
            D.z[l] = const_cast<double*>(P->z_fine);
            D.J[l] = const_cast<double*>(P->J_fine);
        } else {
            D.z[l] = dalloc<double>(ctx->stream, D.owned, vol);
            D.J[l] = dalloc<double>(ctx->stream, D.owned, vol);
        }
        D.AX[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.AY[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.AZ[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.x[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.bv[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.r[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.snap[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.TD[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.TC[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.TU[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.RX[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.RY[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.HZ[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.SX[l] = dalloc<double>(ctx->stream, D.owned, vol);
        D.SY[l] = dalloc<double>(ctx->stream, D.owned, vol);
        if (!D.TD[l] || !D.TC[l] || !D.TU[l] || !D.RX[l] || !D.RY[l] || !D.HZ[l] || !D.SX[l] || !D.SY[l]) {
            set_error("gust: PoissonSolver: cannot allocate the multigrid levels");
            return GB_OOM;
        }
        if (!D.AX[l] || !D.AY[l] || !D.AZ[l] || !D.x[l] || !D.bv[l] || !D.r[l] || !D.snap[l] || (l > 0 && (!D.z[l] || !D.J[l]))) {
            set_error("gust: PoissonSolver: cannot allocate the multigrid levels");
            return GB_OOM;
        }
        if (l > 0) {
            const gb_grid& gf = grids[l - 1];
            const int64_t nz3 = static_cast<int64_t>(g.nx + 3) * (g.ny + 3) * (g.nz + 3);
            k_coarse_z<<<nblocks(nz3), kBlock, 0, ctx->stream>>>(g, D.z[l], gf, D.z[l - 1]);
            double* ax = dalloc<double>(ctx->stream, D.owned, vol);
            double* ay = dalloc<double>(ctx->stream, D.owned, vol);
            double* zcc = dalloc<double>(ctx->stream, D.owned, vol);
            const int64_t nm = static_cast<int64_t>(g.nx + 3) * (g.ny + 3) * (g.nz + 2);
            k_metrics<<<nblocks(nm), kBlock, 0, ctx->stream>>>(g, D.z[l], D.J[l], ax, ay, zcc);
            ctx->launches += 2;
        }
        const int64_t nr = static_cast<int64_t>(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
        k_mesh_ratios<double><<<nblocks(nr), kBlock, 0, ctx->stream>>>(g, D.z[l], D.RX[l], D.RY[l], D.HZ[l], D.SX[l],
                                                                       D.SY[l]);
        ++ctx->launches;
    }
    if (P->opt.precision == 1) {
        auto& F = P->fl;
        for (int l = 0; l < P->nlev; ++l) {
            const gb_grid& g = grids[l];
            F.g[l] = g;
            F.b[l] = D.b[l];
            const int64_t vol = volume(g);
            F.z[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.J[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.AX[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.AY[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.AZ[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.x[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.bv[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.r[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.snap[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.TD[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.TC[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.TU[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.RX[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.RY[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.HZ[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.SX[l] = dalloc<float>(ctx->stream, F.owned, vol);
            F.SY[l] = dalloc<float>(ctx->stream, F.owned, vol);
            if (!F.TD[l] || !F.TC[l] || !F.TU[l] || !F.RX[l] || !F.RY[l] || !F.HZ[l] || !F.SX[l] || !F.SY[l]) {
                set_error("gust: PoissonSolver: cannot allocate the FP32 multigrid levels");
                return GB_OOM;
            }
            const int64_t nr = static_cast<int64_t>(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
            k_mesh_ratios<float><<<nblocks(nr), kBlock, 0, ctx->stream>>>(g, D.z[l], F.RX[l], F.RY[l], F.HZ[l],
                                                                          F.SX[l], F.SY[l]);
            ++ctx->launches;
            if (!F.z[l] || !F.J[l] || !F.AX[l] || !F.AY[l] || !F.AZ[l] || !F.x[l] || !F.bv[l] || !F.r[l] || !F.snap[l]) {
                set_error("gust: PoissonSolver: cannot allocate the FP32 multigrid levels");
                return GB_OOM;
            }
            k_convert_all<float><<<nblocks(vol), kBlock, 0, ctx->stream>>>(F.z[l], D.z[l], vol);
            k_convert_all<float><<<nblocks(vol), kBlock, 0, ctx->stream>>>(F.J[l], D.J[l], vol);
            ctx->launches += 2;
        }
    }
    // Krylov workspace
    const int64_t vol = volume(P->g);
    const int m = P->opt.restart;
    // the basis columns at a stride of whole 256-byte lines: every column's
    // base is 16-byte aligned, as the TMA-staged operator tiles need
    P->vstride = (vol + 31) / 32 * 32;
    P->V = dalloc<double>(ctx->stream, P->owned, P->vstride * (m + 1));
    P->Zv = dalloc<double>(ctx->stream, P->owned, P->vstride * m);
    P->w = dalloc<double>(ctx->stream, P->owned, vol);
    P->t = dalloc<double>(ctx->stream, P->owned, vol);
    P->dot_blocks = std::min(4 * ctx->num_sms, nblocks(static_cast<int64_t>(P->g.nx) * P->g.ny * P->g.nz));
    P->d_partial = dalloc<double>(ctx->stream, P->owned, static_cast<int64_t>(P->dot_blocks) * (m + 2));
    P->d_dots = dalloc<double>(ctx->stream, P->owned, m + 2);
    P->d_coef = dalloc<double>(ctx->stream, P->owned, m + 2);
    P->d_step = dalloc<double>(ctx->stream, P->owned, 3 * (m + 2));
    P->d_err = dalloc<unsigned long long>(ctx->stream, P->owned, 1);
    if (!P->V || !P->Zv || !P->w || !P->t || !P->d_partial || !P->d_dots || !P->d_coef || !P->d_err) {
        set_error("gust: PoissonSolver: cannot allocate the Krylov workspace");
        return GB_OOM;
    }
    if (cudaMallocHost(&P->h_step, sizeof(double) * 3 * (m + 2)) != cudaSuccess) {
        cudaGetLastError();
        P->h_step = nullptr;
        set_error("gust: PoissonSolver: out of pinned host memory");
        return GB_OOM;
    }
    if (cudaMallocHost(&P->h_dots, sizeof(double) * (m + 2)) != cudaSuccess) {
        cudaGetLastError();
        set_error("gust: PoissonSolver: cannot allocate pinned host words");
        return GB_OOM;
    }
    return check_cuda("PoissonSolver");
}

gb_status poisson_set_coeffs(gb_poisson* P, const double* ax, const double* ay, const double* az, const double* bx,
                             const double* by, const double* bz)
{
    gb_ctx* ctx = P->ctx;
    auto& D = P->dl;
    const gb_grid& g = P->g;
    const int64_t vol = volume(g);
    // premultiplied areas a beta (Source/Poisson.cpp:442-447)
    const double* a[3] = {ax, ay, az};
    const double* b[3] = {bx, by, bz};
    double* out[3] = {D.AX[0], D.AY[0], D.AZ[0]};
    for (int d = 0; d < 3; ++d) {
        cudaMemcpyAsync(out[d], a[d], sizeof(double) * vol, cudaMemcpyDeviceToDevice, ctx->stream);
        if (b[d]) { multiply_inplace(ctx, out[d], b[d], vol); }
    }
    for (int l = 1; l < P->nlev; ++l) {
        const gb_grid& gc = D.g[l];
        k_coarse_areas<<<cols_grid(gc, gc.nz + 1, 1), kColsBlock, 0, ctx->stream>>>(
            gc, D.AX[l], D.AY[l], D.AZ[l], D.g[l - 1], D.AX[l - 1], D.AY[l - 1], D.AZ[l - 1]);
        ++ctx->launches;
    }
    if (P->opt.precision == 1) {
        auto& F = P->fl;
        for (int l = 0; l < P->nlev; ++l) {
            const int64_t v = volume(F.g[l]);
            k_convert_all<float><<<nblocks(v), kBlock, 0, ctx->stream>>>(F.AX[l], D.AX[l], v);
            k_convert_all<float><<<nblocks(v), kBlock, 0, ctx->stream>>>(F.AY[l], D.AY[l], v);
            k_convert_all<float><<<nblocks(v), kBlock, 0, ctx->stream>>>(F.AZ[l], D.AZ[l], v);
            ctx->launches += 3;
        }
    }
    if (P->opt.precision == 1) { build_line_tridiag(P, P->fl); } else { build_line_tridiag(P, P->dl); }
    P->coeffs_set = true;
    return check_cuda("PoissonSolver::set_coeffs");
}

__global__ void k_multiply(double* __restrict__ a, const double* __restrict__ b, int64_t n)
{
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t < n) { a[t] *= b[t]; }
}

void multiply_inplace(gb_ctx* ctx, double* a, const double* b, int64_t n)
{
    k_multiply<<<nblocks(n), kBlock, 0, ctx->stream>>>(a, b, n);
    ++ctx->launches;
}

__global__ void k_cross_coeffs(int64_t n, const double* __restrict__ az, const double* __restrict__ bz,
                               const double* __restrict__ zc, double* __restrict__ d, double* __restrict__ ad)
{
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= n) { return; }
    const double v = (bz ? bz[t] : 1.0) - zc[t];
    d[t] = v;
    ad[t] = az[t] * v;
}

gb_status poisson_set_z_cross(gb_poisson* P, const double* az, const double* bz, const double* z_cross)
{
    gb_ctx* ctx = P->ctx;
    if (z_cross == nullptr) {
        P->cross_d = P->cross_ad = nullptr;  // the arrays stay owned until the solver goes
        return GB_OK;
    }
    if (P->bc[2] == GB_POISSON_DIRICHLET) {
        set_error("gust: FaceCoeffs::z_cross with a Dirichlet ground is not supported");
        return GB_BAD_ARG;
    }
    const int64_t vol = volume(P->g);
    if (P->cross_store[0] == nullptr) {
        P->cross_store[0] = dalloc<double>(ctx->stream, P->owned, vol);
        P->cross_store[1] = dalloc<double>(ctx->stream, P->owned, vol);
        if (!P->cross_store[0] || !P->cross_store[1]) {
            set_error("gust: PoissonSolver::set_z_cross: cannot allocate the split coefficients");
            return GB_OOM;
        }
    }
    P->cross_d = P->cross_store[0];
    P->cross_ad = P->cross_store[1];
    // FaceCoeffs::z_cross (Source/Poisson.cpp:461-479): d = (beta_z or 1) - z_cross
    k_cross_coeffs<<<nblocks(vol), kBlock, 0, ctx->stream>>>(vol, az, bz, z_cross, P->cross_d, P->cross_ad);
    ++ctx->launches;
    return check_cuda("PoissonSolver::set_z_cross");
}

gb_status poisson_apply(gb_poisson* P, const double* phi, double* y)
{
    apply_fine(P, phi, nullptr, y);
    return check_cuda("PoissonSolver::apply");
}

gb_status poisson_vcycle(gb_poisson* P, const double* r, double* e)
{
    precondition(P, r, e);
    return check_cuda("PoissonSolver::vcycle");
}

gb_status poisson_fluxes(gb_poisson* P, const double* phi, const double* bx, const double* by, const double* bz,
                         double* fx, double* fy, double* fz)
{
    gb_ctx* ctx = P->ctx;
    const gb_grid& g = P->g;
    if (P->bc[2] == PF_DIRICHLET) {
        // the pressure correction's fluxes have a zero-flux ground; a Dirichlet
        // ground's one-sided flux is in the operator (the Tucker solve) only
        set_error("gust: PoissonSolver::fluxes with a Dirichlet ground is not supported");
        return GB_BAD_ARG;
    }
    Span span(ctx, GB_KERNEL_POISSON_APPLY);
    k_fluxes<<<cols_grid(g, g.nz + 1, 1), kColsBlock, 0, ctx->stream>>>(g, P->dl.b[0], phi, P->dl.ratios(0), bx, by, bz, fx,
                                                                        fy, fz);
    ++ctx->launches;
    if (P->cross_d != nullptr) {
        k_cross_flux<<<cols_grid(g, g.nz + 1), kColsBlock, 0, ctx->stream>>>(g, P->dl.b[0], phi, P->cross_d,
                                                                              P->dl.ratios(0), fz);
        ++ctx->launches;
    }
    return check_cuda("PoissonSolver::fluxes");
}

//! J-weighted mean of the valid cells of f into d_coef[slot] (device) and host.
gb_status weighted_mean(gb_poisson* P, const double* f, double* host_mean, int slot)
{
    double num = 0, den = 0;
    gb_status st = multidot(P, P->dl.J[0], f, 0, 1, &num);
    if (st != GB_OK) { return st; }
    if (P->J_sum == 0) {
        // sum of J: <J, 1> via a ones vector in t
        gb_ctx* ctx = P->ctx;
        const int64_t vol = volume(P->g);
        k_fill<<<nblocks(vol), kBlock, 0, ctx->stream>>>(P->t, vol, 1.0);
        ++ctx->launches;
        if ((st = multidot(P, P->dl.J[0], P->t, 0, 1, &den)) != GB_OK) { return st; }
        P->J_sum = den;
    }
    *host_mean = num / P->J_sum;
    cudaMemcpyAsync(P->d_coef + slot, host_mean, sizeof(double), cudaMemcpyHostToDevice, P->ctx->stream);
    return GB_OK;
}

gb_status poisson_solve(gb_poisson* P, double* rhs, double* phi, gb_poisson_result* res)
{
    gb_ctx* ctx = P->ctx;
    const gb_grid& g = P->g;
    const int64_t ncell = static_cast<int64_t>(g.nx) * g.ny * g.nz;
    const int64_t vol = volume(g);
    const int m = P->opt.restart;
    *res = gb_poisson_result{};
    bool singular = true;
    for (int f = 0; f < 6; ++f) {
        if (P->bc[f] == PF_DIRICHLET) { singular = false; }
    }
    res->singular = singular ? 1 : 0;
    gb_status st;
    if (singular) {
        double mean = 0;
        if ((st = weighted_mean(P, rhs, &mean, m + 1)) != GB_OK) { return st; }
        res->removed_mean = mean;
        k_add_const<<<nblocks(ncell), kBlock, 0, ctx->stream>>>(g, rhs, P->d_coef + m + 1, -1.0);
        ++ctx->launches;
    }
    cudaMemsetAsync(phi, 0, sizeof(double) * vol, ctx->stream);
    double bn2 = 0;
    if ((st = multidot(P, rhs, rhs, 0, 1, &bn2)) != GB_OK) { return st; }
    const double bnorm = std::sqrt(bn2);
    res->initial_residual = bnorm;
    const double tol = std::max(P->opt.reltol * bnorm, P->opt.abstol);
    std::vector<double> H(static_cast<size_t>(m + 1) * m), cs(m), sn(m), s(m + 1), y(m), h(m + 1);
    int it = 0;
    bool converged = !(bnorm > tol);
    while (!converged && it < P->opt.max_iter) {
        apply_fine(P, phi, rhs, P->w);  // w = rhs - A phi
        double b2 = 0;
        if ((st = multidot(P, P->w, P->w, 0, 1, &b2)) != GB_OK) { return st; }
        const double beta = std::sqrt(b2);
        if (!(beta > tol)) {
            converged = true;
            break;
        }
        if (!std::isfinite(beta)) {
            set_error("gust: the Poisson solve produced a non-finite residual");
            return GB_NONFINITE;
        }
        cudaMemsetAsync(P->V, 0, sizeof(double) * vol, ctx->stream);
        k_axpby<<<nblocks(ncell), kBlock, 0, ctx->stream>>>(g, 1.0 / beta, P->w, 0.0, P->V);
        ++ctx->launches;
        std::fill(s.begin(), s.end(), 0.0);
        std::fill(H.begin(), H.end(), 0.0);
        s[0] = beta;
        int jj = 0;
        for (; jj < m && it < P->opt.max_iter; ++jj) {
            ++it;
            double* vj = P->V + P->vstride * jj;
            double* zj = P->Zv + P->vstride * jj;
            precondition(P, vj, zj);
            apply_fine(P, zj, nullptr, P->w);
            // classical Gram-Schmidt, twice, and the norm of what is left: the
            // dots stay on the device (each projection reads its coefficients
            // there) and come back to the host once per step, for the Givens
            // rotations and the convergence test
            std::fill(h.begin(), h.end(), 0.0);
            const int64_t st3 = m + 2;
            for (int pass = 0; pass < 2; ++pass) {
                double* dots = P->d_step + pass * st3;
                multidot_device(P, P->w, P->V, P->vstride, jj + 1, dots);
                k_subtract_projection<<<nblocks(ncell), kBlock, 0, ctx->stream>>>(g, P->w, P->V, P->vstride, jj + 1,
                                                                                   dots);
                ++ctx->launches;
            }
            multidot_device(P, P->w, P->w, 0, 1, P->d_step + 2 * st3);
            double* vn = P->V + P->vstride * (jj + 1);
            cudaMemsetAsync(vn, 0, sizeof(double) * vol, ctx->stream);
            k_scale_by_norm<<<nblocks(ncell), kBlock, 0, ctx->stream>>>(g, P->w, P->d_step + 2 * st3, vn);
            ++ctx->launches;
            cudaMemcpyAsync(P->h_step, P->d_step, sizeof(double) * 3 * st3, cudaMemcpyDeviceToHost, ctx->stream);
            if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("poisson dot"); }
            for (int pass = 0; pass < 2; ++pass) {
                for (int q = 0; q <= jj; ++q) { h[q] += P->h_step[pass * st3 + q]; }
            }
            const double hn = std::sqrt(P->h_step[2 * st3]);
            for (int q = 0; q <= jj; ++q) { H[q * m + jj] = h[q]; }
            H[(jj + 1) * m + jj] = hn;
            for (int q = 0; q < jj; ++q) {
                const double a = H[q * m + jj], b2q = H[(q + 1) * m + jj];
                H[q * m + jj] = cs[q] * a + sn[q] * b2q;
                H[(q + 1) * m + jj] = -sn[q] * a + cs[q] * b2q;
            }
            const double a = H[jj * m + jj], b2j = H[(jj + 1) * m + jj];
            const double rr = std::sqrt(a * a + b2j * b2j);
            cs[jj] = (rr > 0) ? a / rr : 1.0;
            sn[jj] = (rr > 0) ? b2j / rr : 0.0;
            H[jj * m + jj] = rr;
            H[(jj + 1) * m + jj] = 0;
            s[jj + 1] = -sn[jj] * s[jj];
            s[jj] = cs[jj] * s[jj];
            if (std::fabs(s[jj + 1]) <= tol) {
                ++jj;
                break;
            }
        }
        for (int q = jj - 1; q >= 0; --q) {
            double acc = s[q];
            for (int p = q + 1; p < jj; ++p) { acc -= H[q * m + p] * y[p]; }
            y[q] = acc / H[q * m + q];
        }
        cudaMemcpyAsync(P->d_coef, y.data(), sizeof(double) * jj, cudaMemcpyHostToDevice, ctx->stream);
        k_add_combination<<<nblocks(ncell), kBlock, 0, ctx->stream>>>(g, phi, P->Zv, P->vstride, jj, P->d_coef);
        ++ctx->launches;
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("poisson solve"); }
    }
    if (singular) {
        double mean = 0;
        if ((st = weighted_mean(P, phi, &mean, m + 1)) != GB_OK) { return st; }
        k_add_const<<<nblocks(ncell), kBlock, 0, ctx->stream>>>(g, phi, P->d_coef + m + 1, -1.0);
        ++ctx->launches;
    }
    apply_fine(P, phi, rhs, P->w);
    double r2 = 0;
    if ((st = multidot(P, P->w, P->w, 0, 1, &r2)) != GB_OK) { return st; }
    res->final_residual = std::sqrt(r2);
    res->iterations = it;
    if (!std::isfinite(res->final_residual)) {
        set_error("gust: the Poisson solve returned non-finite values");
        return GB_NONFINITE;
    }
    {
        unsigned long long tile_err = 0;
        cudaMemcpyAsync(&tile_err, P->d_err, sizeof(tile_err), cudaMemcpyDeviceToHost, ctx->stream);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { return check_cuda("PoissonSolver::solve"); }
        if (tile_err != 0) {
            cudaMemsetAsync(P->d_err, 0, sizeof(tile_err), ctx->stream);
            set_error("gust: the Poisson solve: a wait for a TMA-staged operator tile gave up");
            return GB_TIMEOUT;
        }
    }
    if (!(res->final_residual <= tol * (1 + 1e-7)) && !converged) {
        set_error("gust: the Poisson solve did not converge in solver.poisson_max_iter = %d iterations (residual %g of "
                  "%g; solver.poisson_reltol = %g, solver.poisson_abstol = %g)",
                  P->opt.max_iter, res->final_residual, res->initial_residual, P->opt.reltol, P->opt.abstol);
        return GB_NOT_CONVERGED;
    }
    return check_cuda("PoissonSolver::solve");
}

// ------------------------------------------------------ free functions ---

gb_status mesh_metrics(gb_ctx* ctx, const gb_grid& g, const double* z, double* J, double* ax, double* ay, double* az,
                       double* zcc)
{
    const int64_t vol = volume(g);
    cudaMemsetAsync(J, 0, sizeof(double) * vol, ctx->stream);
    cudaMemsetAsync(ax, 0, sizeof(double) * vol, ctx->stream);
    cudaMemsetAsync(ay, 0, sizeof(double) * vol, ctx->stream);
    cudaMemsetAsync(zcc, 0, sizeof(double) * vol, ctx->stream);
    k_fill<<<nblocks(vol), kBlock, 0, ctx->stream>>>(az, vol, 1.0);
    const int64_t nm = static_cast<int64_t>(g.nx + 3) * (g.ny + 3) * (g.nz + 2);
    k_metrics<<<nblocks(nm), kBlock, 0, ctx->stream>>>(g, z, J, ax, ay, zcc);
    ctx->launches += 2;
    return check_cuda("mesh_metrics");
}

gb_status face_divergence(gb_ctx* ctx, const gb_grid& g, const double* ax, const double* ay, const double* az,
                          const double* J, const double* fx, const double* fy, const double* fz, double* div)
{
    Span span(ctx, GB_KERNEL_MASSFLUX);
    k_face_divergence<<<cols_grid(g, g.nz), kColsBlock, 0, ctx->stream>>>(g, ax, ay, az, J, fx, fy, fz, div);
    ++ctx->launches;
    return check_cuda("face_divergence");
}

template struct PoissonLevels<double>;
template struct PoissonLevels<float>;

}  // namespace gb
