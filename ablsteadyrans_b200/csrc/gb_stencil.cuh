// Staggered-grid stencils of the terrain-following C-grid (the reference's
// Source/Stencil_K.H:18-129), specialised at compile time on the location
// types, and a box launcher for one-thread-per-point kernels.
//
// A location type is a bit mask: bit d set means nodal in direction d (CC
// cell centres, XF/YF/ZF faces, their XOR pairs the edges, NODE the nodes).
#pragma once

#include "gb_common.cuh"

namespace gb {
namespace st {

constexpr int CC = 0, XF = 1, YF = 2, ZF = 4, NODE = 7, NONE = 3;

__host__ __device__ constexpr bool nodal(int t, int d) { return ((t >> d) & 1) != 0; }
__host__ __device__ constexpr int face(int c) { return 1 << c; }
__host__ __device__ constexpr int lo_off(int tq, int ts, int d) { return (nodal(tq, d) == nodal(ts, d) || nodal(tq, d)) ? 0 : -1; }
__host__ __device__ constexpr int npts(int tq, int ts, int d) { return (nodal(tq, d) == nodal(ts, d)) ? 1 : 2; }
__host__ __device__ constexpr int flux_lo(int ts, int d) { return nodal(ts, d) ? -1 : 0; }

//! Value of q (type TQ) at the TS location (i, j, k): the mean of the
//! bracketing points, summed in the order z, y, x (Stencil_K.H:46-74).
template <int TQ, int TS, typename T>
__device__ __forceinline__ T interp(const T* __restrict__ q, const gb_grid& g, int i, int j, int k)
{
    constexpr int lx = lo_off(TQ, TS, 0), ly = lo_off(TQ, TS, 1), lz = lo_off(TQ, TS, 2);
    constexpr int nx = npts(TQ, TS, 0), ny = npts(TQ, TS, 1), nz = npts(TQ, TS, 2);
    T s = T(0);
#pragma unroll
    for (int c = 0; c < nz; ++c) {
#pragma unroll
        for (int b = 0; b < ny; ++b) {
#pragma unroll
            for (int a = 0; a < nx; ++a) { s += q[at(g, i + lx + a, j + ly + b, k + lz + c)]; }
        }
    }
    return s * (T(1) / T(nx * ny * nz));
}

//! d q / d(index M) at the TS location (Stencil_K.H:76-92).
template <int TQ, int TS, int M, typename T>
__device__ __forceinline__ T deriv(const T* __restrict__ q, const gb_grid& g, int i, int j, int k)
{
    constexpr bool same = (nodal(TQ, M) == nodal(TS, M));
    constexpr int m0 = same ? -1 : lo_off(TQ, TS, M);
    constexpr int m1 = same ? 1 : m0 + 1;
    constexpr int ex = (M == 0) ? 1 : 0, ey = (M == 1) ? 1 : 0, ez = (M == 2) ? 1 : 0;
    constexpr int lx = (M == 0) ? 0 : lo_off(TQ, TS, 0), ly = (M == 1) ? 0 : lo_off(TQ, TS, 1),
                  lz = (M == 2) ? 0 : lo_off(TQ, TS, 2);
    constexpr int nx = (M == 0) ? 1 : npts(TQ, TS, 0), ny = (M == 1) ? 1 : npts(TQ, TS, 1),
                  nz = (M == 2) ? 1 : npts(TQ, TS, 2);
    const T w = same ? T(0.5) : T(1);
    T s = T(0);
#pragma unroll
    for (int c = 0; c < nz; ++c) {
#pragma unroll
        for (int b = 0; b < ny; ++b) {
#pragma unroll
            for (int a = 0; a < nx; ++a) {
                const int ii = i + lx + a, jj = j + ly + b, kk = k + lz + c;
                s += q[at(g, ii + m1 * ex, jj + m1 * ey, kk + m1 * ez)] - q[at(g, ii + m0 * ex, jj + m0 * ey, kk + m0 * ez)];
            }
        }
    }
    return w * (s * (T(1) / T(nx * ny * nz)));
}

template <typename T>
struct Metric {
    T zx, zy, zz;
};

//! Slopes of the coordinate surface and z_zeta at a location (Stencil_K.H:103-110).
template <int TS, typename T>
__device__ __forceinline__ Metric<T> metric_at(const T* __restrict__ z, const gb_grid& g, int i, int j, int k)
{
    return {deriv<NODE, TS, 0>(z, g, i, j, k) * T(1.0 / g.dx), deriv<NODE, TS, 1>(z, g, i, j, k) * T(1.0 / g.dy),
            deriv<NODE, TS, 2>(z, g, i, j, k) * T(1.0 / g.dzeta)};
}

//! Physical gradient (Stencil_K.H:115-124).
template <int TQ, int TS, typename T>
__device__ __forceinline__ void grad_at(const T* __restrict__ q, const gb_grid& g, int i, int j, int k, const Metric<T>& m,
                                        T out[3])
{
    const T qx = deriv<TQ, TS, 0>(q, g, i, j, k) * T(1.0 / g.dx);
    const T qy = deriv<TQ, TS, 1>(q, g, i, j, k) * T(1.0 / g.dy);
    const T qz = deriv<TQ, TS, 2>(q, g, i, j, k) * T(1.0 / g.dzeta) / m.zz;
    out[0] = qx - m.zx * qz;
    out[1] = qy - m.zy * qz;
    out[2] = qz;
}

}  // namespace st

//! An index box [lo, hi] (inclusive) in the grid's index space.
struct Box {
    int lo[3], hi[3];
    __host__ __device__ int64_t count() const
    {
        return static_cast<int64_t>(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
    }
};

//! The valid points of a location type.
inline Box valid_box(const gb_grid& g, int t)
{
    return Box{{0, 0, 0}, {g.nx - 1 + (t & 1), g.ny - 1 + ((t >> 1) & 1), g.nz - 1 + ((t >> 2) & 1)}};
}

template <typename F>
__global__ void k_box(Box b, F f)
{
    pdl_entry();
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int nx = b.hi[0] - b.lo[0] + 1, ny = b.hi[1] - b.lo[1] + 1;
    if (n >= b.count()) { return; }
    const int i = b.lo[0] + static_cast<int>(n % nx);
    const int j = b.lo[1] + static_cast<int>((n / nx) % ny);
    const int k = b.lo[2] + static_cast<int>(n / (static_cast<int64_t>(nx) * ny));
    f(i, j, k);
}

//! One thread per point of b (i fastest), on the context's stream.
template <typename F>
void for_box(gb_ctx* ctx, const Box& b, F f, int family = -1)
{
    const int64_t n = b.count();
    if (n <= 0) { return; }
    if (family >= 0) { span_begin(ctx, family); }
    launch_pdl(ctx->tune[GB_TUNE_PDL] != 1, k_box<F>, dim3(static_cast<unsigned>((n + 255) / 256)), dim3(256), 0,
               ctx->stream, b, f);
    if (family >= 0) { span_end(ctx); }
    ++ctx->launches;
}

}  // namespace gb
