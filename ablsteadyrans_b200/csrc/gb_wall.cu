// Tucker's differential wall distance on the GPU (the reference's
// tucker_wall_distance, Source/WallDistance.cpp:78-94, with its
// distance_from_phi, :13-62, and the ghost extension of
// Source/Sequencing.cpp:43-60): one terrain Poisson solve of
// laplacian(phi) = -1 with phi = 0 on the ground (tucker_bc,
// Source/WallDistance.cpp:65-76: periodic lateral directions stay periodic,
// the other lateral faces and the top carry no flux), then
//   d = -|grad phi| + sqrt(|grad phi|^2 + 2 phi)
// with ERF's cell-centred physical gradient, cell by cell.
#include "gb_common.cuh"
#include "gb_poisson.cuh"

#include <cmath>

namespace gb {

namespace {

__global__ void k_fill_valid(gb_grid g, double* __restrict__ a, double v)
{
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= static_cast<int64_t>(g.nx) * g.ny * g.nz) { return; }
    const int i = static_cast<int>(n % g.nx), j = static_cast<int>((n / g.nx) % g.ny);
    const int k = static_cast<int>(n / (static_cast<int64_t>(g.nx) * g.ny));
    a[at(g, i, j, k)] = v;
}

//! The solution's value at a lateral or upper neighbour of a valid cell with
//! the Tucker conditions' ghosts: a periodic image, or across a zero-flux
//! face the cell itself (an even copy); the ground's odd ghost only enters
//! the centred z difference of the first cell, which the one-sided form
//! replaces.
__device__ __forceinline__ double phi_at(const gb_grid& g, const double* __restrict__ p, int i, int j, int k)
{
    if (i < 0) { i = g.periodic_x ? i + g.nx : -1 - i; } else if (i >= g.nx) { i = g.periodic_x ? i - g.nx : 2 * g.nx - 1 - i; }
    if (j < 0) { j = g.periodic_y ? j + g.ny : -1 - j; } else if (j >= g.ny) { j = g.periodic_y ? j - g.ny : 2 * g.ny - 1 - j; }
    if (k >= g.nz) { k = 2 * g.nz - 1 - k; }
    if (k < 0) { return -p[at(g, i, j, -1 - k)]; }
    return p[at(g, i, j, k)];
}

//! distance_from_phi (Source/WallDistance.cpp:13-62) on the valid cells.
__global__ void k_tucker_distance(gb_grid g, const double* __restrict__ z, const double* __restrict__ p,
                                  double* __restrict__ d)
{
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= static_cast<int64_t>(g.nx) * g.ny * g.nz) { return; }
    const int i = static_cast<int>(n % g.nx), j = static_cast<int>((n / g.nx) % g.ny);
    const int k = static_cast<int>(n / (static_cast<int64_t>(g.nx) * g.ny));
    const double dxinv = 1.0 / g.dx, dyinv = 1.0 / g.dy, dzinv = 1.0 / g.dzeta;
#define ZN(a, b, c) z[at(g, a, b, c)]
    const double dpdxi = 0.5 * (phi_at(g, p, i + 1, j, k) - phi_at(g, p, i - 1, j, k)) * dxinv;
    const double dpdeta = 0.5 * (phi_at(g, p, i, j + 1, k) - phi_at(g, p, i, j - 1, k)) * dyinv;
    const double dpdzeta = 0.5 * (phi_at(g, p, i, j, k + 1) - phi_at(g, p, i, j, k - 1)) * dzinv;
    const double h_zeta = 0.25 * dzinv * (ZN(i + 1, j, k + 1) + ZN(i + 1, j + 1, k + 1) + ZN(i, j, k + 1)
                                          + ZN(i, j + 1, k + 1) - ZN(i + 1, j, k) - ZN(i + 1, j + 1, k)
                                          - ZN(i, j, k) - ZN(i, j + 1, k));
    const double h_xi = 0.25 * dxinv * (ZN(i + 1, j, k) + ZN(i + 1, j + 1, k) + ZN(i + 1, j, k + 1)
                                        + ZN(i + 1, j + 1, k + 1) - ZN(i, j, k) - ZN(i, j + 1, k)
                                        - ZN(i, j, k + 1) - ZN(i, j + 1, k + 1));
    const double h_eta = 0.25 * dyinv * (ZN(i, j + 1, k) + ZN(i + 1, j + 1, k) + ZN(i, j + 1, k + 1)
                                         + ZN(i + 1, j + 1, k + 1) - ZN(i, j, k) - ZN(i + 1, j, k)
                                         - ZN(i, j, k + 1) - ZN(i + 1, j, k + 1));
    double dpdz = dpdzeta / h_zeta;
    if (k == 0) {
        // the quadratic along the column through phi = 0 on the ground and the
        // two lowest cell centres, a and b above the ground
        const double zw = 0.25 * (ZN(i, j, 0) + ZN(i + 1, j, 0) + ZN(i, j + 1, 0) + ZN(i + 1, j + 1, 0));
        const double c1 = 0.25 * (ZN(i, j, 1) + ZN(i + 1, j, 1) + ZN(i, j + 1, 1) + ZN(i + 1, j + 1, 1));
        const double c2 = 0.25 * (ZN(i, j, 2) + ZN(i + 1, j, 2) + ZN(i, j + 1, 2) + ZN(i + 1, j + 1, 2));
        const double a = 0.5 * (zw + c1) - zw;
        const double b = 0.5 * (c1 + c2) - zw;
        dpdz = (p[at(g, i, j, 0)] * b * (b - 2.0 * a) + phi_at(g, p, i, j, 1) * a * a) / (a * b * (b - a));
    }
#undef ZN
    const double dpdx = dpdxi - h_xi * dpdz;
    const double dpdy = dpdeta - h_eta * dpdz;
    const double g2 = dpdx * dpdx + dpdy * dpdy + dpdz * dpdz;
    d[at(g, i, j, k)] = -sqrt(g2) + sqrt(g2 + 2.0 * p[at(g, i, j, k)]);
}

//! extend_by_zero_gradient (Source/Sequencing.cpp:43-60): every ghost of d
//! takes the valid cell of its periodic image or, across a non-periodic
//! face, the nearest one.
__global__ void k_extend_distance(gb_grid g, double* __restrict__ d)
{
    const int ng = g.ng;
    const int ex = g.nx + 1 + 2 * ng, ey = g.ny + 1 + 2 * ng, ez = g.nz + 1 + 2 * ng;
    const int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (n >= static_cast<int64_t>(ex) * ey * ez) { return; }
    const int i = static_cast<int>(n % ex) - ng, j = static_cast<int>((n / ex) % ey) - ng;
    const int k = static_cast<int>(n / (static_cast<int64_t>(ex) * ey)) - ng;
    if (i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz) { return; }
    const int ii = g.periodic_x ? ((i % g.nx) + g.nx) % g.nx : min(max(i, 0), g.nx - 1);
    const int jj = g.periodic_y ? ((j % g.ny) + g.ny) % g.ny : min(max(j, 0), g.ny - 1);
    const int kk = min(max(k, 0), g.nz - 1);
    d[at(g, i, j, k)] = d[at(g, ii, jj, kk)];
}

}  // namespace

}  // namespace gb

extern "C" {

gb_status gb_tucker_wall_distance(gb_ctx* ctx, const gb_grid* g, const double* z_nd, const gb_poisson_opts* opt,
                                  double* dist, gb_poisson_result* res)
{
    gb::clear_error();
    if (ctx == nullptr || z_nd == nullptr || dist == nullptr || res == nullptr) {
        gb::set_error("gust: tucker_wall_distance: null argument");
        return GB_BAD_ARG;
    }
    gb_status st = gb::check_grid("tucker_wall_distance", g);
    if (st != GB_OK) { return st; }
    if (g->nz < 3) {
        gb::set_error("gust: tucker_wall_distance: needs nz >= 3 (the first cell's quadratic uses two cells above it)");
        return GB_BAD_ARG;
    }
    gb_poisson_opts o{};
    if (opt != nullptr) {
        o = *opt;
    } else if ((st = gb_poisson_options_default(&o)) != GB_OK) {
        return st;
    }
    const int64_t vol = gb::volume(*g);
    double* buf = nullptr;
    if (cudaMalloc(&buf, sizeof(double) * vol * 6) != cudaSuccess) {
        cudaGetLastError();
        gb::set_error("gust: tucker_wall_distance: cannot allocate its work arrays");
        return GB_OOM;
    }
    double* J = buf;
    double* ax = buf + vol;
    double* ay = buf + 2 * vol;
    double* az = buf + 3 * vol;
    double* rhs = buf + 4 * vol;
    double* phi = buf + 5 * vol;
    cudaMemsetAsync(buf, 0, sizeof(double) * vol * 6, ctx->stream);
    gb_poisson* P = nullptr;
    // the cell-centre heights go to dist, which the distance overwrites everywhere
    st = gb_mesh_metrics(ctx, g, z_nd, J, ax, ay, az, dist);
    if (st == GB_OK) {
        const int32_t lat_x = g->periodic_x ? gb::PF_PERIODIC : gb::PF_NEUMANN;
        const int32_t lat_y = g->periodic_y ? gb::PF_PERIODIC : gb::PF_NEUMANN;
        const int32_t bc[6] = {lat_x, lat_y, gb::PF_DIRICHLET, lat_x, lat_y, gb::PF_NEUMANN};
        st = gb_poisson_create(ctx, g, bc, z_nd, J, &o, &P);
    }
    if (st == GB_OK) { st = gb_poisson_set_coeffs(P, ax, ay, az, nullptr, nullptr, nullptr); }
    const int64_t cells = static_cast<int64_t>(g->nx) * g->ny * g->nz;
    const unsigned blocks = static_cast<unsigned>((cells + 255) / 256);
    if (st == GB_OK) {
        gb::k_fill_valid<<<blocks, 256, 0, ctx->stream>>>(*g, rhs, -1.0);
        st = gb_poisson_solve(P, rhs, phi, res);
    }
    if (st == GB_OK) {
        gb::k_tucker_distance<<<blocks, 256, 0, ctx->stream>>>(*g, z_nd, phi, dist);
        const int64_t all = static_cast<int64_t>(g->nx + 1 + 2 * g->ng) * (g->ny + 1 + 2 * g->ng) * (g->nz + 1 + 2 * g->ng);
        gb::k_extend_distance<<<static_cast<unsigned>((all + 255) / 256), 256, 0, ctx->stream>>>(*g, dist);
        ctx->launches += 3;
        st = gb::check_cuda("tucker_wall_distance");
    }
    if (P != nullptr) { gb_poisson_destroy(P); }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(buf);
    return st;
}

}  // extern "C"
