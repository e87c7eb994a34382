// Device kernels of the terrain-following Poisson operator, shared by the
// operator apply, the fluxes and the multigrid smoother (templated on the
// arithmetic type: FP64 for the defect residual, FP32 for the inner solver).
//
// Ghost values are never filled by separate launches: a read outside the
// valid cells is resolved by index arithmetic into the source cell and the
// mirror sign of the face (the composition of the reference's fills, x, then
// y, then z, Source/Poisson.cpp:84-125 and ERF_TerrainPoisson.cpp:103-210, is
// a product of per-direction reflections and periodic shifts, so it does not
// depend on the fill order).
#pragma once

#include "gb_common.cuh"

namespace gb {

enum { PF_PERIODIC = 0, PF_NEUMANN = 1, PF_DIRICHLET = 2 };
enum { TP_XLO = 1, TP_XHI = 2, TP_YLO = 4, TP_YHI = 8, TP_ZLO = 16, TP_ZHI = 32 };
//! zf bit: a Dirichlet ground (phi = 0 on it: the odd ghost below the ground
//! and the ground-face flux, Source/Poisson.cpp:158-189)
enum { TP_DGROUND = 64 };

//! Boundary description of one Poisson level: periodic flags, the mirror
//! sign of each non-periodic face (+1 Neumann, -1 Dirichlet), and the
//! zero-flux faces (the Neumann faces, ground excepted: ERF_TerrainPoisson.cpp:53-66).
struct PBC {
    int per_x, per_y;
    int sxl, sxh, syl, syh, szl, szh;
    int zf;
};

inline PBC make_pbc(const gb_grid& g, const int* bc, bool ground_even)
{
    PBC b;
    b.per_x = g.periodic_x;
    b.per_y = g.periodic_y;
    auto sgn = [](int f) { return f == PF_DIRICHLET ? -1 : 1; };
    b.sxl = sgn(bc[0]);
    b.syl = sgn(bc[1]);
    b.szl = ground_even ? 1 : sgn(bc[2]);
    b.sxh = sgn(bc[3]);
    b.syh = sgn(bc[4]);
    b.szh = sgn(bc[5]);
    b.zf = 0;
    if (!g.periodic_x && bc[0] == PF_NEUMANN) { b.zf |= TP_XLO; }
    if (!g.periodic_x && bc[3] == PF_NEUMANN) { b.zf |= TP_XHI; }
    if (!g.periodic_y && bc[1] == PF_NEUMANN) { b.zf |= TP_YLO; }
    if (!g.periodic_y && bc[4] == PF_NEUMANN) { b.zf |= TP_YHI; }
    if (bc[5] == PF_NEUMANN) { b.zf |= TP_ZHI; }
    if (bc[2] == PF_DIRICHLET) { b.zf |= TP_DGROUND; }
    return b;
}

//! x(i, j, k) of a cell field with its one ghost layer resolved for the BC.
//! `wrap` (may equal x) serves the reads that cross a periodic seam.
template <typename T>
__device__ __forceinline__ T ldc(const T* x, const T* wrap, const gb_grid& g, const PBC& b,
                                 int i, int j, int k)
{
    int s = 1;
    const T* src = x;
    if (i < 0) {
        if (b.per_x) { i += g.nx; src = wrap; } else { s *= b.sxl; i = -1 - i; }
    } else if (i >= g.nx) {
        if (b.per_x) { i -= g.nx; src = wrap; } else { s *= b.sxh; i = 2 * g.nx - 1 - i; }
    }
    if (j < 0) {
        if (b.per_y) { j += g.ny; src = wrap; } else { s *= b.syl; j = -1 - j; }
    } else if (j >= g.ny) {
        if (b.per_y) { j -= g.ny; src = wrap; } else { s *= b.syh; j = 2 * g.ny - 1 - j; }
    }
    if (k < 0) { s *= b.szl; k = -1 - k; } else if (k >= g.nz) { s *= b.szh; k = 2 * g.nz - 1 - k; }
    const T v = src[at(g, i, j, k)];
    return (s < 0) ? -v : v;
}

//! The mesh-only factors of the operator, precomputed once per level from the
//! node heights (they do not depend on the coefficients or the iterate):
//!   rx(I, j, K) = h_xi / h_zeta on the x-z edge at x-node I, z-node K,
//!   ry(i, J, K) = h_eta / h_zeta on the y-z edge at y-node J, z-node K,
//!   hz(i, j, K) = 1 / (h_zeta / 8) on z-face K,
//!   sx(i, j, K), sy(i, j, K) = the x and y slopes of z-face K,
//! each the exact expression terrpoisson_adotx evaluates inline
//! (ERF_TerrainPoisson_3D_K.H:316-530), so the products are unchanged.
template <typename T>
struct MeshRatios {
    const T* __restrict__ rx;
    const T* __restrict__ ry;
    const T* __restrict__ hz;
    const T* __restrict__ sx;
    const T* __restrict__ sy;
    const T* __restrict__ zn;  // the level's node heights (the Dirichlet ground's one-sided flux)
};

//! One value of the iterate at offset (di, dj, dk) from cell (i, j, k) at
//! flat index o: a direct load inside, the BC-resolved ghost otherwise.
template <typename T, bool INTERIOR>
__device__ __forceinline__ T xoff(const T* x, const gb_grid& g, const PBC& b, int64_t o, int i, int j,
                                  int k, int di, int dj, int dk)
{
    if (INTERIOR) { return x[o + di + dj * g.sy + dk * g.sz]; }
    return ldc<T>(x, x, g, b, i + di, j + dj, k + dk);
}

//! terrpoisson_flux_zlo_dir (ERF_TerrainPoisson_3D_K.H:214-275): the ground
//! face's flux of column (i, j) with phi = 0 on the ground (one-sided), the
//! iterate's values at the ground level read by X(di, dj, 0) (resolved
//! lateral neighbours), the node heights from zn.
template <typename T, typename XA>
__device__ __forceinline__ T ground_flux_dir(const gb_grid& g, int i, int j, XA&& X, const T* __restrict__ zn)
{
    const int k = 0;
    const T dxinv = static_cast<T>(1.0 / g.dx), dyinv = static_cast<T>(1.0 / g.dy);
    const T h = T(0.5), q = T(0.25);
#define ZN(a, b, c) zn[at(g, a, b, c)]
    const T x00 = X(0, 0, 0);
    T pz_lo = x00;
    const T hzeta_inv_on_zlo = T(8) / ((ZN(i, j, k + 1) + ZN(i + 1, j, k + 1) + ZN(i, j + 1, k + 1) + ZN(i + 1, j + 1, k + 1))
                                       - (ZN(i, j, k) + ZN(i + 1, j, k) + ZN(i, j + 1, k) + ZN(i + 1, j + 1, k)));
    pz_lo *= hzeta_inv_on_zlo;
    const T px_hi_md_lo = T(0), px_lo_md_lo = T(0), py_md_hi_lo = T(0), py_md_lo_lo = T(0);
    T h_xi, h_eta, h_zeta;
    T pz_hi_md_lo = h * (X(1, 0, 0) + x00);
    h_xi = q * (ZN(i + 2, j, k) - ZN(i, j, k) + ZN(i + 2, j + 1, k) - ZN(i, j + 1, k)) * dxinv;
    h_zeta = q * (ZN(i + 1, j, k + 1) - ZN(i + 1, j, k) + ZN(i + 1, j + 1, k + 1) - ZN(i + 1, j + 1, k));
    pz_hi_md_lo *= h_xi / h_zeta;
    T pz_lo_md_lo = h * (x00 + X(-1, 0, 0));
    h_xi = q * (ZN(i + 1, j, k) - ZN(i - 1, j, k) + ZN(i + 1, j + 1, k) - ZN(i - 1, j + 1, k)) * dxinv;
    h_zeta = q * (ZN(i, j, k + 1) - ZN(i, j, k) + ZN(i, j + 1, k + 1) - ZN(i, j + 1, k));
    pz_lo_md_lo *= h_xi / h_zeta;
    T pz_md_hi_lo = h * (X(0, 1, 0) + x00);
    h_eta = q * (ZN(i, j + 2, k) - ZN(i, j, k) + ZN(i + 1, j + 2, k) - ZN(i + 1, j, k)) * dyinv;
    h_zeta = q * (ZN(i, j + 1, k + 1) - ZN(i, j + 1, k) + ZN(i + 1, j + 1, k + 1) - ZN(i + 1, j + 1, k));
    pz_md_hi_lo *= h_eta / h_zeta;
    T pz_md_lo_lo = h * (x00 + X(0, -1, 0));
    h_eta = q * (ZN(i, j + 1, k) - ZN(i, j - 1, k) + ZN(i + 1, j + 1, k) - ZN(i + 1, j - 1, k)) * dyinv;
    h_zeta = q * (ZN(i, j, k + 1) - ZN(i, j, k) + ZN(i + 1, j, k + 1) - ZN(i + 1, j, k));
    pz_md_lo_lo *= h_eta / h_zeta;
    const T h_xi_on_zlo = h * (ZN(i + 1, j + 1, k) + ZN(i + 1, j, k) - ZN(i, j + 1, k) - ZN(i, j, k)) * dxinv;
    const T h_eta_on_zlo = h * (ZN(i + 1, j + 1, k) + ZN(i, j + 1, k) - ZN(i + 1, j, k) - ZN(i, j, k)) * dyinv;
#undef ZN
    pz_lo -= h * h_xi_on_zlo * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo));
    pz_lo -= h * h_eta_on_zlo * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));
    return -pz_lo;
}

//! The terrain operator at cell (i, j, k) with the iterate's 15 values read by
//! X(di, dj, dk): terrpoisson_adotx (ERF_TerrainPoisson_3D_K.H:316-530) with
//! the premultiplied areas a beta and the zero-flux mask (MASKS: the cell may
//! touch a boundary), the mesh ratios precomputed (MeshRatios): the same
//! operations in the same order on the same values, without its ~19
//! divisions per cell.
template <typename T, bool MASKS, typename XA>
__device__ __forceinline__ T adotx_body(const gb_grid& g, const PBC& b, int i, int j, int k, int64_t o, XA&& X,
                                        const T* __restrict__ axa, const T* __restrict__ aya, const T* __restrict__ aza,
                                        const T* __restrict__ Jc, const MeshRatios<T>& m)
{
    const T dxinv = static_cast<T>(1.0 / g.dx), dyinv = static_cast<T>(1.0 / g.dy), dzinv = static_cast<T>(1.0 / g.dzeta);
    const T h = T(0.5);
    const T x000 = X(0, 0, 0), xp00 = X(1, 0, 0), xm00 = X(-1, 0, 0), x0p0 = X(0, 1, 0), x0m0 = X(0, -1, 0);
    const T x00p = X(0, 0, 1), x00m = X(0, 0, -1);
    const T xp0p = X(1, 0, 1), xp0m = X(1, 0, -1), xm0p = X(-1, 0, 1), xm0m = X(-1, 0, -1);
    const T x0pp = X(0, 1, 1), x0pm = X(0, 1, -1), x0mp = X(0, -1, 1), x0mm = X(0, -1, -1);
    const int sy = static_cast<int>(g.sy), sz = static_cast<int>(g.sz);
    T px_hi = (xp00 - x000) * dxinv;
    T pz_hi_md_hi = h * (xp0p + x00p - xp00 - x000);
    pz_hi_md_hi *= m.rx[o + 1 + sz];
    T pz_hi_md_lo = h * (xp00 + x000 - xp0m - x00m);
    pz_hi_md_lo *= m.rx[o + 1];
    px_hi -= h * (pz_hi_md_hi + pz_hi_md_lo);

    T px_lo = (x000 - xm00) * dxinv;
    T pz_lo_md_hi = h * (x00p + xm0p - x000 - xm00);
    pz_lo_md_hi *= m.rx[o + sz];
    T pz_lo_md_lo = h * (x000 + xm00 - x00m - xm0m);
    pz_lo_md_lo *= m.rx[o];
    px_lo -= h * (pz_lo_md_hi + pz_lo_md_lo);

    T py_hi = (x0p0 - x000) * dyinv;
    T pz_md_hi_hi = h * (x0pp + x00p - x0p0 - x000);
    pz_md_hi_hi *= m.ry[o + sy + sz];
    T pz_md_hi_lo = h * (x0p0 + x000 - x0pm - x00m);
    pz_md_hi_lo *= m.ry[o + sy];
    py_hi -= h * (pz_md_hi_hi + pz_md_hi_lo);

    T py_lo = (x000 - x0m0) * dyinv;
    T pz_md_lo_hi = h * (x00p + x0mp - x000 - x0m0);
    pz_md_lo_hi *= m.ry[o + sz];
    T pz_md_lo_lo = h * (x000 + x0m0 - x00m - x0mm);
    pz_md_lo_lo *= m.ry[o];
    py_lo -= h * (pz_md_lo_hi + pz_md_lo_lo);

    T pz_hi = x00p - x000;
    pz_hi *= m.hz[o + sz];
    const T px_hi_md_hi = h * (xp0p - x00p + xp00 - x000) * dxinv;
    const T px_lo_md_hi = h * (x00p - xm0p + x000 - xm00) * dxinv;
    const T py_md_hi_hi = h * (x0pp - x00p + x0p0 - x000) * dyinv;
    const T py_md_lo_hi = h * (x00p - x0mp + x000 - x0m0) * dyinv;
    pz_hi -= h * m.sx[o + sz] * ((px_hi_md_hi + px_lo_md_hi) - (pz_hi_md_hi + pz_lo_md_hi));
    pz_hi -= h * m.sy[o + sz] * ((py_md_hi_hi + py_md_lo_hi) - (pz_md_hi_hi + pz_md_lo_hi));

    T pz_lo = x000 - x00m;
    pz_lo *= m.hz[o];
    const T px_hi_md_lo = h * (xp00 - x000 + xp0m - x00m) * dxinv;
    const T px_lo_md_lo = h * (x000 - xm00 + x00m - xm0m) * dxinv;
    const T py_md_hi_lo = h * (x0p0 - x000 + x0pm - x00m) * dyinv;
    const T py_md_lo_lo = h * (x000 - x0m0 + x00m - x0mm) * dyinv;
    pz_lo -= h * m.sx[o] * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo));
    pz_lo -= h * m.sy[o] * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));
    if (MASKS) {
        if (k == 0) { pz_lo = T(0); }
        if ((b.zf & TP_XLO) && i == 0) { px_lo = T(0); }
        if ((b.zf & TP_XHI) && i == g.nx - 1) { px_hi = T(0); }
        if ((b.zf & TP_YLO) && j == 0) { py_lo = T(0); }
        if ((b.zf & TP_YHI) && j == g.ny - 1) { py_hi = T(0); }
        if ((b.zf & TP_ZHI) && k == g.nz - 1) { pz_hi = T(0); }
    }
    const T y = (axa[o + 1] * px_hi - axa[o] * px_lo) * dxinv
              + (aya[o + sy] * py_hi - aya[o] * py_lo) * dyinv
              + (aza[o + sz] * pz_hi - aza[o] * pz_lo) * dzinv;
    T v = y / Jc[o];
    if (MASKS && (b.zf & TP_DGROUND) && k == 0) {
        // a Dirichlet ground: the ground-face flux ERF's kernel leaves out (Source/Poisson.cpp:162-189)
        v += aza[o] * ground_flux_dir<T>(g, i, j, X, m.zn) * dzinv / Jc[o];
    }
    return v;
}

//! The operator at (i, j, k) with the neighbours read directly (INTERIOR: all
//! 18 lie in the valid cells) or through ldc's ghost resolution. x is not
//! declared restrict: one kernel may update it between applications.
template <typename T, bool INTERIOR>
__device__ __forceinline__ T adotx_r(const gb_grid& g, const PBC& b, int i, int j, int k, const T* x,
                                     const T* __restrict__ axa, const T* __restrict__ aya, const T* __restrict__ aza,
                                     const T* __restrict__ Jc, const MeshRatios<T>& m)
{
    const int64_t o = at(g, i, j, k);
    auto X = [&](int di, int dj, int dk) { return xoff<T, INTERIOR>(x, g, b, o, i, j, k, di, dj, dk); };
    return adotx_body<T, !INTERIOR>(g, b, i, j, k, o, X, axa, aya, aza, Jc, m);
}

//! One direction's neighbour indices of index i (n cells) and their mirror
//! signs: i - 1, i + 1 wrapped (periodic) or reflected into the cell itself
//! with the face's sign (ldc's resolution for offsets of one).
__device__ __forceinline__ void resolve_neighbours(int i, int n, int periodic, int s_lo, int s_hi, int& im, int& ip,
                                                   int& sm, int& sp)
{
    const bool lo = (i == 0), hi = (i == n - 1);
    im = lo ? (periodic ? n - 1 : 0) : i - 1;
    ip = hi ? (periodic ? 0 : n - 1) : i + 1;
    sm = (lo && !periodic) ? s_lo : 1;
    sp = (hi && !periodic) ? s_hi : 1;
}

//! adotx at any valid cell, one code path for every cell (no divergence
//! between a warp's interior and boundary lanes): each direction's neighbour
//! indices and mirror signs resolved once, a neighbour's value the product of
//! its directions' signs (+-1, exact) times one load at the resolved point,
//! ldc's value (the composition of per-direction reflections and shifts).
template <typename T>
__device__ __forceinline__ T adotx_cell(const gb_grid& g, const PBC& b, int i, int j, int k, const T* x,
                                        const T* __restrict__ axa, const T* __restrict__ aya,
                                        const T* __restrict__ aza, const T* __restrict__ Jc, const MeshRatios<T>& m)
{
    int im, ip, sim, sip, jm, jp, sjm, sjp;
    resolve_neighbours(i, g.nx, b.per_x, b.sxl, b.sxh, im, ip, sim, sip);
    resolve_neighbours(j, g.ny, b.per_y, b.syl, b.syh, jm, jp, sjm, sjp);
    const int km = (k == 0) ? 0 : k - 1, kp = (k == g.nz - 1) ? k : k + 1;
    const int skm = (k == 0) ? b.szl : 1, skp = (k == g.nz - 1) ? b.szh : 1;
    const int sy = static_cast<int>(g.sy), sz = static_cast<int>(g.sz);
    const int ng = g.ng;
    const int cx[3] = {im + ng, i + ng, ip + ng};
    const int cy[3] = {(jm + ng) * sy, (j + ng) * sy, (jp + ng) * sy};
    const int cz[3] = {(km + ng) * sz, (k + ng) * sz, (kp + ng) * sz};
    const int sx3[3] = {sim, 1, sip}, sy3[3] = {sjm, 1, sjp}, sz3[3] = {skm, 1, skp};
    auto X = [&](int di, int dj, int dk) {
        const T v = x[cx[di + 1] + cy[dj + 1] + cz[dk + 1]];
        return (sx3[di + 1] * sy3[dj + 1] * sz3[dk + 1] < 0) ? -v : v;
    };
    const int64_t o = at(g, i, j, k);
    return adotx_body<T, true>(g, b, i, j, k, o, X, axa, aya, aza, Jc, m);
}

//! The principal tridiagonal of the operator on column (i, j) at level k
//! (the multigrid line smoother's T; the oracle's og_line_tridiag).
template <typename T>
__device__ __forceinline__ void line_tridiag(const gb_grid& g, const PBC& b, const T* __restrict__ AX,
                                             const T* __restrict__ AY, const T* __restrict__ AZ,
                                             const T* __restrict__ Jc, const T* __restrict__ zp, int i, int j, int k,
                                             T& D, T& C, T& U)
{
    const T dxinv = static_cast<T>(1.0 / g.dx), dyinv = static_cast<T>(1.0 / g.dy), dzinv = static_cast<T>(1.0 / g.dzeta);
    T c = T(0);
    const T mxl = ((b.zf & TP_XLO) && i == 0) ? T(0) : T(1);
    const T mxh = ((b.zf & TP_XHI) && i == g.nx - 1) ? T(0) : T(1);
    T cxl = dxinv, cxh = dxinv;
    if (!b.per_x && i == 0 && b.sxl < 0) { cxl = T(2) * dxinv; }
    if (!b.per_x && i == g.nx - 1 && b.sxh < 0) { cxh = T(2) * dxinv; }
    c -= (mxh * AX[at(g, i + 1, j, k)] * cxh + mxl * AX[at(g, i, j, k)] * cxl) * dxinv;
    const T myl = ((b.zf & TP_YLO) && j == 0) ? T(0) : T(1);
    const T myh = ((b.zf & TP_YHI) && j == g.ny - 1) ? T(0) : T(1);
    T cyl = dyinv, cyh = dyinv;
    if (!b.per_y && j == 0 && b.syl < 0) { cyl = T(2) * dyinv; }
    if (!b.per_y && j == g.ny - 1 && b.syh < 0) { cyh = T(2) * dyinv; }
    c -= (myh * AY[at(g, i, j + 1, k)] * cyh + myl * AY[at(g, i, j, k)] * cyl) * dyinv;
#define Z(a, bb, cc) zp[at(g, a, bb, cc)]
    const T hzi_hi = T(8) / ((Z(i, j, k + 2) + Z(i + 1, j, k + 2) + Z(i, j + 1, k + 2) + Z(i + 1, j + 1, k + 2))
                             - (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k)));
    const T hzi_lo = T(8) / ((Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1))
                             - (Z(i, j, k - 1) + Z(i + 1, j, k - 1) + Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k - 1)));
#undef Z
    const T mzl = (k != 0) ? T(1) : T(0);
    const T mzh = ((b.zf & TP_ZHI) && k == g.nz - 1) ? T(0) : T(1);
    const T wh = mzh * AZ[at(g, i, j, k + 1)] * hzi_hi * dzinv;
    const T wl = mzl * AZ[at(g, i, j, k)] * hzi_lo * dzinv;
    c -= wh + wl;
    if (k == 0 && (b.zf & TP_DGROUND)) {
        // a Dirichlet ground: the ground face's principal part, one-sided
        const T hzi_g = T(8) / ((zp[at(g, i, j, 1)] + zp[at(g, i + 1, j, 1)] + zp[at(g, i, j + 1, 1)]
                                 + zp[at(g, i + 1, j + 1, 1)])
                                - (zp[at(g, i, j, 0)] + zp[at(g, i + 1, j, 0)] + zp[at(g, i, j + 1, 0)]
                                   + zp[at(g, i + 1, j + 1, 0)]));
        c -= AZ[at(g, i, j, 0)] * hzi_g * dzinv;
    }
    T u = wh, d = wl;
    if (k == g.nz - 1) {
        c += (b.szh < 0 ? T(-1) : T(1)) * u;
        u = T(0);
    }
    if (k == 0) { d = T(0); }
    const T Ji = T(1) / Jc[at(g, i, j, k)];
    D = d * Ji;
    C = c * Ji;
    U = u * Ji;
}

}  // namespace gb
