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
    return b;
}

//! x(i, j, k) of a cell field with its one ghost layer resolved for the BC.
//! `wrap` (may equal x) serves the reads that cross a periodic seam.
template <typename T>
__device__ __forceinline__ T ldc(const T* __restrict__ x, const T* __restrict__ wrap, const gb_grid& g, const PBC& b,
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

//! The terrain operator at cell (i, j, k): ERF_TerrainPoisson_3D_K.H:316-530
//! (terrpoisson_adotx) with the premultiplied areas a beta and the zero-flux mask.
template <typename T>
__device__ __forceinline__ T adotx(const gb_grid& g, const PBC& b, int i, int j, int k, const T* __restrict__ x,
                                   const T* __restrict__ wrap, const T* __restrict__ axa, const T* __restrict__ aya,
                                   const T* __restrict__ aza, const T* __restrict__ Jc, const T* __restrict__ zp)
{
    const T dxinv = static_cast<T>(1.0 / g.dx), dyinv = static_cast<T>(1.0 / g.dy), dzinv = static_cast<T>(1.0 / g.dzeta);
    const T h = T(0.5), q = T(0.25);
#define X(a, bb, c) ldc<T>(x, wrap, g, b, a, bb, c)
#define Z(a, bb, c) zp[at(g, a, bb, c)]
    T h_xi, h_eta, h_zeta;
    T px_hi = (X(i + 1, j, k) - X(i, j, k)) * dxinv;
    T pz_hi_md_hi = h * (X(i + 1, j, k + 1) + X(i, j, k + 1) - X(i + 1, j, k) - X(i, j, k));
    h_xi = q * (Z(i + 2, j, k + 1) - Z(i, j, k + 1) + Z(i + 2, j + 1, k + 1) - Z(i, j + 1, k + 1)) * dxinv;
    h_zeta = q * (Z(i + 1, j, k + 2) - Z(i + 1, j, k) + Z(i + 1, j + 1, k + 2) - Z(i + 1, j + 1, k));
    pz_hi_md_hi *= h_xi / h_zeta;
    T pz_hi_md_lo = h * (X(i + 1, j, k) + X(i, j, k) - X(i + 1, j, k - 1) - X(i, j, k - 1));
    h_xi = q * (Z(i + 2, j, k) - Z(i, j, k) + Z(i + 2, j + 1, k) - Z(i, j + 1, k)) * dxinv;
    h_zeta = q * (Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k - 1));
    pz_hi_md_lo *= h_xi / h_zeta;
    px_hi -= h * (pz_hi_md_hi + pz_hi_md_lo);

    T px_lo = (X(i, j, k) - X(i - 1, j, k)) * dxinv;
    T pz_lo_md_hi = h * (X(i, j, k + 1) + X(i - 1, j, k + 1) - X(i, j, k) - X(i - 1, j, k));
    h_xi = q * (Z(i + 1, j, k + 1) - Z(i - 1, j, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i - 1, j + 1, k + 1)) * dxinv;
    h_zeta = q * (Z(i, j, k + 2) - Z(i, j, k) + Z(i, j + 1, k + 2) - Z(i, j + 1, k));
    pz_lo_md_hi *= h_xi / h_zeta;
    T pz_lo_md_lo = h * (X(i, j, k) + X(i - 1, j, k) - X(i, j, k - 1) - X(i - 1, j, k - 1));
    h_xi = q * (Z(i + 1, j, k) - Z(i - 1, j, k) + Z(i + 1, j + 1, k) - Z(i - 1, j + 1, k)) * dxinv;
    h_zeta = q * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1));
    pz_lo_md_lo *= h_xi / h_zeta;
    px_lo -= h * (pz_lo_md_hi + pz_lo_md_lo);

    T py_hi = (X(i, j + 1, k) - X(i, j, k)) * dyinv;
    T pz_md_hi_hi = h * (X(i, j + 1, k + 1) + X(i, j, k + 1) - X(i, j + 1, k) - X(i, j, k));
    h_eta = q * (Z(i, j + 2, k + 1) - Z(i, j, k + 1) + Z(i + 1, j + 2, k + 1) - Z(i + 1, j, k + 1)) * dyinv;
    h_zeta = q * (Z(i, j + 1, k + 2) - Z(i, j + 1, k) + Z(i + 1, j + 1, k + 2) - Z(i + 1, j + 1, k));
    pz_md_hi_hi *= h_eta / h_zeta;
    T pz_md_hi_lo = h * (X(i, j + 1, k) + X(i, j, k) - X(i, j + 1, k - 1) - X(i, j, k - 1));
    h_eta = q * (Z(i, j + 2, k) - Z(i, j, k) + Z(i + 1, j + 2, k) - Z(i + 1, j, k)) * dyinv;
    h_zeta = q * (Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k - 1));
    pz_md_hi_lo *= h_eta / h_zeta;
    py_hi -= h * (pz_md_hi_hi + pz_md_hi_lo);

    T py_lo = (X(i, j, k) - X(i, j - 1, k)) * dyinv;
    T pz_md_lo_hi = h * (X(i, j, k + 1) + X(i, j - 1, k + 1) - X(i, j, k) - X(i, j - 1, k));
    h_eta = q * (Z(i, j + 1, k + 1) - Z(i, j - 1, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j - 1, k + 1)) * dyinv;
    h_zeta = q * (Z(i, j, k + 2) - Z(i, j, k) + Z(i + 1, j, k + 2) - Z(i + 1, j, k));
    pz_md_lo_hi *= h_eta / h_zeta;
    T pz_md_lo_lo = h * (X(i, j, k) + X(i, j - 1, k) - X(i, j, k - 1) - X(i, j - 1, k - 1));
    h_eta = q * (Z(i, j + 1, k) - Z(i, j - 1, k) + Z(i + 1, j + 1, k) - Z(i + 1, j - 1, k)) * dyinv;
    h_zeta = q * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1));
    pz_md_lo_lo *= h_eta / h_zeta;
    py_lo -= h * (pz_md_lo_hi + pz_md_lo_lo);

    T pz_hi = X(i, j, k + 1) - X(i, j, k);
    const T hzi_hi = T(8) / ((Z(i, j, k + 2) + Z(i + 1, j, k + 2) + Z(i, j + 1, k + 2) + Z(i + 1, j + 1, k + 2))
                             - (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k)));
    pz_hi *= hzi_hi;
    const T px_hi_md_hi = h * (X(i + 1, j, k + 1) - X(i, j, k + 1) + X(i + 1, j, k) - X(i, j, k)) * dxinv;
    const T px_lo_md_hi = h * (X(i, j, k + 1) - X(i - 1, j, k + 1) + X(i, j, k) - X(i - 1, j, k)) * dxinv;
    const T py_md_hi_hi = h * (X(i, j + 1, k + 1) - X(i, j, k + 1) + X(i, j + 1, k) - X(i, j, k)) * dyinv;
    const T py_md_lo_hi = h * (X(i, j, k + 1) - X(i, j - 1, k + 1) + X(i, j, k) - X(i, j - 1, k)) * dyinv;
    const T h_xi_on_zhi = h * (Z(i + 1, j + 1, k + 1) + Z(i + 1, j, k + 1) - Z(i, j + 1, k + 1) - Z(i, j, k + 1)) * dxinv;
    const T h_eta_on_zhi = h * (Z(i + 1, j + 1, k + 1) + Z(i, j + 1, k + 1) - Z(i + 1, j, k + 1) - Z(i, j, k + 1)) * dyinv;
    pz_hi -= h * h_xi_on_zhi * ((px_hi_md_hi + px_lo_md_hi) - (pz_hi_md_hi + pz_lo_md_hi));
    pz_hi -= h * h_eta_on_zhi * ((py_md_hi_hi + py_md_lo_hi) - (pz_md_hi_hi + pz_md_lo_hi));

    T pz_lo = X(i, j, k) - X(i, j, k - 1);
    const T hzi_lo = T(8) / ((Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1))
                             - (Z(i, j, k - 1) + Z(i + 1, j, k - 1) + Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k - 1)));
    pz_lo *= hzi_lo;
    const T px_hi_md_lo = h * (X(i + 1, j, k) - X(i, j, k) + X(i + 1, j, k - 1) - X(i, j, k - 1)) * dxinv;
    const T px_lo_md_lo = h * (X(i, j, k) - X(i - 1, j, k) + X(i, j, k - 1) - X(i - 1, j, k - 1)) * dxinv;
    const T py_md_hi_lo = h * (X(i, j + 1, k) - X(i, j, k) + X(i, j + 1, k - 1) - X(i, j, k - 1)) * dyinv;
    const T py_md_lo_lo = h * (X(i, j, k) - X(i, j - 1, k) + X(i, j, k - 1) - X(i, j - 1, k - 1)) * dyinv;
    const T h_xi_on_zlo = h * (Z(i + 1, j + 1, k) + Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i, j, k)) * dxinv;
    const T h_eta_on_zlo = h * (Z(i + 1, j + 1, k) + Z(i, j + 1, k) - Z(i + 1, j, k) - Z(i, j, k)) * dyinv;
    pz_lo -= h * h_xi_on_zlo * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo));
    pz_lo -= h * h_eta_on_zlo * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));
#undef X
#undef Z
    if (k == 0) { pz_lo = T(0); }
    if ((b.zf & TP_XLO) && i == 0) { px_lo = T(0); }
    if ((b.zf & TP_XHI) && i == g.nx - 1) { px_hi = T(0); }
    if ((b.zf & TP_YLO) && j == 0) { py_lo = T(0); }
    if ((b.zf & TP_YHI) && j == g.ny - 1) { py_hi = T(0); }
    if ((b.zf & TP_ZHI) && k == g.nz - 1) { pz_hi = T(0); }
    const T y = (axa[at(g, i + 1, j, k)] * px_hi - axa[at(g, i, j, k)] * px_lo) * dxinv
              + (aya[at(g, i, j + 1, k)] * py_hi - aya[at(g, i, j, k)] * py_lo) * dyinv
              + (aza[at(g, i, j, k + 1)] * pz_hi - aza[at(g, i, j, k)] * pz_lo) * dzinv;
    return y / Jc[at(g, i, j, k)];
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
