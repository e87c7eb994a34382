/*
 * ORACLE -- test infrastructure, not product code.
 *
 * FP64 restatement of the terrain-following mesh and the pressure-correction
 * Poisson layer of the reference:
 *   - BTF node heights and ghost columns (extern_erf/ERF_TerrainMetrics.cpp:253-420
 *     case 0; Source/Mesh.cpp:49-95 fill_ghost_columns);
 *   - metrics detJ, ax, ay, az, z_cc (extern_erf/ERF_TerrainMetrics.cpp:680-808);
 *   - the 15-point operator terrpoisson_adotx and the face fluxes
 *     (extern_erf/ERF_TerrainPoisson_3D_K.H:22-530), the ghost fills
 *     (Source/Poisson.cpp:84-125 fill_bc_ghosts; extern_erf/ERF_TerrainPoisson.cpp:103-210
 *     apply_bcs), the zero-flux face mask (extern_erf/ERF_TerrainPoisson.cpp:53-66) and
 *     face_divergence (Source/Poisson.cpp:733-764);
 *   - the solve (Source/Poisson.cpp:540-623): J-weighted mean removal for a
 *     singular problem, a Krylov solve to reltol, the true residual, the
 *     coefficient-weighted fluxes.
 * The reference's default back end is AMReX's MLTerrainPoisson multigrid,
 * whose source is not in the reference. The multigrid here is this project's
 * own definition (z-line zebra relaxation, x-y 2:1 coarsening, coarsest-level
 * relaxation), restated identically by the CUDA path; its iterates are parity
 * unpinned against the reference, its solution is pinned through the operator.
 */
#include "og.h"

#include <stdio.h>

enum { PF_PERIODIC = 0, PF_NEUMANN = 1, PF_DIRICHLET = 2 };
enum { FACE_XLO = 0, FACE_YLO = 1, FACE_ZLO = 2, FACE_XHI = 3, FACE_YHI = 4, FACE_ZHI = 5 };
enum { TP_XLO = 1, TP_XHI = 2, TP_YLO = 4, TP_YHI = 8, TP_ZLO = 16, TP_ZHI = 32 };
/* zf bit: a Dirichlet ground (phi = 0 on it: the odd ghost below and the
 * ground-face flux, Source/Poisson.cpp:158-189) */
enum { TP_DGROUND = 64 };

/* ------------------------------------------------------------------ */
/* mesh                                                                */
/* ------------------------------------------------------------------ */

/* BTF node heights (ERF_TerrainMetrics.cpp BTF case: z = ((z_sfc - z_0) z_top
 * + (z_top - z_sfc) z_k) / (z_top - z_0)) from the ground heights of every
 * node column (ground[(j+1)*(nx+3) + (i+1)], i in [-1, nx+1], j in [-1, ny+1],
 * the ghost columns already the periodic image or the clamped edge column),
 * then the rows below the ground and above the top (Source/Mesh.cpp:82-94). */
void og_btf_heights(const og_grid* g, const double* zlev, const double* ground, double* z)
{
    const int nz = g->nz;
    const double ztop = zlev[nz], z0 = zlev[0];
    for (int j = -1; j <= g->ny + 1; ++j) {
        for (int i = -1; i <= g->nx + 1; ++i) {
            const double zs = ground[(int64_t)(j + 1) * (g->nx + 3) + (i + 1)];
            z[IX(g, i, j, 0)] = zs;
            for (int k = 1; k <= nz; ++k) { z[IX(g, i, j, k)] = ((zs - z0) * ztop + (ztop - zs) * zlev[k]) / (ztop - z0); }
            z[IX(g, i, j, -1)] = 2.0 * z[IX(g, i, j, 0)] - z[IX(g, i, j, 1)];
            for (int k = -2; k >= -g->ng; --k) {
                z[IX(g, i, j, k)] = z[IX(g, i, j, 0)] + (0 - k) * (z[IX(g, i, j, 0)] - z[IX(g, i, j, 1)]);
            }
            for (int k = nz + 1; k <= nz + g->ng; ++k) {
                z[IX(g, i, j, k)] = z[IX(g, i, j, nz)] + (k - nz) * (z[IX(g, i, j, nz)] - z[IX(g, i, j, nz - 1)]);
            }
        }
    }
}

/* make_J, make_areas, make_zcc (ERF_TerrainMetrics.cpp:680-808) on the valid
 * points and one ghost layer (J, ax, ay from the ground up; az = 1). */
void og_metrics(const og_grid* g, const double* z, double* J, double* ax, double* ay, double* az, double* zcc)
{
    const double dzi = 1.0 / g->dzeta;
    const int64_t vol = VOL(g);
    memset(J, 0, sizeof(double) * vol);
    memset(ax, 0, sizeof(double) * vol);
    memset(ay, 0, sizeof(double) * vol);
    for (int64_t n = 0; n < vol; ++n) { az[n] = 1.0; }
    memset(zcc, 0, sizeof(double) * vol);
    for (int k = 0; k <= g->nz; ++k) {
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx; ++i) {
                J[IX(g, i, j, k)] = 0.25 * dzi
                    * (z[IX(g, i, j, k + 1)] + z[IX(g, i + 1, j, k + 1)] + z[IX(g, i, j + 1, k + 1)] + z[IX(g, i + 1, j + 1, k + 1)]
                       - z[IX(g, i, j, k)] - z[IX(g, i + 1, j, k)] - z[IX(g, i, j + 1, k)] - z[IX(g, i + 1, j + 1, k)]);
            }
        }
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx + 1; ++i) {
                ax[IX(g, i, j, k)] = 0.5 * dzi * (z[IX(g, i, j, k + 1)] + z[IX(g, i, j + 1, k + 1)] - z[IX(g, i, j, k)] - z[IX(g, i, j + 1, k)]);
            }
        }
        for (int j = -1; j <= g->ny + 1; ++j) {
            for (int i = -1; i <= g->nx; ++i) {
                ay[IX(g, i, j, k)] = 0.5 * dzi * (z[IX(g, i, j, k + 1)] + z[IX(g, i + 1, j, k + 1)] - z[IX(g, i, j, k)] - z[IX(g, i + 1, j, k)]);
            }
        }
    }
    for (int k = -1; k <= g->nz; ++k) {
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx; ++i) {
                zcc[IX(g, i, j, k)] = 0.125 * (z[IX(g, i, j, k)] + z[IX(g, i + 1, j, k)] + z[IX(g, i, j + 1, k)] + z[IX(g, i + 1, j + 1, k)]
                                               + z[IX(g, i, j, k + 1)] + z[IX(g, i + 1, j, k + 1)] + z[IX(g, i, j + 1, k + 1)]
                                               + z[IX(g, i + 1, j + 1, k + 1)]);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* ghost fills and masks                                               */
/* ------------------------------------------------------------------ */

/* fill_bc_ghosts (Source/Poisson.cpp:84-125): periodic images, then even
 * (Neumann) or odd (Dirichlet) copies across the non-periodic faces, x first,
 * then y over the x ghosts, then z over both. ground_even: the ground is an
 * even copy whatever bc says (TerrainPoisson::apply_bcs, ERF_TerrainPoisson.cpp:183-190). */
void og_poisson_fill_ghosts(const og_grid* g, const int* bc, double* phi, int ground_even)
{
    og_fill_periodic(g, 0, phi, 1);
    const int per[3] = {g->periodic_x, g->periodic_y, 0};
    const int n[3] = {g->nx, g->ny, g->nz};
    for (int d = 0; d < 3; ++d) {
        if (per[d]) { continue; }
        for (int side = 0; side < 2; ++side) {
            const int face = d + 3 * side;
            double sign = (bc[face] == PF_DIRICHLET) ? -1.0 : 1.0;
            if (d == 2 && side == 0 && ground_even) { sign = 1.0; }
            int lo[3], hi[3];
            for (int e = 0; e < 3; ++e) {
                lo[e] = 0;
                hi[e] = n[e] - 1;
                if (e == d) { continue; }
                if (e < d || per[e]) { lo[e] = -1; hi[e] = n[e]; }
            }
            const int gidx = side ? n[d] : -1;
            const int sidx = side ? n[d] - 1 : 0;
            lo[d] = hi[d] = gidx;
            for (int k = lo[2]; k <= hi[2]; ++k) {
                for (int j = lo[1]; j <= hi[1]; ++j) {
                    for (int i = lo[0]; i <= hi[0]; ++i) {
                        const int si = (d == 0) ? sidx : i, sj = (d == 1) ? sidx : j, sk = (d == 2) ? sidx : k;
                        phi[IX(g, i, j, k)] = sign * phi[IX(g, si, sj, sk)];
                    }
                }
            }
        }
    }
}

/* The zero-flux faces of the solve region: the Neumann (even) faces of the
 * domain, the ground excepted (ERF_TerrainPoisson.cpp:53-66). */
int og_poisson_zero_flux_faces(const og_grid* g, const int* bc)
{
    int zf = 0;
    if (!g->periodic_x && bc[FACE_XLO] == PF_NEUMANN) { zf |= TP_XLO; }
    if (!g->periodic_x && bc[FACE_XHI] == PF_NEUMANN) { zf |= TP_XHI; }
    if (!g->periodic_y && bc[FACE_YLO] == PF_NEUMANN) { zf |= TP_YLO; }
    if (!g->periodic_y && bc[FACE_YHI] == PF_NEUMANN) { zf |= TP_YHI; }
    if (bc[FACE_ZHI] == PF_NEUMANN) { zf |= TP_ZHI; }
    if (bc[FACE_ZLO] == PF_DIRICHLET) { zf |= TP_DGROUND; }
    return zf;
}

/* The ground's ghost parity of the solve: odd for a Dirichlet ground (fill_bc_ghosts,
 * Source/Poisson.cpp:84-125), else even whatever bc says (TerrainPoisson::apply_bcs). */
static int ground_even(const int* bc) { return bc[FACE_ZLO] != PF_DIRICHLET; }

/* ------------------------------------------------------------------ */
/* the operator                                                        */
/* ------------------------------------------------------------------ */

#define X(a, b, c) x[IX(g, a, b, c)]
#define Z(a, b, c) zp[IX(g, a, b, c)]

/* terrpoisson_flux_zlo_dir (ERF_TerrainPoisson_3D_K.H:214-275): the ground
 * face's flux of column (i, j) with phi = 0 on the ground, one-sided (the
 * ghosts of x filled). */
static double ground_flux_dir(const og_grid* g, int i, int j, const double* x, const double* zp)
{
    const int k = 0;
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy;
    double pz_lo = X(i, j, k);
    const double hzeta_inv_on_zlo = 8.0 / ((Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1))
                                           - (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k)));
    pz_lo *= hzeta_inv_on_zlo;
    const double px_hi_md_lo = 0, px_lo_md_lo = 0, py_md_hi_lo = 0, py_md_lo_lo = 0;
    double h_xi, h_eta, h_zeta;
    double pz_hi_md_lo = 0.5 * (X(i + 1, j, k) + X(i, j, k));
    h_xi = 0.25 * (Z(i + 2, j, k) - Z(i, j, k) + Z(i + 2, j + 1, k) - Z(i, j + 1, k)) * dxinv;
    h_zeta = 0.25 * (Z(i + 1, j, k + 1) - Z(i + 1, j, k) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k));
    pz_hi_md_lo *= h_xi / h_zeta;
    double pz_lo_md_lo = 0.5 * (X(i, j, k) + X(i - 1, j, k));
    h_xi = 0.25 * (Z(i + 1, j, k) - Z(i - 1, j, k) + Z(i + 1, j + 1, k) - Z(i - 1, j + 1, k)) * dxinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k) + Z(i, j + 1, k + 1) - Z(i, j + 1, k));
    pz_lo_md_lo *= h_xi / h_zeta;
    double pz_md_hi_lo = 0.5 * (X(i, j + 1, k) + X(i, j, k));
    h_eta = 0.25 * (Z(i, j + 2, k) - Z(i, j, k) + Z(i + 1, j + 2, k) - Z(i + 1, j, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j + 1, k + 1) - Z(i, j + 1, k) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k));
    pz_md_hi_lo *= h_eta / h_zeta;
    double pz_md_lo_lo = 0.5 * (X(i, j, k) + X(i, j - 1, k));
    h_eta = 0.25 * (Z(i, j + 1, k) - Z(i, j - 1, k) + Z(i + 1, j + 1, k) - Z(i + 1, j - 1, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k) + Z(i + 1, j, k + 1) - Z(i + 1, j, k));
    pz_md_lo_lo *= h_eta / h_zeta;
    const double h_xi_on_zlo = 0.5 * (Z(i + 1, j + 1, k) + Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i, j, k)) * dxinv;
    const double h_eta_on_zlo = 0.5 * (Z(i + 1, j + 1, k) + Z(i, j + 1, k) - Z(i + 1, j, k) - Z(i, j, k)) * dyinv;
    pz_lo -= 0.5 * h_xi_on_zlo * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo));
    pz_lo -= 0.5 * h_eta_on_zlo * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));
    return -pz_lo;
}

/* ERF_TerrainPoisson_3D_K.H:316-530 (terrpoisson_adotx) at cell (i, j, k);
 * with a Dirichlet ground the bottom row adds the ground-face flux
 * (Source/Poisson.cpp:162-189). */
static double adotx_cell(const og_grid* g, int i, int j, int k, const double* x, const double* axa, const double* aya,
                         const double* aza, const double* J, const double* zp, int zf)
{
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy, dzinv = 1.0 / g->dzeta;
    double h_xi, h_eta, h_zeta;
    /* hi x-face */
    double px_hi = (X(i + 1, j, k) - X(i, j, k)) * dxinv;
    double pz_hi_md_hi = 0.5 * (X(i + 1, j, k + 1) + X(i, j, k + 1) - X(i + 1, j, k) - X(i, j, k));
    h_xi = 0.25 * (Z(i + 2, j, k + 1) - Z(i, j, k + 1) + Z(i + 2, j + 1, k + 1) - Z(i, j + 1, k + 1)) * dxinv;
    h_zeta = 0.25 * (Z(i + 1, j, k + 2) - Z(i + 1, j, k) + Z(i + 1, j + 1, k + 2) - Z(i + 1, j + 1, k));
    pz_hi_md_hi *= h_xi / h_zeta;
    double pz_hi_md_lo = 0.5 * (X(i + 1, j, k) + X(i, j, k) - X(i + 1, j, k - 1) - X(i, j, k - 1));
    h_xi = 0.25 * (Z(i + 2, j, k) - Z(i, j, k) + Z(i + 2, j + 1, k) - Z(i, j + 1, k)) * dxinv;
    h_zeta = 0.25 * (Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k - 1));
    pz_hi_md_lo *= h_xi / h_zeta;
    px_hi -= 0.5 * (pz_hi_md_hi + pz_hi_md_lo);
    /* lo x-face */
    double px_lo = (X(i, j, k) - X(i - 1, j, k)) * dxinv;
    double pz_lo_md_hi = 0.5 * (X(i, j, k + 1) + X(i - 1, j, k + 1) - X(i, j, k) - X(i - 1, j, k));
    h_xi = 0.25 * (Z(i + 1, j, k + 1) - Z(i - 1, j, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i - 1, j + 1, k + 1)) * dxinv;
    h_zeta = 0.25 * (Z(i, j, k + 2) - Z(i, j, k) + Z(i, j + 1, k + 2) - Z(i, j + 1, k));
    pz_lo_md_hi *= h_xi / h_zeta;
    double pz_lo_md_lo = 0.5 * (X(i, j, k) + X(i - 1, j, k) - X(i, j, k - 1) - X(i - 1, j, k - 1));
    h_xi = 0.25 * (Z(i + 1, j, k) - Z(i - 1, j, k) + Z(i + 1, j + 1, k) - Z(i - 1, j + 1, k)) * dxinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1));
    pz_lo_md_lo *= h_xi / h_zeta;
    px_lo -= 0.5 * (pz_lo_md_hi + pz_lo_md_lo);
    /* hi y-face */
    double py_hi = (X(i, j + 1, k) - X(i, j, k)) * dyinv;
    double pz_md_hi_hi = 0.5 * (X(i, j + 1, k + 1) + X(i, j, k + 1) - X(i, j + 1, k) - X(i, j, k));
    h_eta = 0.25 * (Z(i, j + 2, k + 1) - Z(i, j, k + 1) + Z(i + 1, j + 2, k + 1) - Z(i + 1, j, k + 1)) * dyinv;
    h_zeta = 0.25 * (Z(i, j + 1, k + 2) - Z(i, j + 1, k) + Z(i + 1, j + 1, k + 2) - Z(i + 1, j + 1, k));
    pz_md_hi_hi *= h_eta / h_zeta;
    double pz_md_hi_lo = 0.5 * (X(i, j + 1, k) + X(i, j, k) - X(i, j + 1, k - 1) - X(i, j, k - 1));
    h_eta = 0.25 * (Z(i, j + 2, k) - Z(i, j, k) + Z(i + 1, j + 2, k) - Z(i + 1, j, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k - 1));
    pz_md_hi_lo *= h_eta / h_zeta;
    py_hi -= 0.5 * (pz_md_hi_hi + pz_md_hi_lo);
    /* lo y-face */
    double py_lo = (X(i, j, k) - X(i, j - 1, k)) * dyinv;
    double pz_md_lo_hi = 0.5 * (X(i, j, k + 1) + X(i, j - 1, k + 1) - X(i, j, k) - X(i, j - 1, k));
    h_eta = 0.25 * (Z(i, j + 1, k + 1) - Z(i, j - 1, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j - 1, k + 1)) * dyinv;
    h_zeta = 0.25 * (Z(i, j, k + 2) - Z(i, j, k) + Z(i + 1, j, k + 2) - Z(i + 1, j, k));
    pz_md_lo_hi *= h_eta / h_zeta;
    double pz_md_lo_lo = 0.5 * (X(i, j, k) + X(i, j - 1, k) - X(i, j, k - 1) - X(i, j - 1, k - 1));
    h_eta = 0.25 * (Z(i, j + 1, k) - Z(i, j - 1, k) + Z(i + 1, j + 1, k) - Z(i + 1, j - 1, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1));
    pz_md_lo_lo *= h_eta / h_zeta;
    py_lo -= 0.5 * (pz_md_lo_hi + pz_md_lo_lo);
    /* hi z-face */
    double pz_hi = X(i, j, k + 1) - X(i, j, k);
    const double hzi_hi = 8.0 / ((Z(i, j, k + 2) + Z(i + 1, j, k + 2) + Z(i, j + 1, k + 2) + Z(i + 1, j + 1, k + 2))
                                - (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k)));
    pz_hi *= hzi_hi;
    const double px_hi_md_hi = 0.5 * (X(i + 1, j, k + 1) - X(i, j, k + 1) + X(i + 1, j, k) - X(i, j, k)) * dxinv;
    const double px_lo_md_hi = 0.5 * (X(i, j, k + 1) - X(i - 1, j, k + 1) + X(i, j, k) - X(i - 1, j, k)) * dxinv;
    const double py_md_hi_hi = 0.5 * (X(i, j + 1, k + 1) - X(i, j, k + 1) + X(i, j + 1, k) - X(i, j, k)) * dyinv;
    const double py_md_lo_hi = 0.5 * (X(i, j, k + 1) - X(i, j - 1, k + 1) + X(i, j, k) - X(i, j - 1, k)) * dyinv;
    const double h_xi_on_zhi = 0.5 * (Z(i + 1, j + 1, k + 1) + Z(i + 1, j, k + 1) - Z(i, j + 1, k + 1) - Z(i, j, k + 1)) * dxinv;
    const double h_eta_on_zhi = 0.5 * (Z(i + 1, j + 1, k + 1) + Z(i, j + 1, k + 1) - Z(i + 1, j, k + 1) - Z(i, j, k + 1)) * dyinv;
    pz_hi -= 0.5 * h_xi_on_zhi * ((px_hi_md_hi + px_lo_md_hi) - (pz_hi_md_hi + pz_lo_md_hi));
    pz_hi -= 0.5 * h_eta_on_zhi * ((py_md_hi_hi + py_md_lo_hi) - (pz_md_hi_hi + pz_md_lo_hi));
    /* lo z-face */
    double pz_lo = X(i, j, k) - X(i, j, k - 1);
    const double hzi_lo = 8.0 / ((Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1))
                                - (Z(i, j, k - 1) + Z(i + 1, j, k - 1) + Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k - 1)));
    pz_lo *= hzi_lo;
    const double px_hi_md_lo = 0.5 * (X(i + 1, j, k) - X(i, j, k) + X(i + 1, j, k - 1) - X(i, j, k - 1)) * dxinv;
    const double px_lo_md_lo = 0.5 * (X(i, j, k) - X(i - 1, j, k) + X(i, j, k - 1) - X(i - 1, j, k - 1)) * dxinv;
    const double py_md_hi_lo = 0.5 * (X(i, j + 1, k) - X(i, j, k) + X(i, j + 1, k - 1) - X(i, j, k - 1)) * dyinv;
    const double py_md_lo_lo = 0.5 * (X(i, j, k) - X(i, j - 1, k) + X(i, j, k - 1) - X(i, j - 1, k - 1)) * dyinv;
    const double h_xi_on_zlo = 0.5 * (Z(i + 1, j + 1, k) + Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i, j, k)) * dxinv;
    const double h_eta_on_zlo = 0.5 * (Z(i + 1, j + 1, k) + Z(i, j + 1, k) - Z(i + 1, j, k) - Z(i, j, k)) * dyinv;
    pz_lo -= 0.5 * h_xi_on_zlo * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo));
    pz_lo -= 0.5 * h_eta_on_zlo * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));

    if (k == 0) { pz_lo = 0; }
    if ((zf & TP_XLO) && i == 0) { px_lo = 0; }
    if ((zf & TP_XHI) && i == g->nx - 1) { px_hi = 0; }
    if ((zf & TP_YLO) && j == 0) { py_lo = 0; }
    if ((zf & TP_YHI) && j == g->ny - 1) { py_hi = 0; }
    if ((zf & TP_ZLO) && k == 0) { pz_lo = 0; }
    if ((zf & TP_ZHI) && k == g->nz - 1) { pz_hi = 0; }
    double y = (axa[IX(g, i + 1, j, k)] * px_hi - axa[IX(g, i, j, k)] * px_lo) * dxinv
             + (aya[IX(g, i, j + 1, k)] * py_hi - aya[IX(g, i, j, k)] * py_lo) * dyinv
             + (aza[IX(g, i, j, k + 1)] * pz_hi - aza[IX(g, i, j, k)] * pz_lo) * dzinv;
    double v = y / J[IX(g, i, j, k)];
    if ((zf & TP_DGROUND) && k == 0) { v += aza[IX(g, i, j, k)] * ground_flux_dir(g, i, j, x, zp) * dzinv / J[IX(g, i, j, k)]; }
    return v;
}

/* x-, y- and z-face fluxes (ERF_TerrainPoisson_3D_K.H:22-223: -grad phi on the
 * face with the terrain cross terms). */
static double flux_x(const og_grid* g, int i, int j, int k, const double* x, const double* zp)
{
    const double dxinv = 1.0 / g->dx;
    double px_lo = (X(i, j, k) - X(i - 1, j, k)) * dxinv;
    double pz_lo_md_hi = 0.5 * (X(i, j, k + 1) + X(i - 1, j, k + 1) - X(i, j, k) - X(i - 1, j, k));
    double h_xi = 0.25 * (Z(i + 1, j, k + 1) - Z(i - 1, j, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i - 1, j + 1, k + 1)) * dxinv;
    double h_zeta = 0.25 * (Z(i, j, k + 2) - Z(i, j, k) + Z(i, j + 1, k + 2) - Z(i, j + 1, k));
    pz_lo_md_hi *= h_xi / h_zeta;
    double pz_lo_md_lo = 0.5 * (X(i, j, k) + X(i - 1, j, k) - X(i, j, k - 1) - X(i - 1, j, k - 1));
    h_xi = 0.25 * (Z(i + 1, j, k) - Z(i - 1, j, k) + Z(i + 1, j + 1, k) - Z(i - 1, j + 1, k)) * dxinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1));
    pz_lo_md_lo *= h_xi / h_zeta;
    px_lo -= 0.5 * (pz_lo_md_hi + pz_lo_md_lo);
    return -px_lo;
}

static double flux_y(const og_grid* g, int i, int j, int k, const double* x, const double* zp)
{
    const double dyinv = 1.0 / g->dy;
    double py_lo = (X(i, j, k) - X(i, j - 1, k)) * dyinv;
    double pz_md_lo_hi = 0.5 * (X(i, j, k + 1) + X(i, j - 1, k + 1) - X(i, j, k) - X(i, j - 1, k));
    double h_eta = 0.25 * (Z(i, j + 1, k + 1) - Z(i, j - 1, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j - 1, k + 1)) * dyinv;
    double h_zeta = 0.25 * (Z(i, j, k + 2) - Z(i, j, k) + Z(i + 1, j, k + 2) - Z(i + 1, j, k));
    pz_md_lo_hi *= h_eta / h_zeta;
    double pz_md_lo_lo = 0.5 * (X(i, j, k) + X(i, j - 1, k) - X(i, j, k - 1) - X(i, j - 1, k - 1));
    h_eta = 0.25 * (Z(i, j + 1, k) - Z(i, j - 1, k) + Z(i + 1, j + 1, k) - Z(i + 1, j - 1, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1));
    pz_md_lo_lo *= h_eta / h_zeta;
    py_lo -= 0.5 * (pz_md_lo_hi + pz_md_lo_lo);
    return -py_lo;
}

static double flux_z(const og_grid* g, int i, int j, int k, const double* x, const double* zp)
{
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy;
    double h_xi, h_eta, h_zeta;
    double pz_lo = X(i, j, k) - X(i, j, k - 1);
    const double hzi = 8.0 / ((Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1))
                             - (Z(i, j, k - 1) + Z(i + 1, j, k - 1) + Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k - 1)));
    pz_lo *= hzi;
    const double px_hi_md_lo = 0.5 * (X(i + 1, j, k) - X(i, j, k) + X(i + 1, j, k - 1) - X(i, j, k - 1)) * dxinv;
    const double px_lo_md_lo = 0.5 * (X(i, j, k) - X(i - 1, j, k) + X(i, j, k - 1) - X(i - 1, j, k - 1)) * dxinv;
    const double py_md_hi_lo = 0.5 * (X(i, j + 1, k) - X(i, j, k) + X(i, j + 1, k - 1) - X(i, j, k - 1)) * dyinv;
    const double py_md_lo_lo = 0.5 * (X(i, j, k) - X(i, j - 1, k) + X(i, j, k - 1) - X(i, j - 1, k - 1)) * dyinv;
    double pz_hi_md_lo = 0.5 * (X(i + 1, j, k) + X(i, j, k) - X(i + 1, j, k - 1) - X(i, j, k - 1));
    h_xi = 0.25 * (Z(i + 2, j, k) - Z(i, j, k) + Z(i + 2, j + 1, k) - Z(i, j + 1, k)) * dxinv;
    h_zeta = 0.25 * (Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k - 1));
    pz_hi_md_lo *= h_xi / h_zeta;
    double pz_lo_md_lo = 0.5 * (X(i, j, k) + X(i - 1, j, k) - X(i, j, k - 1) - X(i - 1, j, k - 1));
    h_xi = 0.25 * (Z(i + 1, j, k) - Z(i - 1, j, k) + Z(i + 1, j + 1, k) - Z(i - 1, j + 1, k)) * dxinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1));
    pz_lo_md_lo *= h_xi / h_zeta;
    double pz_md_hi_lo = 0.5 * (X(i, j + 1, k) + X(i, j, k) - X(i, j + 1, k - 1) - X(i, j, k - 1));
    h_eta = 0.25 * (Z(i, j + 2, k) - Z(i, j, k) + Z(i + 1, j + 2, k) - Z(i + 1, j, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k - 1));
    pz_md_hi_lo *= h_eta / h_zeta;
    double pz_md_lo_lo = 0.5 * (X(i, j, k) + X(i, j - 1, k) - X(i, j, k - 1) - X(i, j - 1, k - 1));
    h_eta = 0.25 * (Z(i, j + 1, k) - Z(i, j - 1, k) + Z(i + 1, j + 1, k) - Z(i + 1, j - 1, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1));
    pz_md_lo_lo *= h_eta / h_zeta;
    const double h_xi_on_zlo = 0.5 * (Z(i + 1, j + 1, k) + Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i, j, k)) * dxinv;
    const double h_eta_on_zlo = 0.5 * (Z(i + 1, j + 1, k) + Z(i, j + 1, k) - Z(i + 1, j, k) - Z(i, j, k)) * dyinv;
    pz_lo -= 0.5 * h_xi_on_zlo * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo));
    pz_lo -= 0.5 * h_eta_on_zlo * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));
    if (k == 0) { pz_lo = 0; }
    return -pz_lo;
}

/* z_face_cross (Source/PoissonCross_K.H:16-58): the terrain cross part
 * h_x dphi/dx + h_y dphi/dy of the z-face gradient at the low z-face of cell
 * (i, j, k), in the reference's operation order. phi's ghosts filled. */
static double z_face_cross(const og_grid* g, int i, int j, int k, const double* x, const double* zp)
{
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy;
    const double px_hi_md_lo = 0.5 * (X(i + 1, j, k) - X(i, j, k) + X(i + 1, j, k - 1) - X(i, j, k - 1)) * dxinv;
    const double px_lo_md_lo = 0.5 * (X(i, j, k) - X(i - 1, j, k) + X(i, j, k - 1) - X(i - 1, j, k - 1)) * dxinv;
    const double py_md_hi_lo = 0.5 * (X(i, j + 1, k) - X(i, j, k) + X(i, j + 1, k - 1) - X(i, j, k - 1)) * dyinv;
    const double py_md_lo_lo = 0.5 * (X(i, j, k) - X(i, j - 1, k) + X(i, j, k - 1) - X(i, j - 1, k - 1)) * dyinv;
    double pz_hi_md_lo = 0.5 * (X(i + 1, j, k) + X(i, j, k) - X(i + 1, j, k - 1) - X(i, j, k - 1));
    double h_xi = 0.25 * (Z(i + 2, j, k) - Z(i, j, k) + Z(i + 2, j + 1, k) - Z(i, j + 1, k)) * dxinv;
    double h_zeta = 0.25 * (Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k - 1));
    pz_hi_md_lo *= h_xi / h_zeta;
    double pz_lo_md_lo = 0.5 * (X(i, j, k) + X(i - 1, j, k) - X(i, j, k - 1) - X(i - 1, j, k - 1));
    h_xi = 0.25 * (Z(i + 1, j, k) - Z(i - 1, j, k) + Z(i + 1, j + 1, k) - Z(i - 1, j + 1, k)) * dxinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1));
    pz_lo_md_lo *= h_xi / h_zeta;
    double pz_md_hi_lo = 0.5 * (X(i, j + 1, k) + X(i, j, k) - X(i, j + 1, k - 1) - X(i, j, k - 1));
    double h_eta = 0.25 * (Z(i, j + 2, k) - Z(i, j, k) + Z(i + 1, j + 2, k) - Z(i + 1, j, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j + 1, k + 1) - Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k - 1));
    pz_md_hi_lo *= h_eta / h_zeta;
    double pz_md_lo_lo = 0.5 * (X(i, j, k) + X(i, j - 1, k) - X(i, j, k - 1) - X(i, j - 1, k - 1));
    h_eta = 0.25 * (Z(i, j + 1, k) - Z(i, j - 1, k) + Z(i + 1, j + 1, k) - Z(i + 1, j - 1, k)) * dyinv;
    h_zeta = 0.25 * (Z(i, j, k + 1) - Z(i, j, k - 1) + Z(i + 1, j, k + 1) - Z(i + 1, j, k - 1));
    pz_md_lo_lo *= h_eta / h_zeta;
    const double h_xi_on_zlo = 0.5 * (Z(i + 1, j + 1, k) + Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i, j, k)) * dxinv;
    const double h_eta_on_zlo = 0.5 * (Z(i + 1, j + 1, k) + Z(i, j + 1, k) - Z(i + 1, j, k) - Z(i, j, k)) * dyinv;
    return 0.5 * h_xi_on_zlo * ((px_hi_md_lo + px_lo_md_lo) - (pz_hi_md_lo + pz_lo_md_lo))
         + 0.5 * h_eta_on_zlo * ((py_md_hi_lo + py_md_lo_lo) - (pz_md_hi_lo + pz_md_lo_lo));
}

#undef X
#undef Z

/* The z-faces whose flux the split correction touches: not the ground, not a
 * Neumann top (Source/Poisson.cpp:233-235, 246-249). */
static int cross_face(const og_grid* g, const int* bc, int kf)
{
    return kf != 0 && !(kf == g->nz && bc[FACE_ZHI] == PF_NEUMANN);
}

/* PoissonSolver::Op::add_cross (Source/Poisson.cpp:229-253):
 * y += (1/J) d_zeta (a_z d cross) with d = beta_z - z_cross per z-face.
 * phi's ghosts filled for the boundary types. */
void og_poisson_add_cross(const og_grid* g, const int* bc, const double* az, const double* d, const double* J,
                          const double* z, const double* phi, double* y)
{
    const double dzinv = 1.0 / g->dzeta;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                double hi = 0, lo = 0;
                if (cross_face(g, bc, k + 1)) {
                    hi = az[IX(g, i, j, k + 1)] * d[IX(g, i, j, k + 1)] * z_face_cross(g, i, j, k + 1, phi, z);
                }
                if (cross_face(g, bc, k)) {
                    lo = az[IX(g, i, j, k)] * d[IX(g, i, j, k)] * z_face_cross(g, i, j, k, phi, z);
                }
                y[IX(g, i, j, k)] += (hi - lo) * dzinv / J[IX(g, i, j, k)];
            }
        }
    }
}

/* PoissonSolver::Op::add_cross_flux (Source/Poisson.cpp:255-273):
 * F_z -= d cross on the same faces. phi's ghosts filled. */
void og_poisson_cross_flux(const og_grid* g, const int* bc, const double* d, const double* z, const double* phi,
                           double* fz)
{
    for (int k = 0; k <= g->nz; ++k) {
        if (!cross_face(g, bc, k)) { continue; }
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                fz[IX(g, i, j, k)] -= d[IX(g, i, j, k)] * z_face_cross(g, i, j, k, phi, z);
            }
        }
    }
}

/* TerrainPoisson::apply (ERF_TerrainPoisson.cpp:74-101): ghosts for the BC
 * (ground even), then the operator with the premultiplied areas a beta. */
void og_poisson_apply(const og_grid* g, const int* bc, const double* AX, const double* AY, const double* AZ,
                      const double* J, const double* z, double* phi, double* y)
{
    og_poisson_fill_ghosts(g, bc, phi, ground_even(bc));
    const int zf = og_poisson_zero_flux_faces(g, bc);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) { y[IX(g, i, j, k)] = adotx_cell(g, i, j, k, phi, AX, AY, AZ, J, z, zf); }
        }
    }
}

/* TerrainPoisson::getFluxes (ERF_TerrainPoisson.cpp:212-264) times the face
 * coefficients (Source/Poisson.cpp:603-615; null = 1). phi's ghosts filled. */
void og_poisson_fluxes(const og_grid* g, const int* bc, const double* z, double* phi, const double* bx,
                       const double* by, const double* bz, double* fx, double* fy, double* fz)
{
    og_poisson_fill_ghosts(g, bc, phi, ground_even(bc));
    const int zf = og_poisson_zero_flux_faces(g, bc);
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i <= g->nx; ++i) {
                double f = flux_x(g, i, j, k, phi, z);
                if (((zf & TP_XLO) && i == 0) || ((zf & TP_XHI) && i == g->nx)) { f = 0; }
                fx[IX(g, i, j, k)] = bx ? f * bx[IX(g, i, j, k)] : f;
            }
        }
        for (int j = 0; j <= g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                double f = flux_y(g, i, j, k, phi, z);
                if (((zf & TP_YLO) && j == 0) || ((zf & TP_YHI) && j == g->ny)) { f = 0; }
                fy[IX(g, i, j, k)] = by ? f * by[IX(g, i, j, k)] : f;
            }
        }
    }
    for (int k = 0; k <= g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                double f = flux_z(g, i, j, k, phi, z);
                if (((zf & TP_ZLO) && k == 0) || ((zf & TP_ZHI) && k == g->nz)) { f = 0; }
                fz[IX(g, i, j, k)] = bz ? f * bz[IX(g, i, j, k)] : f;
            }
        }
    }
}

/* face_divergence (Source/Poisson.cpp:733-764). */
void og_face_divergence(const og_grid* g, const double* ax, const double* ay, const double* az, const double* J,
                        const double* fx, const double* fy, const double* fz, double* div)
{
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy, dzinv = 1.0 / g->dzeta;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                div[IX(g, i, j, k)] = ((ax[IX(g, i + 1, j, k)] * fx[IX(g, i + 1, j, k)] - ax[IX(g, i, j, k)] * fx[IX(g, i, j, k)]) * dxinv
                                       + (ay[IX(g, i, j + 1, k)] * fy[IX(g, i, j + 1, k)] - ay[IX(g, i, j, k)] * fy[IX(g, i, j, k)]) * dyinv
                                       + (az[IX(g, i, j, k + 1)] * fz[IX(g, i, j, k + 1)] - az[IX(g, i, j, k)] * fz[IX(g, i, j, k)]) * dzinv)
                                      / J[IX(g, i, j, k)];
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* multigrid (this project's definition)                               */
/* ------------------------------------------------------------------ */

#define OG_MAX_LEVELS 12

typedef struct og_level {
    og_grid g;
    double *z, *J, *AX, *AY, *AZ;  /* node heights, Jacobian, premultiplied areas a beta */
    double *x, *b, *r;             /* solution, right-hand side, residual */
} og_level;

typedef struct og_mg {
    int nlev;
    og_level lev[OG_MAX_LEVELS];
    int bc[6];
    int nu1, nu2, nu_coarse;
    /* the split z-face correction of the Krylov operator (null: none): the raw
     * z areas and d = beta_z - z_cross per z-face; the V-cycle never sees it */
    double *cross_az, *cross_d;
} og_mg;

/* The coarse grid of a level: x and y halved, z kept. */
static og_grid coarse_grid(const og_grid* f)
{
    og_grid c = *f;
    c.nx = f->nx / 2;
    c.ny = f->ny / 2;
    c.dx = 2.0 * f->dx;
    c.dy = 2.0 * f->dy;
    c.sy = c.nx + 1 + 2 * c.ng;
    c.sz = c.sy * (c.ny + 1 + 2 * c.ng);
    return c;
}

/* The fine node column under coarse node column I (with the ghost columns'
 * periodic image or clamped edge, as the fine mesh builds them). */
static int coarse_node_src(int I, int nc, int per)
{
    if (I < 0 || I > nc) {
        if (per) { I = (I < 0) ? I + nc : I - nc; }
        else { I = (I < 0) ? 0 : nc; }
    }
    return 2 * I;
}

int og_mg_can_coarsen(const og_grid* g, int min_coarse)
{
    return (g->nx % 2 == 0) && (g->ny % 2 == 0) && (g->nx / 2 >= min_coarse) && (g->ny / 2 >= min_coarse);
}

/* Build the hierarchy: level 0 is the fine problem (the premultiplied areas and
 * J given); coarse node heights by injection, J from them, the coarse
 * premultiplied areas the means of the fine ones a coarse face covers. */
og_mg* og_mg_create(const og_grid* g, const int* bc, const double* z, const double* J, const double* AX,
                    const double* AY, const double* AZ, int max_levels, int min_coarse, int nu1, int nu2, int nu_coarse)
{
    og_mg* mg = (og_mg*)calloc(1, sizeof(og_mg));
    memcpy(mg->bc, bc, sizeof(int) * 6);
    mg->nu1 = nu1;
    mg->nu2 = nu2;
    mg->nu_coarse = nu_coarse;
    if (max_levels > OG_MAX_LEVELS) { max_levels = OG_MAX_LEVELS; }
    og_grid cur = *g;
    int n = 0;
    for (;;) {
        og_level* L = &mg->lev[n];
        L->g = cur;
        const int64_t vol = VOL(&cur);
        L->z = (double*)calloc(vol, sizeof(double));
        L->J = (double*)calloc(vol, sizeof(double));
        L->AX = (double*)calloc(vol, sizeof(double));
        L->AY = (double*)calloc(vol, sizeof(double));
        L->AZ = (double*)calloc(vol, sizeof(double));
        L->x = (double*)calloc(vol, sizeof(double));
        L->b = (double*)calloc(vol, sizeof(double));
        L->r = (double*)calloc(vol, sizeof(double));
        if (n == 0) {
            memcpy(L->z, z, sizeof(double) * vol);
            memcpy(L->J, J, sizeof(double) * vol);
            memcpy(L->AX, AX, sizeof(double) * vol);
            memcpy(L->AY, AY, sizeof(double) * vol);
            memcpy(L->AZ, AZ, sizeof(double) * vol);
        } else {
            const og_level* F = &mg->lev[n - 1];
            const og_grid* fg = &F->g;
            for (int k = -1; k <= cur.nz + 1; ++k) {
                for (int J2 = -1; J2 <= cur.ny + 1; ++J2) {
                    for (int I = -1; I <= cur.nx + 1; ++I) {
                        const int fi = coarse_node_src(I, cur.nx, cur.periodic_x);
                        const int fj = coarse_node_src(J2, cur.ny, cur.periodic_y);
                        L->z[IX(&cur, I, J2, k)] = F->z[IX(fg, fi, fj, k)];
                    }
                }
            }
            double* ax = (double*)calloc(vol, sizeof(double));
            double* ay = (double*)calloc(vol, sizeof(double));
            double* az = (double*)calloc(vol, sizeof(double));
            double* zcc = (double*)calloc(vol, sizeof(double));
            og_metrics(&cur, L->z, L->J, ax, ay, az, zcc);
            free(ax);
            free(ay);
            free(az);
            free(zcc);
            for (int k = 0; k < cur.nz; ++k) {
                for (int J2 = 0; J2 < cur.ny; ++J2) {
                    for (int I = 0; I <= cur.nx; ++I) {
                        L->AX[IX(&cur, I, J2, k)] = 0.5 * (F->AX[IX(fg, 2 * I, 2 * J2, k)] + F->AX[IX(fg, 2 * I, 2 * J2 + 1, k)]);
                    }
                }
                for (int J2 = 0; J2 <= cur.ny; ++J2) {
                    for (int I = 0; I < cur.nx; ++I) {
                        L->AY[IX(&cur, I, J2, k)] = 0.5 * (F->AY[IX(fg, 2 * I, 2 * J2, k)] + F->AY[IX(fg, 2 * I + 1, 2 * J2, k)]);
                    }
                }
            }
            for (int k = 0; k <= cur.nz; ++k) {
                for (int J2 = 0; J2 < cur.ny; ++J2) {
                    for (int I = 0; I < cur.nx; ++I) {
                        L->AZ[IX(&cur, I, J2, k)] = 0.25 * (F->AZ[IX(fg, 2 * I, 2 * J2, k)] + F->AZ[IX(fg, 2 * I + 1, 2 * J2, k)]
                                                            + F->AZ[IX(fg, 2 * I, 2 * J2 + 1, k)] + F->AZ[IX(fg, 2 * I + 1, 2 * J2 + 1, k)]);
                    }
                }
            }
        }
        ++n;
        if (n >= max_levels || !og_mg_can_coarsen(&cur, min_coarse)) { break; }
        cur = coarse_grid(&cur);
    }
    mg->nlev = n;
    return mg;
}

void og_mg_destroy(og_mg* mg)
{
    if (!mg) { return; }
    for (int n = 0; n < mg->nlev; ++n) {
        og_level* L = &mg->lev[n];
        free(L->z);
        free(L->J);
        free(L->AX);
        free(L->AY);
        free(L->AZ);
        free(L->x);
        free(L->b);
        free(L->r);
    }
    free(mg->cross_az);
    free(mg->cross_d);
    free(mg);
}

/* FaceCoeffs::z_cross (Source/Poisson.cpp:461-479): d = (beta_z or 1) -
 * z_cross on the z-faces, used by the solver's operator and fluxes; z_cross
 * null removes it. */
void og_mg_set_cross(og_mg* mg, const double* az, const double* bz, const double* z_cross)
{
    free(mg->cross_az);
    free(mg->cross_d);
    mg->cross_az = mg->cross_d = NULL;
    if (!z_cross) { return; }
    const int64_t vol = VOL(&mg->lev[0].g);
    mg->cross_az = (double*)malloc(sizeof(double) * (size_t)vol);
    mg->cross_d = (double*)malloc(sizeof(double) * (size_t)vol);
    memcpy(mg->cross_az, az, sizeof(double) * (size_t)vol);
    for (int64_t n = 0; n < vol; ++n) { mg->cross_d[n] = (bz ? bz[n] : 1.0) - z_cross[n]; }
}

/* PoissonSolver::Op::apply (Source/Poisson.cpp:148-156): the terrain operator
 * plus the split correction when set. */
static void mg_apply(og_mg* mg, double* phi, double* y)
{
    og_level* L = &mg->lev[0];
    og_poisson_apply(&L->g, mg->bc, L->AX, L->AY, L->AZ, L->J, L->z, phi, y);
    if (mg->cross_d) { og_poisson_add_cross(&L->g, mg->bc, mg->cross_az, mg->cross_d, L->J, L->z, phi, y); }
}

void og_mg_apply(og_mg* mg, double* phi, double* y) { mg_apply(mg, phi, y); }

int og_mg_levels(const og_mg* mg) { return mg->nlev; }
void og_mg_level_dims(const og_mg* mg, int l, int* nx, int* ny, int* nz)
{
    *nx = mg->lev[l].g.nx;
    *ny = mg->lev[l].g.ny;
    *nz = mg->lev[l].g.nz;
}
double* og_mg_level_array(og_mg* mg, int l, int which)
{
    og_level* L = &mg->lev[l];
    switch (which) {
    case 0: return L->z;
    case 1: return L->J;
    case 2: return L->AX;
    case 3: return L->AY;
    case 4: return L->AZ;
    case 5: return L->x;
    case 6: return L->b;
    default: return L->r;
    }
}

/* The principal tridiagonal of the operator on column (i, j): the orthogonal
 * parts of the six face fluxes (the normal differences with the z-face metric
 * 8/(sum of the face's four node heights above minus below)), with the
 * zero-flux faces dropped, the ground and top ghosts folded by their mirror
 * sign, and the normal difference across a Dirichlet side face folded (odd
 * ghost). The cross-metric terms stay on the residual side. */
void og_line_tridiag(const og_grid* g, const int* bc, int zf, const double* AX, const double* AY, const double* AZ,
                     const double* J, const double* zp, int i, int j, int k, double* Dk, double* Ck, double* Uk)
{
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy, dzinv = 1.0 / g->dzeta;
    double C = 0, D = 0, U = 0;
    /* x faces */
    const int mxl = !((zf & TP_XLO) && i == 0), mxh = !((zf & TP_XHI) && i == g->nx - 1);
    double cxl = dxinv, cxh = dxinv;
    if (!g->periodic_x && i == 0 && bc[FACE_XLO] == PF_DIRICHLET) { cxl = 2.0 * dxinv; }
    if (!g->periodic_x && i == g->nx - 1 && bc[FACE_XHI] == PF_DIRICHLET) { cxh = 2.0 * dxinv; }
    C -= (mxh * AX[IX(g, i + 1, j, k)] * cxh + mxl * AX[IX(g, i, j, k)] * cxl) * dxinv;
    /* y faces */
    const int myl = !((zf & TP_YLO) && j == 0), myh = !((zf & TP_YHI) && j == g->ny - 1);
    double cyl = dyinv, cyh = dyinv;
    if (!g->periodic_y && j == 0 && bc[FACE_YLO] == PF_DIRICHLET) { cyl = 2.0 * dyinv; }
    if (!g->periodic_y && j == g->ny - 1 && bc[FACE_YHI] == PF_DIRICHLET) { cyh = 2.0 * dyinv; }
    C -= (myh * AY[IX(g, i, j + 1, k)] * cyh + myl * AY[IX(g, i, j, k)] * cyl) * dyinv;
    /* z faces */
#define Z(a, b, c) zp[IX(g, a, b, c)]
    const double hzi_hi = 8.0 / ((Z(i, j, k + 2) + Z(i + 1, j, k + 2) + Z(i, j + 1, k + 2) + Z(i + 1, j + 1, k + 2))
                                - (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k)));
    const double hzi_lo = 8.0 / ((Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1))
                                - (Z(i, j, k - 1) + Z(i + 1, j, k - 1) + Z(i, j + 1, k - 1) + Z(i + 1, j + 1, k - 1)));
#undef Z
    const int mzl = (k != 0), mzh = !((zf & TP_ZHI) && k == g->nz - 1);
    const double wh = mzh * AZ[IX(g, i, j, k + 1)] * hzi_hi * dzinv;
    const double wl = mzl * AZ[IX(g, i, j, k)] * hzi_lo * dzinv;
    C -= wh + wl;
    if (k == 0 && (zf & TP_DGROUND)) {
        /* the ground face's principal part (phi = 0 on it): one-sided */
        const double hzi_g = 8.0 / ((zp[IX(g, i, j, 1)] + zp[IX(g, i + 1, j, 1)] + zp[IX(g, i, j + 1, 1)]
                                     + zp[IX(g, i + 1, j + 1, 1)])
                                    - (zp[IX(g, i, j, 0)] + zp[IX(g, i + 1, j, 0)] + zp[IX(g, i, j + 1, 0)]
                                       + zp[IX(g, i + 1, j + 1, 0)]));
        C -= AZ[IX(g, i, j, 0)] * hzi_g * dzinv;
    }
    U = wh;
    D = wl;
    if (k == g->nz - 1) {
        const double s = (bc[FACE_ZHI] == PF_DIRICHLET) ? -1.0 : 1.0;
        C += s * U;
        U = 0;
    }
    if (k == 0) { D = 0; }
    const double Ji = 1.0 / J[IX(g, i, j, k)];
    *Dk = D * Ji;
    *Ck = C * Ji;
    *Uk = U * Ji;
}

/* One zebra z-line relaxation on level L: for colour 0 then 1 ((i + j) even,
 * then odd), the ghosts of x for the BC, then on every column of the colour
 * the residual b - A x (the full operator at the current x), the principal
 * tridiagonal T, and x += T^{-1} (b - A x) by the Thomas recurrences. */
static void mg_smooth(og_mg* mg, og_level* L)
{
    const og_grid* g = &L->g;
    const int zf = og_poisson_zero_flux_faces(g, mg->bc);
    const int nz = g->nz;
    for (int color = 0; color < 2; ++color) {
        og_poisson_fill_ghosts(g, mg->bc, L->x, ground_even(mg->bc));
#pragma omp parallel for collapse(2) schedule(static)
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                if (((i + j) & 1) != color) { continue; }
                double r[1024], c[1024], e[1024];
                for (int k = 0; k < nz; ++k) {
                    r[k] = L->b[IX(g, i, j, k)] - adotx_cell(g, i, j, k, L->x, L->AX, L->AY, L->AZ, L->J, L->z, zf);
                }
                /* Factored Thomas: reciprocal pivots 1/m_k and eliminated uppers
                 * c'_k = U_k (1/m_k), then e_k = (r_k - D_k e_{k-1}) (1/m_k). */
                double cp = 0, ep = 0;
                for (int k = 0; k < nz; ++k) {
                    double D, C, U;
                    og_line_tridiag(g, mg->bc, zf, L->AX, L->AY, L->AZ, L->J, L->z, i, j, k, &D, &C, &U);
                    const double m = (k == 0) ? C : C - D * cp;
                    const double im = 1.0 / m;
                    cp = U * im;
                    ep = ((k == 0) ? r[k] : r[k] - D * ep) * im;
                    c[k] = cp;
                    e[k] = ep;
                }
                double xk = e[nz - 1];
                L->x[IX(g, i, j, nz - 1)] += xk;
                for (int k = nz - 2; k >= 0; --k) {
                    xk = e[k] - c[k] * xk;
                    L->x[IX(g, i, j, k)] += xk;
                }
            }
        }
    }
}

/* r = b - A x on the valid cells of level L. */
static void mg_residual(og_mg* mg, og_level* L)
{
    const og_grid* g = &L->g;
    og_poisson_fill_ghosts(g, mg->bc, L->x, ground_even(mg->bc));
    const int zf = og_poisson_zero_flux_faces(g, mg->bc);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                L->r[IX(g, i, j, k)] = L->b[IX(g, i, j, k)] - adotx_cell(g, i, j, k, L->x, L->AX, L->AY, L->AZ, L->J, L->z, zf);
            }
        }
    }
}

/* Coarse right-hand side: the J-weighted sum of the four fine residuals over
 * 4 J_c (the coarse cell's flux balance is the sum of the fine ones). */
static void mg_restrict(og_level* F, og_level* C)
{
    const og_grid* fg = &F->g;
    const og_grid* cg = &C->g;
    for (int k = 0; k < cg->nz; ++k) {
        for (int J2 = 0; J2 < cg->ny; ++J2) {
            for (int I = 0; I < cg->nx; ++I) {
                const int i = 2 * I, j = 2 * J2;
                const double s = (F->J[IX(fg, i, j, k)] * F->r[IX(fg, i, j, k)] + F->J[IX(fg, i + 1, j, k)] * F->r[IX(fg, i + 1, j, k)])
                               + (F->J[IX(fg, i, j + 1, k)] * F->r[IX(fg, i, j + 1, k)]
                                  + F->J[IX(fg, i + 1, j + 1, k)] * F->r[IX(fg, i + 1, j + 1, k)]);
                C->b[IX(cg, I, J2, k)] = s / (4.0 * C->J[IX(cg, I, J2, k)]);
            }
        }
    }
}

/* Fine correction: bilinear in x-y from the coarse cell centres (weights 9, 3,
 * 3, 1 over 16 towards the fine cell's corner), coarse ghosts from the BC. */
static void mg_prolong_add(og_mg* mg, og_level* C, og_level* F)
{
    const og_grid* fg = &F->g;
    const og_grid* cg = &C->g;
    og_poisson_fill_ghosts(cg, mg->bc, C->x, ground_even(mg->bc));
    for (int k = 0; k < fg->nz; ++k) {
        for (int j = 0; j < fg->ny; ++j) {
            for (int i = 0; i < fg->nx; ++i) {
                const int I = i >> 1, J2 = j >> 1;
                const int si = (i & 1) ? 1 : -1, sj = (j & 1) ? 1 : -1;
                const double v = (9.0 * C->x[IX(cg, I, J2, k)] + 3.0 * C->x[IX(cg, I + si, J2, k)])
                               + (3.0 * C->x[IX(cg, I, J2 + sj, k)] + 1.0 * C->x[IX(cg, I + si, J2 + sj, k)]);
                F->x[IX(fg, i, j, k)] += v * 0.0625;
            }
        }
    }
}

static void zero_valid(const og_grid* g, double* f)
{
    memset(f, 0, sizeof(double) * VOL(g));
}

static void vcycle(og_mg* mg, int l)
{
    og_level* L = &mg->lev[l];
    if (l == mg->nlev - 1) {
        for (int s = 0; s < mg->nu_coarse; ++s) { mg_smooth(mg, L); }
        return;
    }
    for (int s = 0; s < mg->nu1; ++s) { mg_smooth(mg, L); }
    mg_residual(mg, L);
    og_level* C = &mg->lev[l + 1];
    mg_restrict(L, C);
    zero_valid(&C->g, C->x);
    vcycle(mg, l + 1);
    mg_prolong_add(mg, C, L);
    for (int s = 0; s < mg->nu2; ++s) { mg_smooth(mg, L); }
}

/* One V-cycle for A e = r from e = 0: e (fine grid array) receives the
 * correction. The fine level's b is r. */
void og_mg_vcycle(og_mg* mg, const double* r, double* e)
{
    og_level* L = &mg->lev[0];
    const int64_t vol = VOL(&L->g);
    memcpy(L->b, r, sizeof(double) * vol);
    zero_valid(&L->g, L->x);
    vcycle(mg, 0);
    memcpy(e, L->x, sizeof(double) * vol);
}

/* ------------------------------------------------------------------ */
/* the solve                                                           */
/* ------------------------------------------------------------------ */

static double dot_valid(const og_grid* g, const double* a, const double* b)
{
    double s = 0;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) { s += a[IX(g, i, j, k)] * b[IX(g, i, j, k)]; }
        }
    }
    return s;
}

static double sum_valid(const og_grid* g, const double* a)
{
    double s = 0;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) { s += a[IX(g, i, j, k)]; }
        }
    }
    return s;
}

/* Source/Poisson.cpp:37-40 (weighted_mean). */
double og_weighted_mean(const og_grid* g, const double* f, const double* J)
{
    return dot_valid(g, J, f) / sum_valid(g, J);
}

static void add_const_valid(const og_grid* g, double* f, double c)
{
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) { f[IX(g, i, j, k)] += c; }
        }
    }
}

/* Restarted right-preconditioned flexible GMRES for A phi = rhs (phi = 0
 * initially), preconditioned by one V-cycle (precond = 1) or none (0), to
 * ||r|| <= max(reltol ||rhs||, abstol). The singular case (no Dirichlet face)
 * removes the J-weighted mean of rhs first and of phi after (Source/Poisson.cpp:
 * 556-588). Returns iterations (negative when not converged); res[0] initial,
 * res[1] final (true) residual 2-norm, res[2] removed mean. */
int og_poisson_solve(og_mg* mg, double* rhs, double* phi, double reltol, double abstol, int max_iter, int restart,
                     int precond, double* res)
{
    og_level* L = &mg->lev[0];
    const og_grid* g = &L->g;
    const int64_t vol = VOL(g);
    int singular = 1;
    for (int f = 0; f < 6; ++f) {
        if (mg->bc[f] == PF_DIRICHLET) { singular = 0; }
    }
    res[2] = 0;
    if (singular) {
        res[2] = og_weighted_mean(g, rhs, L->J);
        add_const_valid(g, rhs, -res[2]);
    }
    const int m = restart;
    double* V = (double*)calloc((size_t)(m + 1) * vol, sizeof(double));
    double* Zs = (double*)calloc((size_t)m * vol, sizeof(double));
    double* H = (double*)calloc((size_t)(m + 1) * m, sizeof(double));
    double* cs = (double*)calloc(m, sizeof(double));
    double* sn = (double*)calloc(m, sizeof(double));
    double* s = (double*)calloc(m + 1, sizeof(double));
    double* w = (double*)calloc(vol, sizeof(double));
    double* t = (double*)calloc(vol, sizeof(double));
    memset(phi, 0, sizeof(double) * vol);
    const double bnorm = sqrt(dot_valid(g, rhs, rhs));
    res[0] = bnorm;
    const double tol = fmax(reltol * bnorm, abstol);
    int it = 0, converged = (bnorm <= tol);
    while (!converged && it < max_iter) {
        /* r = rhs - A phi */
        mg_apply(mg, phi, t);
        memset(w, 0, sizeof(double) * vol);
        for (int k = 0; k < g->nz; ++k) {
            for (int j = 0; j < g->ny; ++j) {
                for (int i = 0; i < g->nx; ++i) { w[IX(g, i, j, k)] = rhs[IX(g, i, j, k)] - t[IX(g, i, j, k)]; }
            }
        }
        const double beta = sqrt(dot_valid(g, w, w));
        if (beta <= tol) { converged = 1; break; }
        for (int64_t n = 0; n < vol; ++n) { V[n] = w[n] / beta; }
        memset(s, 0, sizeof(double) * (m + 1));
        s[0] = beta;
        int jj = 0;
        for (; jj < m && it < max_iter; ++jj, ++it) {
            double* vj = V + (size_t)jj * vol;
            double* zj = Zs + (size_t)jj * vol;
            if (precond) { og_mg_vcycle(mg, vj, zj); } else { memcpy(zj, vj, sizeof(double) * vol); }
            mg_apply(mg, zj, w);
            /* modified Gram-Schmidt */
            for (int q = 0; q <= jj; ++q) {
                const double* vq = V + (size_t)q * vol;
                const double h = dot_valid(g, w, vq);
                H[q * m + jj] = h;
                for (int k = 0; k < g->nz; ++k) {
                    for (int j2 = 0; j2 < g->ny; ++j2) {
                        for (int i = 0; i < g->nx; ++i) { w[IX(g, i, j2, k)] -= h * vq[IX(g, i, j2, k)]; }
                    }
                }
            }
            const double hn = sqrt(dot_valid(g, w, w));
            H[(jj + 1) * m + jj] = hn;
            double* vn = V + (size_t)(jj + 1) * vol;
            memset(vn, 0, sizeof(double) * vol);
            if (hn > 0) {
                for (int k = 0; k < g->nz; ++k) {
                    for (int j2 = 0; j2 < g->ny; ++j2) {
                        for (int i = 0; i < g->nx; ++i) { vn[IX(g, i, j2, k)] = w[IX(g, i, j2, k)] / hn; }
                    }
                }
            }
            for (int q = 0; q < jj; ++q) {
                const double a = H[q * m + jj], b2 = H[(q + 1) * m + jj];
                H[q * m + jj] = cs[q] * a + sn[q] * b2;
                H[(q + 1) * m + jj] = -sn[q] * a + cs[q] * b2;
            }
            const double a = H[jj * m + jj], b2 = H[(jj + 1) * m + jj];
            const double rr = sqrt(a * a + b2 * b2);
            cs[jj] = (rr > 0) ? a / rr : 1.0;
            sn[jj] = (rr > 0) ? b2 / rr : 0.0;
            H[jj * m + jj] = rr;
            H[(jj + 1) * m + jj] = 0;
            s[jj + 1] = -sn[jj] * s[jj];
            s[jj] = cs[jj] * s[jj];
            if (fabs(s[jj + 1]) <= tol) { ++jj; ++it; break; }
        }
        /* solve the triangular system and update phi */
        double y[1024];
        for (int q = jj - 1; q >= 0; --q) {
            double acc = s[q];
            for (int p = q + 1; p < jj; ++p) { acc -= H[q * m + p] * y[p]; }
            y[q] = acc / H[q * m + q];
        }
        for (int q = 0; q < jj; ++q) {
            const double* zq = Zs + (size_t)q * vol;
            for (int k = 0; k < g->nz; ++k) {
                for (int j2 = 0; j2 < g->ny; ++j2) {
                    for (int i = 0; i < g->nx; ++i) { phi[IX(g, i, j2, k)] += y[q] * zq[IX(g, i, j2, k)]; }
                }
            }
        }
        memset(H, 0, sizeof(double) * (m + 1) * m);
    }
    if (singular) { add_const_valid(g, phi, -og_weighted_mean(g, phi, L->J)); }
    mg_apply(mg, phi, t);
    double rn = 0;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const double d = rhs[IX(g, i, j, k)] - t[IX(g, i, j, k)];
                rn += d * d;
            }
        }
    }
    res[1] = sqrt(rn);
    converged = res[1] <= tol * 1.0000001 || converged;
    free(V);
    free(Zs);
    free(H);
    free(cs);
    free(sn);
    free(s);
    free(w);
    free(t);
    return converged ? it : -it - 1;
}
