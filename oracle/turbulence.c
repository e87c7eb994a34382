/*
 * ORACLE -- test infrastructure, not product code. FP64 C restatement of the
 * reference's k-L closure and surface layer, in its operation order:
 *   Source/Closure_K.H:70-185 (point kernels; extern_erf/ERF_RANSClosure.H),
 *   Source/Closure.cpp:93-103 (live decisions), :270-300 (height above the
 *   ground), :302-345 (N^2 and S^2), :365-460 (evaluate, no relaxation
 *   history, no stratification gate, no realizability cap);
 *   Source/SurfaceLayer.cpp:36-230 (the columns' MOST state), :418-502
 *   (ground fluxes, wall k), :503-569 (the first cells' implicit rows);
 *   Source/StabilityFunctions.H (Businger-Dyer psi_m, phi_m, phi_h);
 *   Source/BoundaryConditions.cpp:549-593 (the wall law's ground gradient)
 *   and :614-648 (its ghost columns);
 *   Source/WallDistance.cpp:13-62 and Source/Sequencing.cpp:43-60 (Tucker's
 *   wall distance from the Poisson solution, and its ghosts).
 * Only tests/, the smoke check and the benchmark's CPU legs use it.
 */
#include <float.h>
#include <math.h>
#include <string.h>

#include "og.h"

#include "../include/gust_b200.h"

enum { CC = 0, XF = 1, YF = 2, ZF = 4, NODE = 7 };

double og_interp(const og_grid* g, const double* q, int tq, int ts, int i, int j, int k);
double og_deriv(const og_grid* g, const double* q, int tq, int ts, int m, int i, int j, int k);
void og_grad_at(const og_grid* g, const double* q, int tq, int ts, const double* z, int i, int j, int k, double out[3]);

/* ------------------------------------------------------------------ */
/* closure point kernels (Closure_K.H)                                 */
/* ------------------------------------------------------------------ */

typedef struct {
    double kappa, Cmu0, Cmu0_pow3, inv_Cb_sq, Rt_crit, Rt_min, l_g_max, tke_floor, n2_eps;
} cconst;

typedef struct {
    int branch, smooth_Rt_g, smooth_Rt, floored;
} switches;

typedef struct {
    double k, L, Rt, cmu, cmu_prime, nut, nut_prime, eps, Ps, Pb;
} cpoint;

/* closure_constants (Closure.cpp:258-272). */
static cconst closure_constants(const gb_physics* ph)
{
    cconst c;
    c.kappa = ph->turb_kappa;
    c.Cmu0 = ph->turb_Cmu0;
    c.Cmu0_pow3 = ph->turb_Cmu0 * ph->turb_Cmu0 * ph->turb_Cmu0;
    c.inv_Cb_sq = 1.0 / (ph->turb_Cb * ph->turb_Cb);
    c.Rt_crit = ph->turb_Rt_crit;
    c.Rt_min = ph->turb_Rt_min;
    c.l_g_max = ph->turb_max_geom_lscale;
    c.tke_floor = fmax(ph->turb_tke_floor, DBL_EPSILON);
    c.n2_eps = DBL_EPSILON;
    return c;
}

static double pos_part(double x) { return 0.5 * (x + fabs(x)); }
static double neg_part(double x) { return 0.5 * (x - fabs(x)); }
static double geom_length(double l_g_raw, double l_g_max) { return l_g_max * l_g_raw / (l_g_max + l_g_raw); }

static double smooth_Rt(double Rt, int smooth, double Rt_crit, double Rt_min)
{
    const double x = neg_part(Rt - Rt_crit);
    const double a = Rt_min - Rt_crit;
    const double smoothed = Rt_crit + a * x / (x + a);
    return smooth ? smoothed : Rt;
}

static switches switches_for(double k, double N2, double l_g, const cconst* c)
{
    switches s;
    s.floored = !(k > c->tke_floor);
    const double kf = s.floored ? c->tke_floor : k;
    s.branch = (fabs(N2) <= c->n2_eps) ? 0 : (N2 > c->n2_eps) ? 1 : 2;
    const double c6 = c->Cmu0_pow3 * c->Cmu0_pow3;
    const double N2s = pos_part(N2), N2u = neg_part(N2);
    const double Rt_g = l_g * l_g * N2u / (kf * c->Cmu0_pow3 * c->Cmu0_pow3);
    s.smooth_Rt_g = (s.branch == 2) && (Rt_g < c->Rt_crit);
    const double L_unstable = l_g * sqrt(1.0 - c6 * c->inv_Cb_sq * smooth_Rt(Rt_g, s.smooth_Rt_g, c->Rt_crit, c->Rt_min));
    const double L_stable = sqrt(1.0 / (1.0 / (l_g * l_g) + c->inv_Cb_sq * N2s / kf));
    const double L = (s.branch == 0) ? l_g : (s.branch == 1) ? L_stable : L_unstable;
    s.smooth_Rt = (L * L * N2 / (kf * c->Cmu0_pow3 * c->Cmu0_pow3) < c->Rt_crit);
    return s;
}

static cpoint closure_point(double k, double N2, double S2, double l_g, const cconst* c, switches s)
{
    cpoint p;
    p.k = s.floored ? c->tke_floor : k;
    const double c6 = c->Cmu0_pow3 * c->Cmu0_pow3;
    const double N2s = pos_part(N2), N2u = neg_part(N2);
    const double L_stable = sqrt(1.0 / (1.0 / (l_g * l_g) + c->inv_Cb_sq * N2s / p.k));
    const double Rt_g = l_g * l_g * N2u / (p.k * c->Cmu0_pow3 * c->Cmu0_pow3);
    const double L_unstable = l_g * sqrt(1.0 - c6 * c->inv_Cb_sq * smooth_Rt(Rt_g, s.smooth_Rt_g, c->Rt_crit, c->Rt_min));
    p.L = (s.branch == 0) ? l_g : (s.branch == 1) ? L_stable : L_unstable;
    p.eps = c->Cmu0_pow3 * pow(p.k, 1.5) / p.L;
    p.Rt = smooth_Rt(p.L * p.L * N2 / (p.k * c->Cmu0_pow3 * c->Cmu0_pow3), s.smooth_Rt, c->Rt_crit, c->Rt_min);
    p.cmu = (c->Cmu0 + 0.108 * p.Rt) / (1.0 + 0.308 * p.Rt + 0.00837 * p.Rt * p.Rt);
    p.cmu_prime = c->Cmu0 / (1.0 + 0.277 * p.Rt);
    p.nut = p.cmu * sqrt(p.k) * p.L;
    p.nut_prime = p.cmu_prime / p.cmu * p.nut;
    p.Ps = p.nut * S2;
    p.Pb = -p.nut_prime * N2;
    return p;
}

/* ------------------------------------------------------------------ */
/* the closure's fields (Closure.cpp)                                  */
/* ------------------------------------------------------------------ */

/* The vertical ghost layers take the adjacent cell's values, over the
 * lateral range -1..nx, -1..ny (copy_vertical_ghosts, :130-146). */
static void copy_vertical_ghosts(const og_grid* g, double* a)
{
    for (int j = -1; j <= g->ny; ++j) {
        for (int i = -1; i <= g->nx; ++i) {
            a[IX(g, i, j, -1)] = a[IX(g, i, j, 0)];
            a[IX(g, i, j, g->nz)] = a[IX(g, i, j, g->nz - 1)];
        }
    }
}

/* height_above_ground (Closure.cpp:270-300): the cell centre's node-mean
 * height minus its column's node-mean ground, on -1..nx, -1..ny. */
void og_height_above_ground(const og_grid* g, const double* z, double* dist)
{
    for (int k = 0; k < g->nz; ++k) {
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx; ++i) {
                double zc = 0, zg = 0;
                for (int a = 0; a < 2; ++a) {
                    for (int b = 0; b < 2; ++b) {
                        zg += z[IX(g, i + a, j + b, 0)];
                        zc += z[IX(g, i + a, j + b, k)] + z[IX(g, i + a, j + b, k + 1)];
                    }
                }
                dist[IX(g, i, j, k)] = 0.125 * zc - 0.25 * zg;
            }
        }
    }
    copy_vertical_ghosts(g, dist);
}

/* stratification_and_strain (Closure.cpp:302-345): N^2 = (g/theta_0)
 * dtheta/dz and S^2 = 2 S_ij S_ij from the physical gradients at the cells. */
void og_stratification_and_strain(const og_grid* g, const gb_physics* ph, const double* u, const double* v,
                                  const double* w, const double* th, const double* z, double* N2, double* S2)
{
    const double g_over_theta0 = ph->gravity / ph->theta0;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < g->nz; ++k) {
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx; ++i) {
                double gt[3], gu[3], gv[3], gw[3];
                og_grad_at(g, th, CC, CC, z, i, j, k, gt);
                N2[IX(g, i, j, k)] = g_over_theta0 * gt[2];
                og_grad_at(g, u, XF, CC, z, i, j, k, gu);
                og_grad_at(g, v, YF, CC, z, i, j, k, gv);
                og_grad_at(g, w, ZF, CC, z, i, j, k, gw);
                const double G[3][3] = {{gu[0], gu[1], gu[2]}, {gv[0], gv[1], gv[2]}, {gw[0], gw[1], gw[2]}};
                double s = 0;
                for (int a = 0; a < 3; ++a) {
                    for (int b = 0; b < 3; ++b) {
                        const double e = G[a][b] + G[b][a];
                        s += e * e;
                    }
                }
                S2[IX(g, i, j, k)] = 0.5 * s;
            }
        }
    }
    copy_vertical_ghosts(g, N2);
    copy_vertical_ghosts(g, S2);
}

/* The roughness the closure's length reads (Closure.cpp:54-91,
 * ground_roughness): a column's map value, the uniform bc.surface_z0, or 0
 * without a surface layer. */
static double column_z0(const og_grid* g, const gb_bc* bc, const double* z0map, int i, int j)
{
    if (bc->face[2] != GB_FACE_SURFACE_LAYER) { return 0.0; }
    return z0map ? z0map[(int64_t)(i + g->ng) + (int64_t)(j + g->ng) * g->sy] : bc->surface_z0;
}

/* Closure::evaluate (Closure.cpp:365-460) with the nu_t relaxation against
 * the history og_set_nut_history gave (weight 1 without one), the
 * stratification gate of turb.ri_gate (gate_stratification,
 * Closure.cpp:337-354: the length and Rt see N^2 N^4 / (N^4 + Ri_0^2 S^4),
 * P_b keeps N^2) and the realizability cap of turb.realizability
 * (nut_cap_field, ClosureWake.cpp:8-29: nu_t <= C_r max(k, floor) / S):
 * nu, gamma_theta, gamma_tke and nu_t on the
 * cells -1..nx, -1..ny (their vertical ghosts copied), the length, Rt, P_s,
 * P_b, eps and the Patankar diagonal on the valid cells. out: 10 arrays in
 * that order (nu, gth, gk, nut, L, Rt, Ps, Pb, eps, dSdk). */
/* The nu_t history of Closure::accept (Closure.cpp:471-479) that
 * og_closure_evaluate blends with (turb.nut_relax < 1); NULL: none. The
 * Python side sets it from the case before each evaluation. */
static const double* g_nut_prev = NULL;
void og_set_nut_history(const double* prev) { g_nut_prev = prev; }

/* The closure's wall distance (ResidualInputs::wall_distance,
 * Source/Residual.H:61-128): an array the Python side sets from the case
 * (the Tucker distance of turb.wall_distance = tucker), or NULL: the
 * height above the ground (turb.wall_distance = terrain_height). */
static const double* g_wall_dist = NULL;
void og_set_wall_distance(const double* d) { g_wall_dist = d; }

/* distance_from_phi (Source/WallDistance.cpp:13-62): Tucker's
 * d = -|grad phi| + sqrt(|grad phi|^2 + 2 phi) on the valid cells, with
 * ERF's cell-centred physical gradient (centred differences, the cell-centre
 * metrics) and, in the first cell, the quadratic through phi = 0 on the
 * ground and the two lowest cell centres; phi's ghosts filled for the
 * Tucker conditions. Then extend_by_zero_gradient (Source/Sequencing.cpp:
 * 43-60): every ghost takes the value of the valid cell its periodic image
 * or, across a non-periodic face, the nearest one. */
void og_tucker_distance(const og_grid* g, const double* z, const double* p, double* d)
{
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy, dzinv = 1.0 / g->dzeta;
#define P(a, b, c) p[IX(g, a, b, c)]
#define ZN(a, b, c) z[IX(g, a, b, c)]
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const double dpdxi = 0.5 * (P(i + 1, j, k) - P(i - 1, j, k)) * dxinv;
                const double dpdeta = 0.5 * (P(i, j + 1, k) - P(i, j - 1, k)) * dyinv;
                const double dpdzeta = 0.5 * (P(i, j, k + 1) - P(i, j, k - 1)) * dzinv;
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
                    const double zw = 0.25 * (ZN(i, j, 0) + ZN(i + 1, j, 0) + ZN(i, j + 1, 0) + ZN(i + 1, j + 1, 0));
                    const double c1 = 0.25 * (ZN(i, j, 1) + ZN(i + 1, j, 1) + ZN(i, j + 1, 1) + ZN(i + 1, j + 1, 1));
                    const double c2 = 0.25 * (ZN(i, j, 2) + ZN(i + 1, j, 2) + ZN(i, j + 1, 2) + ZN(i + 1, j + 1, 2));
                    const double a = 0.5 * (zw + c1) - zw;
                    const double b = 0.5 * (c1 + c2) - zw;
                    dpdz = (P(i, j, 0) * b * (b - 2.0 * a) + P(i, j, 1) * a * a) / (a * b * (b - a));
                }
                const double dpdx = dpdxi - h_xi * dpdz;
                const double dpdy = dpdeta - h_eta * dpdz;
                const double g2 = dpdx * dpdx + dpdy * dpdy + dpdz * dpdz;
                d[IX(g, i, j, k)] = -sqrt(g2) + sqrt(g2 + 2.0 * P(i, j, k));
            }
        }
    }
#undef P
#undef ZN
    const int ng = g->ng;
    for (int k = -ng; k <= g->nz + ng; ++k) {
        for (int j = -ng; j <= g->ny + ng; ++j) {
            for (int i = -ng; i <= g->nx + ng; ++i) {
                if (i >= 0 && i < g->nx && j >= 0 && j < g->ny && k >= 0 && k < g->nz) { continue; }
                int ii = i, jj = j;
                if (g->periodic_x) { ii = ((i % g->nx) + g->nx) % g->nx; } else { ii = i < 0 ? 0 : (i >= g->nx ? g->nx - 1 : i); }
                if (g->periodic_y) { jj = ((j % g->ny) + g->ny) % g->ny; } else { jj = j < 0 ? 0 : (j >= g->ny ? g->ny - 1 : j); }
                const int kk = k < 0 ? 0 : (k >= g->nz ? g->nz - 1 : k);
                d[IX(g, i, j, k)] = d[IX(g, ii, jj, kk)];
            }
        }
    }
}

void og_closure_evaluate(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const double* u, const double* v,
                         const double* w, const double* th, const double* tk, const double* z, const double* z0map,
                         double** out)
{
    const cconst c = closure_constants(ph);
    const int64_t vol = VOL(g);
    double* dist = (double*)calloc(vol, sizeof(double));
    double* N2 = (double*)calloc(vol, sizeof(double));
    double* S2 = (double*)calloc(vol, sizeof(double));
    if (g_wall_dist != NULL) {
        memcpy(dist, g_wall_dist, sizeof(double) * vol);
    } else {
        og_height_above_ground(g, z, dist);
    }
    og_stratification_and_strain(g, ph, u, v, w, th, z, N2, S2);
    const double nu_mol = ph->turb_nu_molecular, alpha_mol = ph->turb_alpha_molecular;
    const double inv_sigma = 1 / ph->turb_sigma_k;
    const double wgt = g_nut_prev ? ph->turb_nut_relax : 1.0;
    const double* prev = g_nut_prev ? g_nut_prev : tk;
    const double ri0 = ph->turb_ri_gate, r2 = ri0 * ri0, cr = ph->turb_realizability;
    double *nu = out[0], *gth = out[1], *gk = out[2], *nut = out[3];
    for (int k = 0; k < g->nz; ++k) {
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx; ++i) {
                const int64_t o = IX(g, i, j, k);
                /* kappa (d + z0): with a map the sum d + z0(i, j) is formed
                 * first and the kernel adds z0 = 0, the same value */
                const double l_g = geom_length(c.kappa * (dist[o] + column_z0(g, bc, z0map, i, j)), c.l_g_max);
                double N2c = N2[o];
                if (ri0 > 0) {
                    const double a = N2[o] * N2[o], b = S2[o] * S2[o];
                    N2c *= a / (a + r2 * b + DBL_MIN);
                }
                const switches s = switches_for(tk[o], N2c, l_g, &c);
                const cpoint p = closure_point(tk[o], N2c, S2[o], l_g, &c, s);
                const double ratio = p.cmu_prime / p.cmu;
                double cap = DBL_MAX;
                if (cr > 0) {
                    const double sr = sqrt(S2[o]);
                    cap = (sr > DBL_MIN) ? cr * fmax(tk[o], c.tke_floor) / sr : DBL_MAX;
                }
                const double nt = wgt * fmin(p.nut, cap) + (1 - wgt) * prev[o];
                nut[o] = nt;
                nu[o] = nu_mol + nt;
                gth[o] = alpha_mol + ratio * nt;
                gk[o] = nu_mol + nt * inv_sigma;
                if (i >= 0 && i < g->nx && j >= 0 && j < g->ny) {
                    const double Ps = nt * S2[o], Pb = -ratio * nt * N2[o];
                    out[4][o] = p.L;
                    out[5][o] = p.Rt;
                    out[6][o] = Ps;
                    out[7][o] = Pb;
                    out[8][o] = p.eps;
                    out[9][o] = (p.eps + pos_part(-Pb)) / p.k;
                }
            }
        }
    }
    for (int n = 0; n < 4; ++n) { copy_vertical_ghosts(g, out[n]); }
    free(dist);
    free(N2);
    free(S2);
}

/* ------------------------------------------------------------------ */
/* the surface layer (SurfaceLayer.cpp)                                */
/* ------------------------------------------------------------------ */

static int64_t PX(const og_grid* g, int i, int j) { return (int64_t)(i + g->ng) + (int64_t)(j + g->ng) * g->sy; }

/* The vertical height of cell (i, j, k)'s centre above its column's ground. */
static double column_height(const og_grid* g, const double* z, int i, int j, int k)
{
    const double ground = 0.25 * ((z[IX(g, i, j, 0)] + z[IX(g, i + 1, j, 0)]) + (z[IX(g, i, j + 1, 0)] + z[IX(g, i + 1, j + 1, 0)]));
    return og_interp(g, z, NODE, CC, i, j, k) - ground;
}

static void tangential_wind(const og_grid* g, const double* u, const double* v, const double* w, int i, int j, int k,
                            const double n[3], double ut[3])
{
    const double U[3] = {0.5 * (u[IX(g, i, j, k)] + u[IX(g, i + 1, j, k)]), 0.5 * (v[IX(g, i, j, k)] + v[IX(g, i, j + 1, k)]),
                         0.5 * (w[IX(g, i, j, k)] + w[IX(g, i, j, k + 1)])};
    const double un = U[0] * n[0] + U[1] * n[1] + U[2] * n[2];
    for (int d = 0; d < 3; ++d) { ut[d] = U[d] - un * n[d]; }
}

static void tangential_wind_ground(const og_grid* g, const double* u, const double* v, int i, int j, int k, double zx,
                                   double zy, const double n[3], double ut[3])
{
    const double uc = 0.5 * (u[IX(g, i, j, k)] + u[IX(g, i + 1, j, k)]);
    const double vc = 0.5 * (v[IX(g, i, j, k)] + v[IX(g, i, j + 1, k)]);
    const double U[3] = {uc, vc, zx * uc + zy * vc};
    const double un = U[0] * n[0] + U[1] * n[1] + U[2] * n[2];
    for (int d = 0; d < 3; ++d) { ut[d] = U[d] - un * n[d]; }
}

/* The stable side (StabilityFunctions.H StableCoefficients): Businger-Dyer
 * (5, 0, 5, 0) or QNSE's coefficients from bc.surface_qnse_*. */
typedef struct {
    int qnse;
    double am, bm, ah, bh;
} stable_c;

static stable_c stable_of(const gb_bc* bc)
{
    stable_c s = {0, 5.0, 0.0, 5.0, 0.0};
    if (bc->surface_qnse) {
        s.qnse = 1;
        s.am = bc->surface_qnse_am;
        s.bm = bc->surface_qnse_bm;
        s.ah = bc->surface_qnse_ah;
        s.bh = bc->surface_qnse_bh;
    }
    return s;
}

/* psi_m (ERF_MOSTUtils.H:102-111 unstable side, StabilityFunctions.H
 * most_psi_m): the stable side -5 zeta or -((a - b)/b) ln(1 + b zeta). */
static double psi_m(double zeta, const stable_c* sc)
{
    const double az = fabs(zeta);
    const double zs = 0.5 * (az + zeta), zu = 0.5 * (zeta - az);
    if (zeta > 0) { return sc->qnse ? -((sc->am - sc->bm) / sc->bm) * log(1.0 + sc->bm * zs) : -5.0 * zs; }
    const double x = sqrt(sqrt(1.0 - 16.0 * zu));
    const double pi = 3.14159265358979323846264338327950288;
    return 2.0 * log(0.5 * (1.0 + x)) + log(0.5 * (1.0 + x * x)) - 2.0 * atan(x) + pi / 2.0;
}

/* most_phi (StabilityFunctions.H) with the stable side's coefficients. */
static void most_phi(double zeta, const stable_c* sc, double* phi_m, double* phi_h)
{
    const double one = 1, gamma = 16, am = sc->am, bm = sc->bm, ah = sc->ah, bh = sc->bh;
    const double az = fabs(zeta);
    const double zs = 0.5 * (az + zeta);
    const double zu = 0.5 * (zeta - az);
    const double r = sqrt(one - gamma * zu);
    *phi_m = (one + am * zs) / (one + bm * zs) + (one / sqrt(r) - one);
    *phi_h = (one + ah * zs) / (one + bh * zs) + (one / r - one);
}

typedef struct {
    double kappa, U, d, lz, den_min, gq, ustar_min;
    stable_c sc;
} most_rel;

static double most_inv_L(const most_rel* F, double u)
{
    const double uf = fmax(u, F->ustar_min);
    return -F->kappa * F->gq / (uf * uf * uf);
}

static double most_F(const most_rel* F, double u)
{
    const double zeta = fmax(fmin(F->d * most_inv_L(F, u), 100.0), -100.0);
    return u - F->kappa * F->U / fmax(F->lz - psi_m(zeta, &F->sc), F->den_min);
}

static int reference_interval(const og_grid* g, const double* z, int i, int j, int n, double zr)
{
    if (zr < column_height(g, z, i, j, 0)) { return -1; }
    if (zr > column_height(g, z, i, j, n - 1)) { return n - 1; }
    int k = 0;
    while (k < n - 2 && !(zr < column_height(g, z, i, j, k + 1))) { ++k; }
    return k;
}

/* compute_surface_state's columns (SurfaceLayer.cpp:97-230) on the columns
 * -1..nx, -1..ny. ss: the planes ustar, speed, zref, d0, inv_L, tau_x,
 * tau_y, tau_z, drag, kwall, area (11). Returns the number of columns
 * without a positive, finite u* or with a non-finite k_w. */
int og_surface_state(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const double* u, const double* v,
                     const double* w, const double* z, const double* z0map, double** ss)
{
    const int nz = g->nz;
    const double kappa = bc->kappa;
    const int heat = bc->surface_stability == GB_SURFACE_HEAT_FLUX;
    const int first = !(bc->surface_zref > 0);
    const int floor_one = bc->surface_denominator_floor == GB_DENOMINATOR_ONE;
    const double gq = (ph->gravity / ph->theta0) * bc->surface_heat_flux;
    const double inv_cmu2 = 1.0 / (bc->Cmu0 * bc->Cmu0);
    const double eps = DBL_EPSILON, tol = 64 * eps, hrel = sqrt(eps);
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy;
    int bad = 0;
    for (int j = -1; j <= g->ny; ++j) {
        for (int i = -1; i <= g->nx; ++i) {
            const double z0 = z0map ? z0map[PX(g, i, j)] : bc->surface_z0;
            const double zx = og_deriv(g, z, NODE, ZF, 0, i, j, 0) * dxinv;
            const double zy = og_deriv(g, z, NODE, ZF, 1, i, j, 0) * dyinv;
            const double area = sqrt(1 + zx * zx + zy * zy);
            const double n[3] = {-zx / area, -zy / area, 1 / area};
            const double h0 = column_height(g, z, i, j, 0);
            const double zr = first ? h0 : bc->surface_zref;
            int k = reference_interval(g, z, i, j, nz, zr);
            k = k < 0 ? 0 : (k > nz - 2 ? nz - 2 : k);
            double ua[3], ub[3];
            if (k == 0) {
                tangential_wind_ground(g, u, v, i, j, 0, zx, zy, n, ua);
            } else {
                tangential_wind(g, u, v, w, i, j, k, n, ua);
            }
            tangential_wind(g, u, v, w, i, j, k + 1, n, ub);
            const double ia = 1.0 / area;
            const double la = log(column_height(g, z, i, j, k) * ia + z0);
            const double f = (log(zr * ia + z0) - la) / (log(column_height(g, z, i, j, k + 1) * ia + z0) - la);
            double ut[3];
            for (int c = 0; c < 3; ++c) { ut[c] = ua[c] + f * (ub[c] - ua[c]); }
            const double mag = sqrt(ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2]);
            const double U = fmax(mag, 0.1);
            const double d = zr * ia;
            const double lz = log((d + z0) / z0);
            double den_min = fmin(lz, 1.0);
            if (floor_one) { den_min = 1.0; }
            double ustar = kappa * U / fmax(lz, den_min);
            double invL = 0;
            if (heat) {
                const most_rel F = {kappa, U, d, lz, den_min, gq, 0.001, stable_of(bc)};
                int converged = 0;
                for (int it = 0; it < 50 && !converged; ++it) {
                    const double fu = most_F(&F, ustar);
                    const double du = hrel * ustar;
                    const double fp = (most_F(&F, ustar + du) - fu) / du;
                    double next = (fp > 0) ? ustar - fu / fp : ustar - 0.5 * fu;
                    next = fmax(0.5 * ustar, fmin(2.0 * ustar, next));
                    converged = fabs(next - ustar) <= tol * next;
                    ustar = next;
                }
                if (!converged) { ustar = NAN; }
                invL = most_inv_L(&F, ustar);
            }
            const double d0 = h0 * ia;
            const int64_t p = PX(g, i, j);
            ss[0][p] = ustar;
            ss[1][p] = U;
            ss[2][p] = zr;
            ss[3][p] = d0;
            ss[4][p] = invL;
            ss[10][p] = area;
            const double cdrag = ustar * ustar / U * area;
            ss[8][p] = cdrag;
            for (int m = 0; m < 3; ++m) { ss[5 + m][p] = cdrag * ut[m]; }
            double kwall = ustar * ustar * inv_cmu2;
            if (heat) { kwall = inv_cmu2 * pow(ustar * ustar * ustar + kappa * fmax(gq, 0.0) * d0, 2.0 / 3.0); }
            ss[9][p] = kwall;
            if (!(ustar == ustar) || !(kwall == kwall) || !(ustar > 0 && ustar < DBL_MAX)) { ++bad; }
        }
    }
    return bad;
}

/* The wall law's gradient of u, v (0, 1) and theta (2) per column
 * (BoundaryConditions.cpp:549-593) on the columns -2..nx+1, -2..ny+1: the
 * surface state's columns, the periodic images, and the nearest domain
 * column for the rest (:614-648). gg: 3 planes. */
void og_ground_gradients(const og_grid* g, const gb_bc* bc, const double* const* ss, const double* z0map, double** gg)
{
    const stable_c sc = stable_of(bc);
    const double unset = DBL_MAX;
    const double kappa = bc->kappa;
    const double qs = (bc->surface_stability == GB_SURFACE_HEAT_FLUX) ? bc->surface_heat_flux : 0.0;
    for (int j = -2; j <= g->ny + 1; ++j) {
        for (int i = -2; i <= g->nx + 1; ++i) {
            for (int n = 0; n < 3; ++n) { gg[n][PX(g, i, j)] = unset; }
        }
    }
    for (int j = -1; j <= g->ny; ++j) {
        for (int i = -1; i <= g->nx; ++i) {
            const int64_t p = PX(g, i, j);
            const double zeta = fmax(fmin(ss[3][p] * ss[4][p], 100.0), -100.0);
            double phi_m, phi_h;
            most_phi(zeta, &sc, &phi_m, &phi_h);
            const double z0 = z0map ? z0map[p] : bc->surface_z0;
            const double s = kappa * (ss[3][p] + z0);
            const double tx = ss[5][p], ty = ss[6][p], tz = ss[7][p];
            const double tmag = sqrt(tx * tx + ty * ty + tz * tz);
            const double tsafe = tmag + DBL_MIN;
            const double dir_x = tx / tsafe, dir_y = ty / tsafe;
            gg[0][p] = ss[0][p] / s * dir_x * phi_m;
            gg[1][p] = ss[0][p] / s * dir_y * phi_m;
            gg[2][p] = -qs / (ss[0][p] * s) * phi_h;
        }
    }
    /* FillBoundary: a column outside the domain that images a domain column
     * across the periodic directions takes its value */
    for (int j = -2; j <= g->ny + 1; ++j) {
        for (int i = -2; i <= g->nx + 1; ++i) {
            const int inside = i >= 0 && i < g->nx && j >= 0 && j < g->ny;
            if (inside) { continue; }
            int si = i, sj = j;
            if (g->periodic_x) { si = ((i % g->nx) + g->nx) % g->nx; }
            if (g->periodic_y) { sj = ((j % g->ny) + g->ny) % g->ny; }
            if (si >= 0 && si < g->nx && sj >= 0 && sj < g->ny) {
                for (int n = 0; n < 3; ++n) { gg[n][PX(g, i, j)] = gg[n][PX(g, si, sj)]; }
            }
        }
    }
    for (int j = -2; j <= g->ny + 1; ++j) {
        for (int i = -2; i <= g->nx + 1; ++i) {
            if (gg[0][PX(g, i, j)] != unset) { continue; }
            const int ic = g->periodic_x ? i : (i < 0 ? 0 : (i > g->nx - 1 ? g->nx - 1 : i));
            const int jc = g->periodic_y ? j : (j < 0 ? 0 : (j > g->ny - 1 ? g->ny - 1 : j));
            for (int n = 0; n < 3; ++n) { gg[n][PX(g, i, j)] = gg[n][PX(g, ic, jc)]; }
        }
    }
}

/* The gradient of column (i, j) for a point of type t on the ground fill
 * (fill_gradient_z, BoundaryConditions.cpp:495-509): the mean of the two
 * columns beside a nodal face point, clamped to the gradient's columns. */
double og_ground_gradient_at(const og_grid* g, const double* gg, int t, int i, int j)
{
    const int lo = -2, hix = g->nx + 1, hiy = g->ny + 1;
#define CL(a, l, h) ((a) < (l) ? (l) : ((a) > (h) ? (h) : (a)))
    const int ia = CL(i, lo, hix), ja = CL(j, lo, hiy);
    const int ib = CL(nodal(t, 0) ? i - 1 : i, lo, hix), jb = CL(nodal(t, 1) ? j - 1 : j, lo, hiy);
#undef CL
    return 0.5 * (gg[PX(g, ib, jb)] + gg[PX(g, ia, ja)]);
}

/* set_ground_fluxes (SurfaceLayer.cpp:418-450): the wall stress on the
 * ground faces of the u and v control volumes (the mean of the two columns),
 * -q |A| for theta, 0 for k. Gu, Gv, Gt, Gk: the z-flux arrays. */
void og_set_ground_fluxes(const og_grid* g, const gb_bc* bc, const double* const* ss, double* Gu, double* Gv,
                          double* Gt, double* Gk)
{
    const double qs = (bc->surface_stability == GB_SURFACE_HEAT_FLUX) ? bc->surface_heat_flux : 0.0;
    for (int j = 0; j < g->ny; ++j) {
        for (int i = 0; i <= g->nx; ++i) { Gu[IX(g, i, j, 0)] = 0.5 * (ss[5][PX(g, i - 1, j)] + ss[5][PX(g, i, j)]); }
    }
    for (int j = 0; j <= g->ny; ++j) {
        for (int i = 0; i < g->nx; ++i) { Gv[IX(g, i, j, 0)] = 0.5 * (ss[6][PX(g, i, j - 1)] + ss[6][PX(g, i, j)]); }
    }
    for (int j = 0; j < g->ny; ++j) {
        for (int i = 0; i < g->nx; ++i) {
            Gt[IX(g, i, j, 0)] = -qs * ss[10][PX(g, i, j)];
            Gk[IX(g, i, j, 0)] = 0;
        }
    }
}

/* apply_wall_k (SurfaceLayer.cpp:452-481): R_k of the first cells
 * a (k - k_w), a = max(u*, 0.01)/d0, replacing the row (dirichlet) or added. */
void og_apply_wall_k(const og_grid* g, const gb_bc* bc, const double* const* ss, const double* tke, double* Rk)
{
    const int dirichlet = bc->surface_wall_k == GB_WALL_K_DIRICHLET;
    for (int j = 0; j < g->ny; ++j) {
        for (int i = 0; i < g->nx; ++i) {
            const int64_t p = PX(g, i, j), o = IX(g, i, j, 0);
            const double r = fmax(ss[0][p], 0.01) / ss[3][p] * (tke[o] - ss[9][p]);
            if (dirichlet) { Rk[o] = r; } else { Rk[o] += r; }
        }
    }
}

/* apply_wall_to_implicit (SurfaceLayer.cpp:483-518): the ground neighbour's
 * weight leaves the first cells' rows; u and v add the wall stress's Picard
 * coefficient drag dzeta^-1 / J (the face's J the mean of the two cells). */
void og_apply_wall_to_implicit(const og_grid* g, const double* const* ss, int loc, const double* J, double* A)
{
    const int64_t cs = VOL(g);
    const double dzinv = 1.0 / g->dzeta;
    const int nxl = g->nx + nodal(loc, 0), nyl = g->ny + nodal(loc, 1);
    for (int j = 0; j < nyl; ++j) {
        for (int i = 0; i < nxl; ++i) {
            const int64_t o = IX(g, i, j, 0);
            A[COEF_P * cs + o] -= A[COEF_ZM * cs + o];
            A[COEF_ZM * cs + o] = 0;
            if (loc == XF) {
                A[COEF_P * cs + o] += 0.5 * (ss[8][PX(g, i - 1, j)] + ss[8][PX(g, i, j)]) * dzinv
                                      / og_interp(g, J, CC, XF, i, j, 0);
            } else if (loc == YF) {
                A[COEF_P * cs + o] += 0.5 * (ss[8][PX(g, i, j - 1)] + ss[8][PX(g, i, j)]) * dzinv
                                      / og_interp(g, J, CC, YF, i, j, 0);
            }
        }
    }
}

/* apply_wall_k_to_implicit (SurfaceLayer.cpp:520-569): the first cells'
 * k rows: the diagonal a alone (dirichlet) or a added (source). */
void og_apply_wall_k_to_implicit(const og_grid* g, const gb_bc* bc, const double* const* ss, double* A)
{
    const int64_t cs = VOL(g);
    const int dirichlet = bc->surface_wall_k == GB_WALL_K_DIRICHLET;
    for (int j = 0; j < g->ny; ++j) {
        for (int i = 0; i < g->nx; ++i) {
            const int64_t p = PX(g, i, j), o = IX(g, i, j, 0);
            const double a = fmax(ss[0][p], 0.01) / ss[3][p];
            if (dirichlet) {
                for (int n = 0; n < N_COEFS; ++n) { A[n * cs + o] = 0; }
                A[COEF_P * cs + o] = a;
            } else {
                A[COEF_P * cs + o] += a;
            }
        }
    }
}
