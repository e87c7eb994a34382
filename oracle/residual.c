/*
 * ORACLE -- test infrastructure, not product code.
 *
 * FP64 restatement of the control-volume stencils of the reference's SIMPLEC
 * residual on the terrain-following C-grid:
 *   - staggered interpolation, derivatives, metrics, physical gradients
 *     (Source/Stencil_K.H:18-129);
 *   - C-grid kinematics: Omega, transport fluxes, divergence, pressure
 *     gradient (Source/MassFlux.cpp:29-179, Source/MassFlux_K.H);
 *   - MUSCL convection with the van Leer / van Albada / upwind limiters, the
 *     bounded form (Source/Convection.cpp:17-144, Source/Limiter_K.H:23-69);
 *   - control-volume flux divergence (Source/CVFluxes.cpp:16-80);
 *   - scalar and full-stress momentum diffusion with the cross-metric terms
 *     and the arithmetic or logarithmic face mean (Source/Diffusion.cpp:10-127,
 *     Source/Diffusion_K.H:35-98);
 *   - the first-order implicit operator A1 (Source/ImplicitOperator.cpp:13-121);
 *   - the local pseudo-time step and its face means (Source/PseudoTime.cpp:12-51,
 *     Source/Predictor.cpp:30-77).
 * Location types are the reference's bit masks (bit d: nodal in d).
 */
#include "og.h"

enum { CC = 0, XF = 1, YF = 2, ZF = 4, NODE = 7 };
enum { LIM_VAN_LEER = 0, LIM_VAN_ALBADA = 1, LIM_UPWIND = 2 };

static inline int lo_off(int tq, int ts, int d) { return (nodal(tq, d) == nodal(ts, d) || nodal(tq, d)) ? 0 : -1; }
static inline int npts(int tq, int ts, int d) { return (nodal(tq, d) == nodal(ts, d)) ? 1 : 2; }
static inline int flux_lo(int ts, int d) { return nodal(ts, d) ? -1 : 0; }

/* Stencil_K.H:67-74 interp<TQ, TS>. */
double og_interp(const og_grid* g, const double* q, int tq, int ts, int i, int j, int k)
{
    const int lx = lo_off(tq, ts, 0), ly = lo_off(tq, ts, 1), lz = lo_off(tq, ts, 2);
    const int nx = npts(tq, ts, 0), ny = npts(tq, ts, 1), nz = npts(tq, ts, 2);
    double s = 0;
    for (int c = 0; c < nz; ++c) {
        for (int b = 0; b < ny; ++b) {
            for (int a = 0; a < nx; ++a) { s += q[IX(g, i + lx + a, j + ly + b, k + lz + c)]; }
        }
    }
    return s * (1.0 / (double)(nx * ny * nz));
}

/* Stencil_K.H:76-92 deriv<TQ, TS, M> (per unit index). */
static double deriv(const og_grid* g, const double* q, int tq, int ts, int m, int i, int j, int k)
{
    const int same = nodal(tq, m) == nodal(ts, m);
    const int m0 = same ? -1 : lo_off(tq, ts, m);
    const int m1 = same ? 1 : m0 + 1;
    const double w = same ? 0.5 : 1.0;
    const int ex = (m == 0), ey = (m == 1), ez = (m == 2);
    const int lx = (m == 0) ? 0 : lo_off(tq, ts, 0), ly = (m == 1) ? 0 : lo_off(tq, ts, 1), lz = (m == 2) ? 0 : lo_off(tq, ts, 2);
    const int nx = (m == 0) ? 1 : npts(tq, ts, 0), ny = (m == 1) ? 1 : npts(tq, ts, 1), nz = (m == 2) ? 1 : npts(tq, ts, 2);
    double s = 0;
    for (int c = 0; c < nz; ++c) {
        for (int b = 0; b < ny; ++b) {
            for (int a = 0; a < nx; ++a) {
                const int ii = i + lx + a, jj = j + ly + b, kk = k + lz + c;
                s += q[IX(g, ii + m1 * ex, jj + m1 * ey, kk + m1 * ez)] - q[IX(g, ii + m0 * ex, jj + m0 * ey, kk + m0 * ez)];
            }
        }
    }
    return w * (s * (1.0 / (double)(nx * ny * nz)));
}

typedef struct { double zx, zy, zz; } metric_t;

/* Stencil_K.H:103-110 metric_at<TS>. */
static metric_t metric_at(const og_grid* g, const double* z, int ts, int i, int j, int k)
{
    metric_t m;
    m.zx = deriv(g, z, NODE, ts, 0, i, j, k) * (1.0 / g->dx);
    m.zy = deriv(g, z, NODE, ts, 1, i, j, k) * (1.0 / g->dy);
    m.zz = deriv(g, z, NODE, ts, 2, i, j, k) * (1.0 / g->dzeta);
    return m;
}

/* Stencil_K.H:115-124 grad_at<TQ, TS>. */
static void grad_at(const og_grid* g, const double* q, int tq, int ts, int i, int j, int k, metric_t m, double out[3])
{
    const double qx = deriv(g, q, tq, ts, 0, i, j, k) * (1.0 / g->dx);
    const double qy = deriv(g, q, tq, ts, 1, i, j, k) * (1.0 / g->dy);
    const double qz = deriv(g, q, tq, ts, 2, i, j, k) * (1.0 / g->dzeta) / m.zz;
    out[0] = qx - m.zx * qz;
    out[1] = qy - m.zy * qz;
    out[2] = qz;
}

/* The stencil helpers for the closure and the wall model (turbulence.c). */
double og_deriv(const og_grid* g, const double* q, int tq, int ts, int m, int i, int j, int k)
{
    return deriv(g, q, tq, ts, m, i, j, k);
}

/* grad_at<TQ, TS> with metric_at<TS> at (i, j, k). */
void og_grad_at(const og_grid* g, const double* q, int tq, int ts, const double* z, int i, int j, int k, double out[3])
{
    grad_at(g, q, tq, ts, i, j, k, metric_at(g, z, ts, i, j, k), out);
}

/* ------------------------------------------------------------------ */
/* mass flux                                                           */
/* ------------------------------------------------------------------ */

static inline double slope_x(const og_grid* g, const double* z, int i, int j, int k)
{
    return deriv(g, z, NODE, ZF, 0, i, j, k) * (1.0 / g->dx);
}
static inline double slope_y(const og_grid* g, const double* z, int i, int j, int k)
{
    return deriv(g, z, NODE, ZF, 1, i, j, k) * (1.0 / g->dy);
}

/* MassFlux.cpp:51-74 omega_from_w on the z-faces grown by ngrow (0 or 1). */
void og_omega_from_w(const og_grid* g, const double* u, const double* v, const double* w, const double* z, double* om,
                     int ngrow)
{
    for (int k = -ngrow; k <= g->nz + ngrow; ++k) {
        for (int j = -ngrow; j < g->ny + ngrow; ++j) {
            for (int i = -ngrow; i < g->nx + ngrow; ++i) {
                om[IX(g, i, j, k)] = w[IX(g, i, j, k)] - slope_x(g, z, i, j, k) * og_interp(g, u, XF, ZF, i, j, k)
                                   - slope_y(g, z, i, j, k) * og_interp(g, v, YF, ZF, i, j, k);
            }
        }
    }
}

/* MassFlux.cpp:76-99 w_from_omega on the valid z-faces. */
void og_w_from_omega(const og_grid* g, const double* u, const double* v, const double* om, const double* z, double* w)
{
    for (int k = 0; k <= g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                w[IX(g, i, j, k)] = om[IX(g, i, j, k)] + slope_x(g, z, i, j, k) * og_interp(g, u, XF, ZF, i, j, k)
                                  + slope_y(g, z, i, j, k) * og_interp(g, v, YF, ZF, i, j, k);
            }
        }
    }
}

/* MassFlux_K.H no_flux_w. */
double og_no_flux_w(const og_grid* g, const double* z, const double* u, const double* v, int i, int j, int k)
{
    return slope_x(g, z, i, j, k) * og_interp(g, u, XF, ZF, i, j, k) + slope_y(g, z, i, j, k) * og_interp(g, v, YF, ZF, i, j, k);
}

/* MassFlux.cpp:101-127 transport_fluxes: a_x u, a_y v, Omega on the valid
 * faces and one ghost face. */
void og_transport_fluxes(const og_grid* g, const double* u, const double* v, const double* w, const double* z,
                         const double* ax, const double* ay, double* F0, double* F1, double* F2)
{
    for (int k = -1; k <= g->nz; ++k) {
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx + 1; ++i) { F0[IX(g, i, j, k)] = ax[IX(g, i, j, k)] * u[IX(g, i, j, k)]; }
        }
        for (int j = -1; j <= g->ny + 1; ++j) {
            for (int i = -1; i <= g->nx; ++i) { F1[IX(g, i, j, k)] = ay[IX(g, i, j, k)] * v[IX(g, i, j, k)]; }
        }
    }
    og_omega_from_w(g, u, v, w, z, F2, 1);
}

void og_face_divergence(const og_grid* g, const double* ax, const double* ay, const double* az, const double* J,
                        const double* fx, const double* fy, const double* fz, double* div);

/* MassFlux.cpp:129-136 velocity_divergence. */
void og_velocity_divergence(const og_grid* g, const double* u, const double* v, const double* w, const double* z,
                            const double* ax, const double* ay, const double* az, const double* J, double* div)
{
    double* om = (double*)calloc(VOL(g), sizeof(double));
    og_omega_from_w(g, u, v, w, z, om, 0);
    og_face_divergence(g, ax, ay, az, J, u, v, om, div);
    free(om);
}

/* MassFlux.cpp:29-39 slope_dp, one-sided at the ground. */
static double slope_dp(const og_grid* g, const double* z, const double* p, int D, int i, int j, int k)
{
    const double s = (D == 0) ? slope_x(g, z, i, j, k) : slope_y(g, z, i, j, k);
    const double dp = (k == 0) ? 3.0 * p[IX(g, i, j, k + 1)] - 2.0 * p[IX(g, i, j, k)] - p[IX(g, i, j, k + 2)]
                               : p[IX(g, i, j, k)] - p[IX(g, i, j, k - 1)];
    return s * dp * (1.0 / g->dzeta);
}

/* MassFlux.cpp:138-179 pressure_gradient on the valid faces. */
void og_pressure_gradient(const og_grid* g, const double* p, const double* z, const double* J, const double* ax,
                          const double* ay, double* gx, double* gy, double* gz)
{
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy, dzinv = 1.0 / g->dzeta;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i <= g->nx; ++i) {
                const double cross = 0.25 * ((slope_dp(g, z, p, 0, i - 1, j, k) + slope_dp(g, z, p, 0, i, j, k))
                                             + (slope_dp(g, z, p, 0, i - 1, j, k + 1) + slope_dp(g, z, p, 0, i, j, k + 1)));
                gx[IX(g, i, j, k)] = (ax[IX(g, i, j, k)] * (p[IX(g, i, j, k)] - p[IX(g, i - 1, j, k)]) * dxinv - cross)
                                   / og_interp(g, J, CC, XF, i, j, k);
            }
        }
        for (int j = 0; j <= g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const double cross = 0.25 * ((slope_dp(g, z, p, 1, i, j - 1, k) + slope_dp(g, z, p, 1, i, j, k))
                                             + (slope_dp(g, z, p, 1, i, j - 1, k + 1) + slope_dp(g, z, p, 1, i, j, k + 1)));
                gy[IX(g, i, j, k)] = (ay[IX(g, i, j, k)] * (p[IX(g, i, j, k)] - p[IX(g, i, j - 1, k)]) * dyinv - cross)
                                   / og_interp(g, J, CC, YF, i, j, k);
            }
        }
    }
    for (int k = 0; k <= g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                gz[IX(g, i, j, k)] = (p[IX(g, i, j, k)] - p[IX(g, i, j, k - 1)]) * dzinv / og_interp(g, J, CC, ZF, i, j, k);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* control volumes                                                     */
/* ------------------------------------------------------------------ */

/* CVFluxes.cpp:52-66 cv_flux_box along d for a field at t: [lo, hi] in d
 * (the other directions span the field's valid points). */
static void cv_range(const og_grid* g, int t, int d, int* lo, int* hi)
{
    const int n = (d == 0) ? g->nx : (d == 1) ? g->ny : g->nz;
    if (nodal(t, d)) { *lo = -1; *hi = n; } else { *lo = 0; *hi = n; }
}

static void valid_range(const og_grid* g, int t, int d, int* lo, int* hi)
{
    const int n = (d == 0) ? g->nx : (d == 1) ? g->ny : g->nz;
    *lo = 0;
    *hi = n - 1 + nodal(t, d);
}

/* The box of the fluxes of a field at t along D: cv_range in D, valid elsewhere. */
static void flux_box(const og_grid* g, int t, int D, int lo[3], int hi[3])
{
    for (int d = 0; d < 3; ++d) {
        if (d == D) { cv_range(g, t, d, &lo[d], &hi[d]); } else { valid_range(g, t, d, &lo[d], &hi[d]); }
    }
}

/* CVFluxes.cpp:16-39 divergence<T>. */
void og_flux_divergence(const og_grid* g, int t, const double* gx, const double* gy, const double* gz, const double* J,
                        double* out)
{
    const int lx = flux_lo(t, 0), ly = flux_lo(t, 1), lz = flux_lo(t, 2);
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy, dzinv = 1.0 / g->dzeta;
    for (int k = 0; k < g->nz + nodal(t, 2); ++k) {
        for (int j = 0; j < g->ny + nodal(t, 1); ++j) {
            for (int i = 0; i < g->nx + nodal(t, 0); ++i) {
                out[IX(g, i, j, k)] = ((gx[IX(g, i + lx + 1, j, k)] - gx[IX(g, i + lx, j, k)]) * dxinv
                                       + (gy[IX(g, i, j + ly + 1, k)] - gy[IX(g, i, j + ly, k)]) * dyinv
                                       + (gz[IX(g, i, j, k + lz + 1)] - gz[IX(g, i, j, k + lz)]) * dzinv)
                                    / og_interp(g, J, CC, t, i, j, k);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* convection                                                          */
/* ------------------------------------------------------------------ */

/* Limiter_K.H:23-47. */
static double limited_slope(int lim, double a, double b, double eps2)
{
    if (lim == LIM_VAN_LEER) {
        const double ab = a * b;
        return (ab > 0) ? 2.0 * ab / (a + b) : 0.0;
    }
    if (lim == LIM_VAN_ALBADA) { return ((b * b + eps2) * a + (a * a + eps2) * b) / (a * a + b * b + 2.0 * eps2); }
    return 0.0;
}

/* Limiter_K.H:52-69 muscl_face. */
static double muscl_face(int lim, double tr, double qm, double q0, double q1, double qp, double eps2)
{
    if (lim == LIM_UPWIND) { return (tr >= 0) ? q0 : q1; }
    return (tr >= 0) ? q0 + 0.5 * limited_slope(lim, q0 - qm, q1 - q0, eps2) : q1 - 0.5 * limited_slope(lim, q1 - q0, qp - q1, eps2);
}

/* Convection.cpp:17-43 flux_kernel<T, D, L> into G (on the flux box). */
static void conv_fluxes(const og_grid* g, int t, int D, const double* q, const double* F, int lim, double eps2, double* G)
{
    const int S = t ^ (1 << D);
    const int TF = 1 << D;
    const int l = lo_off(t, S, D);
    const int ex = (D == 0), ey = (D == 1), ez = (D == 2);
    int lo[3], hi[3];
    flux_box(g, t, D, lo, hi);
    for (int k = lo[2]; k <= hi[2]; ++k) {
        for (int j = lo[1]; j <= hi[1]; ++j) {
            for (int i = lo[0]; i <= hi[0]; ++i) {
                const double tr = og_interp(g, F, TF, S, i, j, k);
                const int i0 = i + l * ex, j0 = j + l * ey, k0 = k + l * ez;
                G[IX(g, i, j, k)] = tr * muscl_face(lim, tr, q[IX(g, i0 - ex, j0 - ey, k0 - ez)], q[IX(g, i0, j0, k0)],
                                                    q[IX(g, i0 + ex, j0 + ey, k0 + ez)],
                                                    q[IX(g, i0 + 2 * ex, j0 + 2 * ey, k0 + 2 * ez)], eps2);
            }
        }
    }
}

/* Convection.cpp:137-144 convection = flux divergence of the MUSCL fluxes,
 * and in the bounded form minus q times the transport divergence (:65-90). */
void og_convection(const og_grid* g, int t, const double* q, const double* F0, const double* F1, const double* F2,
                   const double* J, int lim, double eps, int bounded, double* out)
{
    const int64_t vol = VOL(g);
    double* G[3];
    const double* F[3] = {F0, F1, F2};
    const double eps2 = eps * eps;
    for (int d = 0; d < 3; ++d) {
        G[d] = (double*)calloc(vol, sizeof(double));
        conv_fluxes(g, t, d, q, F[d], lim, eps2, G[d]);
    }
    og_flux_divergence(g, t, G[0], G[1], G[2], J, out);
    if (bounded) {
        const int SX = t ^ XF, SY = t ^ YF, SZ = t ^ ZF;
        const int lx = flux_lo(t, 0), ly = flux_lo(t, 1), lz = flux_lo(t, 2);
        const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy, dzinv = 1.0 / g->dzeta;
        for (int k = 0; k < g->nz + nodal(t, 2); ++k) {
            for (int j = 0; j < g->ny + nodal(t, 1); ++j) {
                for (int i = 0; i < g->nx + nodal(t, 0); ++i) {
                    const double div = (og_interp(g, F0, XF, SX, i + lx + 1, j, k) - og_interp(g, F0, XF, SX, i + lx, j, k)) * dxinv
                                     + (og_interp(g, F1, YF, SY, i, j + ly + 1, k) - og_interp(g, F1, YF, SY, i, j + ly, k)) * dyinv
                                     + (og_interp(g, F2, ZF, SZ, i, j, k + lz + 1) - og_interp(g, F2, ZF, SZ, i, j, k + lz)) * dzinv;
                    out[IX(g, i, j, k)] -= q[IX(g, i, j, k)] * div / og_interp(g, J, CC, t, i, j, k);
                }
            }
        }
    }
    for (int d = 0; d < 3; ++d) { free(G[d]); }
}

/* ------------------------------------------------------------------ */
/* diffusion                                                           */
/* ------------------------------------------------------------------ */

/* Diffusion_K.H:35-47 log_mean. */
static double log_mean(double a, double b)
{
    const double tiny = 2.2250738585072014e-308;
    const double sum = a + b;
    const double x = (a - b) / (sum + tiny);
    const double s = (fabs(x) < 0.01) ? 1.0 : 0.0;
    const double x2 = x * x;
    const double series = 0.5 * sum * (1.0 - x2 * (1.0 / 3 + x2 * (4.0 / 45 + x2 * (44.0 / 945))));
    const double direct = (a - b) / (log(a + tiny) - log(b + tiny) + s);
    return (1.0 - s) * direct + s * series;
}

/* Diffusion_K.H:51-64 face_gamma<S>. */
static double face_gamma(const og_grid* g, const double* gm, int S, int i, int j, int k, int logz)
{
    if (!logz || !nodal(S, 2)) { return og_interp(g, gm, CC, S, i, j, k); }
    const int lx = lo_off(CC, S, 0), ly = lo_off(CC, S, 1);
    const int nx = npts(CC, S, 0), ny = npts(CC, S, 1);
    double sum = 0;
    for (int b = 0; b < ny; ++b) {
        for (int a = 0; a < nx; ++a) { sum += log_mean(gm[IX(g, i + lx + a, j + ly + b, k - 1)], gm[IX(g, i + lx + a, j + ly + b, k)]); }
    }
    return sum * (1.0 / (double)(nx * ny));
}

/* Diffusion_K.H:68-79 area_dot<D>. */
static double area_dot(int D, metric_t m, const double v[3])
{
    if (D == 0) { return m.zz * v[0]; }
    if (D == 1) { return m.zz * v[1]; }
    return v[2] - m.zx * v[0] - m.zy * v[1];
}

/* Diffusion.cpp:10-29 scalar_kernel, all three directions. */
void og_scalar_diffusive_fluxes(const og_grid* g, const double* q, const double* gamma, const double* z, int logz,
                                double* G0, double* G1, double* G2)
{
    double* G[3] = {G0, G1, G2};
    for (int D = 0; D < 3; ++D) {
        const int S = 1 << D;
        int lo[3], hi[3];
        flux_box(g, CC, D, lo, hi);
        for (int k = lo[2]; k <= hi[2]; ++k) {
            for (int j = lo[1]; j <= hi[1]; ++j) {
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    const metric_t m = metric_at(g, z, S, i, j, k);
                    double gr[3];
                    grad_at(g, q, CC, S, i, j, k, m, gr);
                    G[D][IX(g, i, j, k)] = face_gamma(g, gamma, S, i, j, k, logz) * area_dot(D, m, gr);
                }
            }
        }
    }
}

/* Diffusion.cpp:31-57 momentum_kernel<C, D> for one component C, all D. */
void og_momentum_diffusive_fluxes(const og_grid* g, int C, const double* u, const double* v, const double* w,
                                  const double* nu, const double* z, int logz, double* G0, double* G1, double* G2)
{
    double* G[3] = {G0, G1, G2};
    const int T = 1 << C;
    for (int D = 0; D < 3; ++D) {
        const int S = T ^ (1 << D);
        int lo[3], hi[3];
        flux_box(g, T, D, lo, hi);
        for (int k = lo[2]; k <= hi[2]; ++k) {
            for (int j = lo[1]; j <= hi[1]; ++j) {
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    const metric_t m = metric_at(g, z, S, i, j, k);
                    double gu[3], gv[3], gw[3];
                    grad_at(g, u, XF, S, i, j, k, m, gu);
                    grad_at(g, v, YF, S, i, j, k, m, gv);
                    grad_at(g, w, ZF, S, i, j, k, m, gw);
                    const double* gc = (C == 0) ? gu : (C == 1) ? gv : gw;
                    const double tau[3] = {gc[0] + gu[C], gc[1] + gv[C], gc[2] + gw[C]};
                    G[D][IX(g, i, j, k)] = face_gamma(g, nu, S, i, j, k, logz) * area_dot(D, m, tau);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* implicit operator                                                   */
/* ------------------------------------------------------------------ */

/* ImplicitOperator.cpp:13-37 face_weight<T, C, D>. */
static double face_weight(const og_grid* g, int T, int C, int D, int side, int i, int j, int k, const double* f,
                          const double* gm, const double* z, int logz)
{
    const int S = T ^ (1 << D);
    const double dxinv[3] = {1.0 / g->dx, 1.0 / g->dy, 1.0 / g->dzeta};
    const metric_t m = metric_at(g, z, S, i, j, k);
    const double gs = face_gamma(g, gm, S, i, j, k, logz);
    const double tr = og_interp(g, f, 1 << D, S, i, j, k);
    double dif;
    if (D < 2) {
        const double own = (C == D) ? 2.0 : 1.0;
        dif = gs * m.zz * own * dxinv[D];
    } else {
        double nc2 = 0;
        if (C == 0) { nc2 = m.zx * m.zx; }
        if (C == 1) { nc2 = m.zy * m.zy; }
        if (C == 2) { nc2 = 1; }
        dif = gs * (1 + m.zx * m.zx + m.zy * m.zy + nc2) / m.zz * dxinv[2];
    }
    const double inflow = (side == 0) ? fmax(tr, 0.0) : fmax(-tr, 0.0);
    return (dif + inflow) * dxinv[D];
}

/* ImplicitOperator.cpp:39-74 coefficients<C> (C = -1: a scalar at cells). */
void og_implicit_coefficients(const og_grid* g, int C, const double* F0, const double* F1, const double* F2,
                              const double* gm, const double* z, const double* J, int logz, double* A)
{
    const int T = (C < 0) ? CC : (1 << C);
    const int lx = flux_lo(T, 0), ly = flux_lo(T, 1), lz = flux_lo(T, 2);
    const int64_t cs = VOL(g);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < g->nz + nodal(T, 2); ++k) {
        for (int j = 0; j < g->ny + nodal(T, 1); ++j) {
            for (int i = 0; i < g->nx + nodal(T, 0); ++i) {
                const double Jinv = 1.0 / og_interp(g, J, CC, T, i, j, k);
                const double xm = face_weight(g, T, C, 0, 0, i + lx, j, k, F0, gm, z, logz) * Jinv;
                const double xp = face_weight(g, T, C, 0, 1, i + lx + 1, j, k, F0, gm, z, logz) * Jinv;
                const double ym = face_weight(g, T, C, 1, 0, i, j + ly, k, F1, gm, z, logz) * Jinv;
                const double yp = face_weight(g, T, C, 1, 1, i, j + ly + 1, k, F1, gm, z, logz) * Jinv;
                const double zm = face_weight(g, T, C, 2, 0, i, j, k + lz, F2, gm, z, logz) * Jinv;
                const double zp = face_weight(g, T, C, 2, 1, i, j, k + lz + 1, F2, gm, z, logz) * Jinv;
                const int64_t o = IX(g, i, j, k);
                A[COEF_XM * cs + o] = xm;
                A[COEF_XP * cs + o] = xp;
                A[COEF_YM * cs + o] = ym;
                A[COEF_YP * cs + o] = yp;
                A[COEF_ZM * cs + o] = zm;
                A[COEF_ZP * cs + o] = zp;
                A[COEF_P * cs + o] = ((xm + xp) + (ym + yp)) + (zm + zp);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* pseudo-time step                                                    */
/* ------------------------------------------------------------------ */

/* PseudoTime.cpp:12-51 local_dtau (nu may be null). */
void og_local_dtau(const og_grid* g, const double* u, const double* v, const double* w, const double* z,
                   const double* J, const double* nu, double cfl, double* dtau)
{
    double* om = (double*)calloc(VOL(g), sizeof(double));
    og_omega_from_w(g, u, v, w, z, om, 0);
    const double dxinv = 1.0 / g->dx, dyinv = 1.0 / g->dy, dzinv = 1.0 / g->dzeta;
    const double diff_h = 2 * (dxinv * dxinv + dyinv * dyinv);
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const double uc = og_interp(g, u, XF, CC, i, j, k), vc = og_interp(g, v, YF, CC, i, j, k),
                             oc = og_interp(g, om, ZF, CC, i, j, k);
                double rate = fabs(uc) * dxinv + fabs(vc) * dyinv + fabs(oc) * dzinv / J[IX(g, i, j, k)];
                if (nu) { rate += nu[IX(g, i, j, k)] * diff_h; }
                dtau[IX(g, i, j, k)] = cfl / fmax(rate, 1.0e-12);
            }
        }
    }
    free(om);
}

/* Predictor.cpp:30-77 face_dtau: the mean of the two cells sharing a face
 * (periodic images; the one cell on a non-periodic face, the ground, the top). */
void og_face_dtau(const og_grid* g, double* dc, double* fx, double* fy, double* fz)
{
    og_fill_periodic(g, CC, dc, 1);
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i <= g->nx; ++i) {
                const int lo = (!g->periodic_x && i == 0), hi = (!g->periodic_x && i == g->nx);
                fx[IX(g, i, j, k)] = lo ? dc[IX(g, i, j, k)] : hi ? dc[IX(g, i - 1, j, k)]
                                                                  : 0.5 * (dc[IX(g, i - 1, j, k)] + dc[IX(g, i, j, k)]);
            }
        }
        for (int j = 0; j <= g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const int lo = (!g->periodic_y && j == 0), hi = (!g->periodic_y && j == g->ny);
                fy[IX(g, i, j, k)] = lo ? dc[IX(g, i, j, k)] : hi ? dc[IX(g, i, j - 1, k)]
                                                                  : 0.5 * (dc[IX(g, i, j - 1, k)] + dc[IX(g, i, j, k)]);
            }
        }
    }
    for (int k = 0; k <= g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const int lo = (k == 0), hi = (k == g->nz);
                fz[IX(g, i, j, k)] = lo ? dc[IX(g, i, j, k)] : hi ? dc[IX(g, i, j, k - 1)]
                                                                 : 0.5 * (dc[IX(g, i, j, k - 1)] + dc[IX(g, i, j, k)]);
            }
        }
    }
}
