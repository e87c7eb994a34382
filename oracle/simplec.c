/*
 * ORACLE -- test infrastructure, not product code.
 *
 * FP64 restatement of the reference's SIMPLEC outer iteration without a
 * closure and a wall model (given diffusivities):
 *   - boundary conditions: ghost fills, Dirichlet rows, implicit folds
 *     (Source/BoundaryConditions.cpp:37-66 rule_for, :418-546 fill_face /
 *     fill_gradient_z / fill_field, :597-663 fill_ghosts, :754-799
 *     fill_no_flux_w, :801-852 apply_rows, :854-883 dirichlet_rows,
 *     :885-941 apply_to_implicit) and the log-law inflow (Source/InflowProfile.H eval);
 *   - forcing (Source/Forcing.cpp: fill_theta_ref, subtract_buoyancy,
 *     subtract_coriolis, subtract_pressure_gradient, coriolis_parameter);
 *   - the residual (Source/Residual.cpp:159-256) and the implicit rows (:272-304);
 *   - the momentum predictor (Source/Predictor.cpp:129-405), the pressure
 *     correction (Source/Simplec.cpp:87-220), the scalar sweeps (:222-281),
 *     the stage iterate (:452-506) and its norms (:373-409).
 * The struct layouts are the C ABI's (include/gust_b200.h): a data format
 * shared by the checker and the product, not code.
 */
#include "og.h"

#include "../include/gust_b200.h"

enum { CC = 0, XF = 1, YF = 2, ZF = 4, NODE = 7 };
enum { R_EVEN = 0, R_ODD, R_VALUE, R_PROFILE, R_GRADIENT };
enum { F_U = 0, F_V, F_W, F_P, F_THETA, F_TKE };

/* residual.c, poisson.c */
double og_interp(const og_grid* g, const double* q, int tq, int ts, int i, int j, int k);
double og_no_flux_w(const og_grid* g, const double* z, const double* u, const double* v, int i, int j, int k);
void og_omega_from_w(const og_grid* g, const double* u, const double* v, const double* w, const double* z, double* om, int ngrow);
void og_w_from_omega(const og_grid* g, const double* u, const double* v, const double* om, const double* z, double* w);
void og_transport_fluxes(const og_grid* g, const double* u, const double* v, const double* w, const double* z,
                         const double* ax, const double* ay, double* F0, double* F1, double* F2);
void og_velocity_divergence(const og_grid* g, const double* u, const double* v, const double* w, const double* z,
                            const double* ax, const double* ay, const double* az, const double* J, double* div);
void og_pressure_gradient(const og_grid* g, const double* p, const double* z, const double* J, const double* ax,
                          const double* ay, double* gx, double* gy, double* gz);
void og_flux_divergence(const og_grid* g, int t, const double* gx, const double* gy, const double* gz, const double* J,
                        double* out);
void og_convection(const og_grid* g, int t, const double* q, const double* F0, const double* F1, const double* F2,
                   const double* J, int lim, double eps, int bounded, double* out);
void og_scalar_diffusive_fluxes(const og_grid* g, const double* q, const double* gamma, const double* z, int logz,
                                double* G0, double* G1, double* G2);
void og_momentum_diffusive_fluxes(const og_grid* g, int C, const double* u, const double* v, const double* w,
                                  const double* nu, const double* z, int logz, double* G0, double* G1, double* G2);
void og_implicit_coefficients(const og_grid* g, int C, const double* F0, const double* F1, const double* F2,
                              const double* gm, const double* z, const double* J, int logz, double* A);
void og_face_dtau(const og_grid* g, double* dc, double* fx, double* fy, double* fz);
double og_zline_jacobi(const og_grid* g, int loc, const double* A, const double* ap, const double* rhs, int sweeps,
                       double* delta);
double og_zline_lusgs(const og_grid* g, int loc, const double* A, const double* ap, const double* rhs, int sweeps,
                      int order, int alternate, double* delta);
void og_poisson_fluxes(const og_grid* g, const int* bc, const double* z, double* phi, const double* bx,
                       const double* by, const double* bz, double* fx, double* fy, double* fz);
typedef struct og_mg og_mg;
og_mg* og_mg_create(const og_grid* g, const int* bc, const double* z, const double* J, const double* AX,
                    const double* AY, const double* AZ, int max_levels, int min_coarse, int nu1, int nu2, int nu_coarse);
void og_mg_destroy(og_mg* mg);
void og_mg_set_cross(og_mg* mg, const double* az, const double* bz, const double* z_cross);
void og_poisson_cross_flux(const og_grid* g, const int* bc, const double* d, const double* z, const double* phi,
                           double* fz);
int og_poisson_solve(og_mg* mg, double* rhs, double* phi, double reltol, double abstol, int max_iter, int restart,
                     int precond, double* res);
void og_face_divergence(const og_grid* g, const double* ax, const double* ay, const double* az, const double* J,
                        const double* fx, const double* fy, const double* fz, double* div);

/* turbulence.c: the closure and the wall model */
void og_closure_evaluate(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const double* u, const double* v,
                         const double* w, const double* th, const double* tk, const double* z, const double* z0map,
                         double** out);
int og_surface_state(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const double* u, const double* v,
                     const double* w, const double* z, const double* z0map, double** ss);
void og_ground_gradients(const og_grid* g, const gb_bc* bc, const double* const* ss, const double* z0map, double** gg);
double og_ground_gradient_at(const og_grid* g, const double* gg, int t, int i, int j);
void og_set_ground_fluxes(const og_grid* g, const gb_bc* bc, const double* const* ss, double* Gu, double* Gv,
                          double* Gt, double* Gk);
void og_apply_wall_k(const og_grid* g, const gb_bc* bc, const double* const* ss, const double* tke, double* Rk);
void og_apply_wall_to_implicit(const og_grid* g, const double* const* ss, int loc, const double* J, double* A);
void og_apply_wall_k_to_implicit(const og_grid* g, const gb_bc* bc, const double* const* ss, double* A);

enum { N_CF = 10, N_SS = 11 };
enum { CF_NU = 0, CF_GTH, CF_GK, CF_NUT, CF_L, CF_RT, CF_PS, CF_PB, CF_EPS, CF_DSDK };

/* The closure's fields (N_CF volumes) and the surface state (N_SS planes) an
 * iteration evaluates once and its parts read (null: none). */
typedef struct og_turb {
    double* const* cf;
    double* const* ss;
} og_turb;

static double* zalloc(const og_grid* g) { return (double*)calloc(VOL(g), sizeof(double)); }
static double* palloc(const og_grid* g) { return (double*)calloc((size_t)(g->sy * (g->ny + 1 + 2 * g->ng)), sizeof(double)); }
static int ext(const og_grid* g, int t, int d) { return ((d == 0) ? g->nx : (d == 1) ? g->ny : g->nz) + nodal(t, d); }
static int is_per(const og_grid* g, int d) { return d == 0 ? g->periodic_x : d == 1 ? g->periodic_y : 0; }

/* ------------------------------------------------------------------ */
/* inflow profile and heights                                          */
/* ------------------------------------------------------------------ */

/* NodeZ (Source/Heights_K.H:22-35): lateral clamp to the stored nodes, linear
 * vertical extrapolation beyond them (stored: one ghost layer). */
static double node_z(const og_grid* g, const double* z, int i, int j, int k)
{
    const int lo = -1, hix = g->nx + 1, hiy = g->ny + 1, hiz = g->nz + 1;
    i = i < lo ? lo : (i > hix ? hix : i);
    j = j < lo ? lo : (j > hiy ? hiy : j);
    if (k < lo) { return z[IX(g, i, j, lo)] + (lo - k) * (z[IX(g, i, j, lo)] - z[IX(g, i, j, lo + 1)]); }
    if (k > hiz) { return z[IX(g, i, j, hiz)] + (k - hiz) * (z[IX(g, i, j, hiz)] - z[IX(g, i, j, hiz - 1)]); }
    return z[IX(g, i, j, k)];
}

/* Heights_K.H:40-56 height_above_ground<T>. */
static double height_above_ground(const og_grid* g, const double* z, int t, int i, int j, int k)
{
    const int nx = nodal(t, 0) ? 1 : 2, ny = nodal(t, 1) ? 1 : 2, nz = nodal(t, 2) ? 1 : 2;
    double zp = 0, zg = 0;
    for (int a = 0; a < nx; ++a) {
        for (int b = 0; b < ny; ++b) {
            zg += node_z(g, z, i + a, j + b, 0);
            for (int c = 0; c < nz; ++c) { zp += node_z(g, z, i + a, j + b, k + c); }
        }
    }
    return zp / (nx * ny * nz) - zg / (nx * ny);
}

/* Heights_K.H:60-71 point_z<T>. */
static double point_z(const og_grid* g, const double* z, int t, int i, int j, int k)
{
    const int nx = nodal(t, 0) ? 1 : 2, ny = nodal(t, 1) ? 1 : 2, nz = nodal(t, 2) ? 1 : 2;
    double zp = 0;
    for (int a = 0; a < nx; ++a) {
        for (int b = 0; b < ny; ++b) {
            for (int c = 0; c < nz; ++c) { zp += node_z(g, z, i + a, j + b, k + c); }
        }
    }
    return zp / (nx * ny * nz);
}

/* InflowProfile.H table_interp. */
static double table_interp(const double* x, const double* y, int n, double xq)
{
    if (n == 1 || xq <= x[0]) { return y[0]; }
    if (xq >= x[n - 1]) { return y[n - 1]; }
    int m = 1;
    while (m < n - 1 && !(xq < x[m])) { ++m; }
    const double w = (xq - x[m - 1]) / (x[m] - x[m - 1]);
    return y[m - 1] + w * (y[m] - y[m - 1]);
}

/* InflowProfile::View::eval, log law (Source/InflowProfile.H). */
static double profile_value(const gb_bc* bc, int f, double z)
{
    z = fmax(z, 0.0);
    const double c = 1.0 / (1.0 + bc->kappa * (z + bc->inflow_z0) * bc->inflow_inv_lmax);
    const double S = bc->inflow_ustar / bc->kappa * log((z + bc->inflow_z0) / bc->inflow_z0);
    const double ustar_l = bc->inflow_ustar * c;
    const double pi = 3.14159265358979323846;
    const double dir = bc->inflow_direction * pi / 180.0;
    switch (f) {
    case F_U: return S * cos(dir);
    case F_V: return S * sin(dir);
    case F_THETA: return table_interp(bc->theta_ref_z, bc->theta_ref_theta, bc->theta_ref_n, z);
    case F_TKE: return ustar_l * ustar_l / (bc->Cmu0 * bc->Cmu0);
    default: return 0;
    }
}

/* ------------------------------------------------------------------ */
/* ghost fills                                                         */
/* ------------------------------------------------------------------ */

/* BoundaryConditions.cpp:37-66 rule_for. */
static int rule_for(int f, int t, int d, int lo)
{
    const int normal_vel = (f == F_U && d == 0) || (f == F_V && d == 1) || (f == F_W && d == 2);
    const int vel = (f == F_U || f == F_V || f == F_W);
    switch (t) {
    case GB_FACE_INFLOW: return (f == F_P) ? R_EVEN : R_PROFILE;
    case GB_FACE_OUTFLOW: return (f == F_P) ? R_ODD : R_EVEN;
    case GB_FACE_SLIP_WALL:
        if (normal_vel) { return R_VALUE; }
        return (f == F_THETA && d == 2 && !lo) ? R_GRADIENT : R_EVEN;
    case GB_FACE_NO_SLIP_WALL: return vel ? R_VALUE : R_EVEN;
    case GB_FACE_SURFACE_LAYER:
        if (normal_vel) { return R_VALUE; }
        return (vel || f == F_THETA) ? R_GRADIENT : R_EVEN;
    default: return R_EVEN;
    }
}

/* The ghost slab's extent in direction e for a fill along d (ghost_slab,
 * BoundaryConditions.cpp:86-105): fully grown over e < d, over e > d only
 * across periodic faces. */
static void slab_range(const og_grid* g, int t, int d, int e, int* lo, int* hi)
{
    const int ng = g->ng;
    if (e < d || is_per(g, e)) {
        *lo = -ng;
        *hi = ext(g, t, e) - 1 + ng;
    } else {
        *lo = 0;
        *hi = ext(g, t, e) - 1;
    }
}

/* FillBoundary of the lateral ghosts (two layers) for the periodic
 * directions: x over the valid y and z, then y over the x ghosts. */
static void fill_periodic2(const og_grid* g, int t, double* f)
{
    const int nvx = ext(g, t, 0), nvy = ext(g, t, 1), nvz = ext(g, t, 2);
    if (g->periodic_x) {
        for (int k = 0; k < nvz; ++k) {
            for (int j = 0; j < nvy; ++j) {
                for (int l = 1; l <= g->ng; ++l) {
                    f[IX(g, -l, j, k)] = f[IX(g, g->nx - l, j, k)];
                    f[IX(g, nvx - 1 + l, j, k)] = f[IX(g, nvx - 1 + l - g->nx, j, k)];
                }
            }
        }
    }
    if (g->periodic_y) {
        const int ilo = g->periodic_x ? -g->ng : 0, ihi = g->periodic_x ? nvx - 1 + g->ng : nvx - 1;
        for (int k = 0; k < nvz; ++k) {
            for (int i = ilo; i <= ihi; ++i) {
                for (int l = 1; l <= g->ng; ++l) {
                    f[IX(g, i, -l, k)] = f[IX(g, i, g->ny - l, k)];
                    f[IX(g, i, nvy - 1 + l, k)] = f[IX(g, i, nvy - 1 + l - g->ny, k)];
                }
            }
        }
    }
}

/* fill_face<T> (BoundaryConditions.cpp:418-472) for one face and rule. */
static void fill_face(const og_grid* g, int t, double* a, const double* z, int d, int lo, int f, int rule, double V,
                      const gb_bc* bc)
{
    const int nd = (d == 0) ? g->nx : (d == 1) ? g->ny : g->nz;
    const int nod = nodal(t, d);
    const int edge = lo ? 0 : (nod ? nd : nd - 1);
    const int sgn = (rule == R_ODD) ? -1 : 1;
    int rlo[3], rhi[3];
    for (int e = 0; e < 3; ++e) { slab_range(g, t, d, e, &rlo[e], &rhi[e]); }
    /* the face point of a normal velocity takes the value itself */
    if (nod && (rule == R_VALUE || rule == R_PROFILE)) {
        rlo[d] = rhi[d] = edge;
        for (int k = rlo[2]; k <= rhi[2]; ++k) {
            for (int j = rlo[1]; j <= rhi[1]; ++j) {
                for (int i = rlo[0]; i <= rhi[0]; ++i) {
                    a[IX(g, i, j, k)] = (rule == R_PROFILE) ? profile_value(bc, f, height_above_ground(g, z, t, i, j, k)) : V;
                }
            }
        }
    }
    const int mirror = nod ? 2 * edge : (lo ? 2 * edge - 1 : 2 * edge + 1);
    for (int layer = 1; layer <= g->ng; ++layer) {
        const int gidx = lo ? edge - layer : edge + layer;
        rlo[d] = rhi[d] = gidx;
        const int m = mirror - gidx;
        for (int k = rlo[2]; k <= rhi[2]; ++k) {
            for (int j = rlo[1]; j <= rhi[1]; ++j) {
                for (int i = rlo[0]; i <= rhi[0]; ++i) {
                    const int si = (d == 0) ? m : i, sj = (d == 1) ? m : j, sk = (d == 2) ? m : k;
                    double* dst = &a[IX(g, i, j, k)];
                    if (rule == R_PROFILE) {
                        *dst = profile_value(bc, f, height_above_ground(g, z, t, i, j, k));
                    } else if (rule == R_VALUE) {
                        *dst = 2 * V - a[IX(g, si, sj, sk)];
                    } else {
                        *dst = sgn * a[IX(g, si, sj, sk)];
                    }
                }
            }
        }
    }
}

/* fill_gradient_z<T> (BoundaryConditions.cpp:474-517): a constant gradient
 * G, or per column from gg (the wall law's, og_ground_gradient_at). */
static void fill_gradient_z(const og_grid* g, int t, double* a, const double* z, int lo, double Gc, const double* gg)
{
    const int edge = lo ? 0 : g->nz - 1 + nodal(t, 2);
    const int c1 = lo ? edge + 1 : edge - 1;
    const int g1 = lo ? edge - 1 : edge + 1, g2 = lo ? edge - 2 : edge + 2;
    int rlo[3], rhi[3];
    for (int e = 0; e < 2; ++e) { slab_range(g, t, 2, e, &rlo[e], &rhi[e]); }
    for (int j = rlo[1]; j <= rhi[1]; ++j) {
        for (int i = rlo[0]; i <= rhi[0]; ++i) {
            const double G = gg ? og_ground_gradient_at(g, gg, t, i, j) : Gc;
            const double zc1 = point_z(g, z, t, i, j, c1), zg1 = point_z(g, z, t, i, j, g1), zg2 = point_z(g, z, t, i, j, g2);
            a[IX(g, i, j, g1)] = a[IX(g, i, j, c1)] + (zg1 - zc1) * G;
            a[IX(g, i, j, g2)] = a[IX(g, i, j, g1)] + (zg2 - zg1) * G;
        }
    }
}

static void fill_field(const og_grid* g, int t, double* q, int f, int d, const gb_bc* bc, const double* z,
                       double* const* gg)
{
    for (int lo = 1; lo >= 0; --lo) {
        const int face = d + (lo ? 0 : 3);
        const int ft = bc->face[face];
        const int rule = rule_for(f, ft, d, lo);
        double value = 0;
        if (ft == GB_FACE_NO_SLIP_WALL && f <= F_W) { value = bc->wall_velocity[face][f]; }
        if (rule == R_GRADIENT) {
            if (ft == GB_FACE_SURFACE_LAYER) {
                fill_gradient_z(g, t, q, z, lo, 0.0, gg[f == F_U ? 0 : f == F_V ? 1 : 2]);
            } else {
                fill_gradient_z(g, t, q, z, lo, bc->zhi_theta_grad, NULL);
            }
        } else {
            fill_face(g, t, q, z, d, lo, f, rule, value, bc);
        }
    }
}

static int dirichlet_normal(const gb_bc* bc, int face)
{
    const int t = bc->face[face];
    return t == GB_FACE_INFLOW || t == GB_FACE_SLIP_WALL || t == GB_FACE_NO_SLIP_WALL || t == GB_FACE_SURFACE_LAYER;
}

/* fill_no_flux_w (BoundaryConditions.cpp:754-799): the ground and top faces
 * of w take Omega = 0 with the two ghost layers mirrored about it. */
static void fill_no_flux_w(const og_grid* g, const gb_bc* bc, double* u, double* v, double* w, const double* z)
{
    for (int lo = 1; lo >= 0; --lo) {
        if (!dirichlet_normal(bc, lo ? 2 : 5)) { continue; }
        const int face = lo ? 0 : g->nz;
        const int sgn = lo ? -1 : 1;
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx; ++i) {
                const double V = og_no_flux_w(g, z, u, v, i, j, face);
                w[IX(g, i, j, face)] = V;
                for (int m = 1; m <= g->ng; ++m) { w[IX(g, i, j, face + sgn * m)] = 2 * V - w[IX(g, i, j, face - sgn * m)]; }
            }
        }
    }
    fill_periodic2(g, ZF, w);
}

/* BoundaryConditions::fill_ghosts (BoundaryConditions.cpp:597-663):
 * periodic images, then x, y and z faces for every field in order (u, v, w,
 * the no-flux w faces, p, theta, k), then the periodic images of the rows the
 * face fills rewrote (sync_ghost_copies). A surface_layer ground: the surface
 * state from the laterally filled state (into ss_out, N_SS planes, when
 * given) and the wall law's gradient for the ground fills of u, v, theta. */
static const gb_physics* default_buoyancy(void)
{
    static gb_physics ph;
    ph.gravity = 9.81;
    ph.theta0 = 300.0;
    return &ph;
}

void og_fill_ghosts2(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const double* z0map, double* u, double* v,
                     double* w, double* p, double* th, double* tk, const double* z, double** ss_out)
{
    double* f[6] = {u, v, w, p, th, tk};
    const int t[6] = {XF, YF, ZF, CC, CC, CC};
    const int wall = bc->face[2] == GB_FACE_SURFACE_LAYER;
    double* ssl[N_SS] = {0};
    double* gg[3] = {0};
    double* const* ss = ss_out;
    if (wall) {
        if (!ss_out) {
            for (int n = 0; n < N_SS; ++n) { ssl[n] = palloc(g); }
            ss = ssl;
        }
        for (int n = 0; n < 3; ++n) { gg[n] = palloc(g); }
    }
    for (int n = 0; n < 6; ++n) { fill_periodic2(g, t[n], f[n]); }
    for (int d = 0; d < 3; ++d) {
        if (d == 2 && wall) {
            og_surface_state(g, bc, ph ? ph : default_buoyancy(), u, v, w, z, z0map, (double**)ss);
            og_ground_gradients(g, bc, (const double* const*)ss, z0map, gg);
        }
        if (is_per(g, d)) { continue; }
        fill_field(g, XF, u, F_U, d, bc, z, gg);
        fill_field(g, YF, v, F_V, d, bc, z, gg);
        fill_field(g, ZF, w, F_W, d, bc, z, gg);
        if (d == 2) { fill_no_flux_w(g, bc, u, v, w, z); }
        fill_field(g, CC, p, F_P, d, bc, z, gg);
        fill_field(g, CC, th, F_THETA, d, bc, z, gg);
        fill_field(g, CC, tk, F_TKE, d, bc, z, gg);
    }
    for (int n = 0; n < 6; ++n) { fill_periodic2(g, t[n], f[n]); }
    for (int n = 0; n < N_SS; ++n) { free(ssl[n]); }
    for (int n = 0; n < 3; ++n) { free(gg[n]); }
}

void og_fill_ghosts(const og_grid* g, const gb_bc* bc, double* u, double* v, double* w, double* p, double* th,
                    double* tk, const double* z)
{
    og_fill_ghosts2(g, bc, NULL, NULL, u, v, w, p, th, tk, z, NULL);
}

/* apply_rows (BoundaryConditions.cpp:801-852): R = q - V on the Dirichlet
 * face points of the normal velocities. */
static void apply_rows(const og_grid* g, const gb_bc* bc, const double* u, const double* v, const double* w,
                       const double* z, double* Ru, double* Rv, double* Rw)
{
    const double* q[3] = {u, v, w};
    double* R[3] = {Ru, Rv, Rw};
    for (int d = 0; d < 3; ++d) {
        if (is_per(g, d)) { continue; }
        for (int lo = 1; lo >= 0; --lo) {
            const int fc = d + (lo ? 0 : 3);
            if (!dirichlet_normal(bc, fc)) { continue; }
            const int is_profile = bc->face[fc] == GB_FACE_INFLOW;
            const int t = 1 << d;
            const int face = lo ? 0 : ((d == 0) ? g->nx : (d == 1) ? g->ny : g->nz);
            int rlo[3], rhi[3];
            for (int e = 0; e < 3; ++e) { rlo[e] = 0; rhi[e] = ext(g, t, e) - 1; }
            rlo[d] = rhi[d] = face;
            for (int k = rlo[2]; k <= rhi[2]; ++k) {
                for (int j = rlo[1]; j <= rhi[1]; ++j) {
                    for (int i = rlo[0]; i <= rhi[0]; ++i) {
                        double V;
                        if (d < 2) {
                            V = is_profile ? profile_value(bc, d, height_above_ground(g, z, t, i, j, k)) : 0.0;
                        } else {
                            V = og_no_flux_w(g, z, u, v, i, j, k);
                        }
                        R[d][IX(g, i, j, k)] = q[d][IX(g, i, j, k)] - V;
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* damping (BoundaryConditions.cpp:945-1099)                            */
/* ------------------------------------------------------------------ */

static int damping_on(const gb_bc* bc) { return bc->rayleigh_zdamp > 0 || bc->sponge_width > 0; }

/* DampingCoef::rayleigh_part with z_top the top node height. */
static double rayleigh_part(const gb_bc* bc, double ztop, double z)
{
    const double pi = 3.14159265358979323846;
    if (bc->rayleigh_zdamp > 0 && z > bc->rayleigh_zdamp) {
        const double s = sin(0.5 * pi * (z - bc->rayleigh_zdamp) / (ztop - bc->rayleigh_zdamp));
        return bc->rayleigh_dampcoef * s * s;
    }
    return 0;
}

/* DampingCoef::sponge_part: the distances to the inflow and outflow faces
 * (the domain from 0 to nx dx, 0 to ny dy). */
static double sponge_part(const og_grid* g, const gb_bc* bc, double x, double y)
{
    double c = 0;
    if (bc->sponge_width > 0) {
        const double inv_w = 1 / bc->sponge_width;
        const double dist[4] = {x - 0.0, g->nx * g->dx - x, y - 0.0, g->ny * g->dy - y};
        const int faces[4] = {0, 3, 1, 4};
        for (int n = 0; n < 4; ++n) {
            const int t = bc->face[faces[n]];
            if ((t == GB_FACE_INFLOW || t == GB_FACE_OUTFLOW) && dist[n] < bc->sponge_width) {
                const double r = 1 - dist[n] * inv_w;
                c += bc->sponge_strength * r * r;
            }
        }
    }
    return c;
}

/* The Rayleigh and sponge coefficients of point (i, j, k) of type t, and
 * its heights above the ground (h) and absolute (zc). */
static void damping_at(const og_grid* g, const gb_bc* bc, const double* z, int f, int t, int i, int j, int k,
                       double* cr, double* cs, double* h, double* zc)
{
    *h = height_above_ground(g, z, t, i, j, k);
    *zc = point_z(g, z, t, i, j, k);
    const double ztop = z[IX(g, 0, 0, g->nz)];
    const double x = (i + (nodal(t, 0) ? 0 : 0.5)) * g->dx;
    const double y = (j + (nodal(t, 1) ? 0 : 0.5)) * g->dy;
    const double zr = bc->rayleigh_above_ground ? *h : *zc;
    const int field = (f == F_THETA) ? 3 : (f == F_TKE) ? 4 : f;
    *cr = ((bc->rayleigh_fields >> field) & 1) ? rayleigh_part(bc, ztop, zr) : 0.0;
    *cs = sponge_part(g, bc, x, y);
}

/* BoundaryConditions::add_damping (:1022-1071): R += c (q - q_ref) on the
 * valid points of u, v, w, theta, k. */
static void add_damping(const og_grid* g, const gb_bc* bc, const gb_state* q, double** R)
{
    if (!damping_on(bc)) { return; }
    const double* qf[5] = {q->u, q->v, q->w, q->theta, q->tke};
    double* rf[5] = {R[0], R[1], R[2], R[4], R[5]};
    const int ff[5] = {F_U, F_V, F_W, F_THETA, F_TKE};
    for (int n = 0; n < 5; ++n) {
        const int f = ff[n];
        const int t = (n < 3) ? (1 << n) : CC;
        for (int k = 0; k < ext(g, t, 2); ++k) {
            for (int j = 0; j < ext(g, t, 1); ++j) {
                for (int i = 0; i < ext(g, t, 0); ++i) {
                    double cr, cs, h, zc;
                    damping_at(g, bc, q->z_nd, f, t, i, j, k, &cr, &cs, &h, &zc);
                    const int64_t o = IX(g, i, j, k);
                    if (cr > 0) {
                        const double zr = bc->rayleigh_above_ground ? h : zc;
                        const double ref = (f == F_W) ? 0.0 : profile_value(bc, f, (f == F_THETA) ? zr : h);
                        rf[n][o] += cr * (qf[n][o] - ref);
                    }
                    if (cs > 0) {
                        const double ref = (f == F_W) ? 0.0 : profile_value(bc, f, h);
                        rf[n][o] += cs * (qf[n][o] - ref);
                    }
                }
            }
        }
    }
}

/* add_damping_to_implicit (:1073-1099): a_P += the Rayleigh and sponge parts. */
static void add_damping_to_implicit(const og_grid* g, const gb_bc* bc, const double* z, int f, int t, double* A)
{
    if (!damping_on(bc)) { return; }
    const int64_t cs = VOL(g);
    for (int k = 0; k < ext(g, t, 2); ++k) {
        for (int j = 0; j < ext(g, t, 1); ++j) {
            for (int i = 0; i < ext(g, t, 0); ++i) {
                double cr, csp, h, zc;
                damping_at(g, bc, z, f, t, i, j, k, &cr, &csp, &h, &zc);
                A[COEF_P * cs + IX(g, i, j, k)] += cr + csp;
            }
        }
    }
}

/* dirichlet_rows (BoundaryConditions.cpp:854-883). */
static void dirichlet_rows(const og_grid* g, const gb_bc* bc, int f, int t, double* mask)
{
    memset(mask, 0, sizeof(double) * VOL(g));
    for (int d = 0; d < 3; ++d) {
        if (is_per(g, d)) { continue; }
        for (int lo = 1; lo >= 0; --lo) {
            const int fc = d + (lo ? 0 : 3);
            const int rule = rule_for(f, bc->face[fc], d, lo);
            if (!(nodal(t, d) && (rule == R_VALUE || rule == R_PROFILE))) { continue; }
            const int edge = lo ? 0 : ((d == 0) ? g->nx : (d == 1) ? g->ny : g->nz);
            int rlo[3], rhi[3];
            for (int e = 0; e < 3; ++e) { rlo[e] = 0; rhi[e] = ext(g, t, e) - 1; }
            rlo[d] = rhi[d] = edge;
            for (int k = rlo[2]; k <= rhi[2]; ++k) {
                for (int j = rlo[1]; j <= rhi[1]; ++j) {
                    for (int i = rlo[0]; i <= rhi[0]; ++i) { mask[IX(g, i, j, k)] = 1.0; }
                }
            }
        }
    }
}

void og_dirichlet_rows(const og_grid* g, const gb_bc* bc, int f, int t, double* mask) { dirichlet_rows(g, bc, f, t, mask); }

/* apply_to_implicit (BoundaryConditions.cpp:885-941): the damping first,
 * then the folds (a Dirichlet face point's row becomes the identity). */
static void apply_to_implicit(const og_grid* g, const gb_bc* bc, const double* z, int f, int t, double* A)
{
    add_damping_to_implicit(g, bc, z, f, t, A);
    const int64_t cs = VOL(g);
    for (int d = 0; d < 3; ++d) {
        if (is_per(g, d)) { continue; }
        for (int lo = 1; lo >= 0; --lo) {
            const int fc = d + (lo ? 0 : 3);
            const int rule = rule_for(f, bc->face[fc], d, lo);
            const int nod = nodal(t, d);
            const int dirichlet_pt = nod && (rule == R_VALUE || rule == R_PROFILE);
            const int nd = (d == 0) ? g->nx : (d == 1) ? g->ny : g->nz;
            const int edge = lo ? 0 : (nod ? nd : nd - 1);
            const int cm = (d == 0) ? COEF_XM : (d == 1) ? COEF_YM : COEF_ZM;
            const int cp = (d == 0) ? COEF_XP : (d == 1) ? COEF_YP : COEF_ZP;
            const int ghost_coef = lo ? cm : cp, other_coef = lo ? cp : cm;
            double fold = 0;
            int to_other = 0;
            if (nod) { to_other = 1; }
            else if (rule == R_EVEN) { fold = -1; }
            else if (rule == R_ODD || rule == R_VALUE) { fold = 1; }
            else if (rule == R_GRADIENT) { to_other = 1; }
            int rlo[3], rhi[3];
            for (int e = 0; e < 3; ++e) { rlo[e] = 0; rhi[e] = ext(g, t, e) - 1; }
            rlo[d] = rhi[d] = edge;
            for (int k = rlo[2]; k <= rhi[2]; ++k) {
                for (int j = rlo[1]; j <= rhi[1]; ++j) {
                    for (int i = rlo[0]; i <= rhi[0]; ++i) {
                        const int64_t o = IX(g, i, j, k);
                        if (dirichlet_pt) {
                            for (int n = 0; n < N_COEFS; ++n) { A[n * cs + o] = 0; }
                            A[COEF_P * cs + o] = 1;
                        } else {
                            const double ag = A[ghost_coef * cs + o];
                            A[ghost_coef * cs + o] = 0;
                            if (to_other) { A[other_coef * cs + o] += ag; } else { A[COEF_P * cs + o] += fold * ag; }
                        }
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* forcing                                                             */
/* ------------------------------------------------------------------ */

static double coriolis_parameter(const gb_physics* ph)
{
    if (!ph->coriolis) { return 0; }
    const double pi = 3.14159265358979323846;
    return 4 * pi * sin(ph->latitude * pi / 180) / ph->rotation_period;
}

/* Forcing.cpp fill_theta_ref over the cells and one ghost layer. */
static void fill_theta_ref(const og_grid* g, const gb_bc* bc, const double* z, double* tr)
{
    const int n = bc->theta_ref_n;
    const double* zp = bc->theta_ref_z;
    const double* tp = bc->theta_ref_theta;
    for (int k = -1; k <= g->nz; ++k) {
        for (int j = -1; j <= g->ny; ++j) {
            for (int i = -1; i <= g->nx; ++i) {
                const double zc = og_interp(g, z, NODE, CC, i, j, k);
                double v = tp[0];
                if (zc >= zp[n - 1]) {
                    v = tp[n - 1];
                } else {
                    for (int m = 1; m < n; ++m) {
                        if (zc < zp[m]) {
                            if (zc > zp[m - 1]) {
                                const double w = (zc - zp[m - 1]) / (zp[m] - zp[m - 1]);
                                v = tp[m - 1] + w * (tp[m] - tp[m - 1]);
                            } else {
                                v = tp[m - 1];
                            }
                            break;
                        }
                    }
                }
                tr[IX(g, i, j, k)] = v;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* residual                                                            */
/* ------------------------------------------------------------------ */

typedef struct og_fields {
    double *u, *v, *w, *p, *th, *tk;
    const double* z;
} og_fields;

/* Residual.cpp:159-256 residual(): the diffusivities given (ph->closure = 0)
 * or the closure's at q (its fields into t->cf), the wall model's ground
 * fluxes and wall-k rows with a surface_layer ground (the surface state into
 * t->ss). R[6]: u, v, w, p, theta, k. */
static void residual_t(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const gb_state* q,
                       const gb_mesh_fields* m, const gb_diffusivities* df, double** R, const og_turb* t)
{
    const int64_t vol = VOL(g);
    const int wall = bc->face[2] == GB_FACE_SURFACE_LAYER;
    const double *nu = df ? df->nu : NULL, *gamma_theta = df ? df->gamma_theta : NULL, *gamma_tke = df ? df->gamma_tke : NULL;
    if (ph->closure) {
        og_closure_evaluate(g, bc, ph, q->u, q->v, q->w, q->theta, q->tke, q->z_nd, m->z0, (double**)t->cf);
        nu = t->cf[CF_NU];
        gamma_theta = t->cf[CF_GTH];
        gamma_tke = t->cf[CF_GK];
    }
    double* F[3];
    for (int d = 0; d < 3; ++d) { F[d] = zalloc(g); }
    og_transport_fluxes(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, F[0], F[1], F[2]);
    const double* vel[3] = {q->u, q->v, q->w};
    double* tmp = zalloc(g);
    double* Gm[3][3];
    for (int c = 0; c < 3; ++c) {
        og_convection(g, 1 << c, vel[c], F[0], F[1], F[2], m->detJ, ph->limiter, ph->smooth_eps_velocity, 0, R[c]);
        for (int d = 0; d < 3; ++d) { Gm[c][d] = zalloc(g); }
        og_momentum_diffusive_fluxes(g, c, q->u, q->v, q->w, nu, q->z_nd, ph->log_mean, Gm[c][0], Gm[c][1], Gm[c][2]);
    }
    double *Gt[3], *Gk[3];
    for (int d = 0; d < 3; ++d) {
        Gt[d] = zalloc(g);
        Gk[d] = zalloc(g);
    }
    og_scalar_diffusive_fluxes(g, q->theta, gamma_theta, q->z_nd, ph->log_mean, Gt[0], Gt[1], Gt[2]);
    og_scalar_diffusive_fluxes(g, q->tke, gamma_tke, q->z_nd, ph->log_mean, Gk[0], Gk[1], Gk[2]);
    if (wall) {
        og_surface_state(g, bc, ph, q->u, q->v, q->w, q->z_nd, m->z0, (double**)t->ss);
        og_set_ground_fluxes(g, bc, (const double* const*)t->ss, Gm[0][2], Gm[1][2], Gt[2], Gk[2]);
    }
    for (int c = 0; c < 3; ++c) {
        og_flux_divergence(g, 1 << c, Gm[c][0], Gm[c][1], Gm[c][2], m->detJ, tmp);
        for (int64_t n = 0; n < vol; ++n) { R[c][n] -= tmp[n]; }
    }
    double* Gp[3] = {zalloc(g), zalloc(g), zalloc(g)};
    og_pressure_gradient(g, q->p, q->z_nd, m->detJ, m->ax, m->ay, Gp[0], Gp[1], Gp[2]);
    for (int c = 0; c < 3; ++c) {
        for (int k = 0; k < ext(g, 1 << c, 2); ++k) {
            for (int j = 0; j < ext(g, 1 << c, 1); ++j) {
                for (int i = 0; i < ext(g, 1 << c, 0); ++i) { R[c][IX(g, i, j, k)] += Gp[c][IX(g, i, j, k)]; }
            }
        }
    }
    /* buoyancy (Forcing.cpp subtract_buoyancy) */
    if (ph->gravity > 0) {
        double* tr = zalloc(g);
        fill_theta_ref(g, bc, q->z_nd, tr);
        const double gt = ph->gravity / ph->theta0;
        for (int k = 0; k <= g->nz; ++k) {
            for (int j = 0; j < g->ny; ++j) {
                for (int i = 0; i < g->nx; ++i) {
                    R[2][IX(g, i, j, k)] -= gt * 0.5 * ((q->theta[IX(g, i, j, k - 1)] - tr[IX(g, i, j, k - 1)])
                                                        + (q->theta[IX(g, i, j, k)] - tr[IX(g, i, j, k)]));
                }
            }
        }
        free(tr);
    }
    /* Coriolis (Forcing.cpp subtract_coriolis) */
    if (ph->coriolis) {
        const double pi = 3.14159265358979323846;
        const double phi = ph->latitude * pi / 180;
        const double fc = 4 * pi / ph->rotation_period;
        const double fs = fc * sin(phi);
        const double fcos = ph->coriolis_3d ? fc * cos(phi) : 0.0;
        const double ug = ph->geostrophic ? ph->ug : 0.0, vg = ph->geostrophic ? ph->vg : 0.0;
        for (int k = 0; k < g->nz; ++k) {
            for (int j = 0; j < g->ny; ++j) {
                for (int i = 0; i <= g->nx; ++i) {
                    R[0][IX(g, i, j, k)] -= fs * (og_interp(g, q->v, YF, XF, i, j, k) - vg) - fcos * og_interp(g, q->w, ZF, XF, i, j, k);
                }
            }
            for (int j = 0; j <= g->ny; ++j) {
                for (int i = 0; i < g->nx; ++i) { R[1][IX(g, i, j, k)] += fs * (og_interp(g, q->u, XF, YF, i, j, k) - ug); }
            }
        }
        if (ph->coriolis_3d) {
            for (int k = 0; k <= g->nz; ++k) {
                for (int j = 0; j < g->ny; ++j) {
                    for (int i = 0; i < g->nx; ++i) { R[2][IX(g, i, j, k)] -= fcos * og_interp(g, q->u, XF, ZF, i, j, k); }
                }
            }
        }
    }
    /* constant pressure-gradient force */
    for (int c = 0; c < 3; ++c) {
        if (ph->pressure_gradient[c] == 0) { continue; }
        for (int k = 0; k < ext(g, 1 << c, 2); ++k) {
            for (int j = 0; j < ext(g, 1 << c, 1); ++j) {
                for (int i = 0; i < ext(g, 1 << c, 0); ++i) { R[c][IX(g, i, j, k)] += -ph->pressure_gradient[c]; }
            }
        }
    }
    /* continuity */
    og_velocity_divergence(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, m->az, m->detJ, R[3]);
    /* scalars */
    og_convection(g, CC, q->theta, F[0], F[1], F[2], m->detJ, ph->limiter, ph->smooth_eps_theta, 0, R[4]);
    og_flux_divergence(g, CC, Gt[0], Gt[1], Gt[2], m->detJ, tmp);
    for (int64_t n = 0; n < vol; ++n) { R[4][n] -= tmp[n]; }
    og_convection(g, CC, q->tke, F[0], F[1], F[2], m->detJ, 2 /* upwind */, 1e-5, 1, R[5]);
    og_flux_divergence(g, CC, Gk[0], Gk[1], Gk[2], m->detJ, tmp);
    for (int64_t n = 0; n < vol; ++n) { R[5][n] -= tmp[n]; }
    if (ph->closure) {
        /* R_k -= S_k = P_s + P_b - eps on the valid cells */
        for (int k = 0; k < g->nz; ++k) {
            for (int j = 0; j < g->ny; ++j) {
                for (int i = 0; i < g->nx; ++i) { R[5][IX(g, i, j, k)] -= t->cf[CF_PS][IX(g, i, j, k)]; }
            }
        }
        for (int k = 0; k < g->nz; ++k) {
            for (int j = 0; j < g->ny; ++j) {
                for (int i = 0; i < g->nx; ++i) { R[5][IX(g, i, j, k)] -= t->cf[CF_PB][IX(g, i, j, k)]; }
            }
        }
        for (int k = 0; k < g->nz; ++k) {
            for (int j = 0; j < g->ny; ++j) {
                for (int i = 0; i < g->nx; ++i) { R[5][IX(g, i, j, k)] += t->cf[CF_EPS][IX(g, i, j, k)]; }
            }
        }
    }
    if (wall) { og_apply_wall_k(g, bc, (const double* const*)t->ss, q->tke, R[5]); }
    add_damping(g, bc, q, R);
    apply_rows(g, bc, q->u, q->v, q->w, q->z_nd, R[0], R[1], R[2]);
    og_override_sync(g, XF, R[0]);
    og_override_sync(g, YF, R[1]);
    og_override_sync(g, ZF, R[2]);
    for (int d = 0; d < 3; ++d) {
        free(F[d]);
        free(Gt[d]);
        free(Gk[d]);
        free(Gp[d]);
        for (int c = 0; c < 3; ++c) { free(Gm[c][d]); }
    }
    free(tmp);
}

/* The residual with the closure's fields (N_CF volumes) and the surface
 * state (N_SS planes) into cf_out, ss_out when given. */
void og_residual2(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const gb_state* q, const gb_mesh_fields* m,
                  const gb_diffusivities* df, double** R, double** cf_out, double** ss_out)
{
    double* cfl[N_CF] = {0};
    double* ssl[N_SS] = {0};
    og_turb t = {cf_out, ss_out};
    if (ph->closure && !cf_out) {
        for (int n = 0; n < N_CF; ++n) { cfl[n] = zalloc(g); }
        t.cf = cfl;
    }
    if (bc->face[2] == GB_FACE_SURFACE_LAYER && !ss_out) {
        for (int n = 0; n < N_SS; ++n) { ssl[n] = palloc(g); }
        t.ss = ssl;
    }
    residual_t(g, bc, ph, q, m, df, R, &t);
    for (int n = 0; n < N_CF; ++n) { free(cfl[n]); }
    for (int n = 0; n < N_SS; ++n) { free(ssl[n]); }
}

void og_residual(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const gb_state* q, const gb_mesh_fields* m,
                 const gb_diffusivities* df, double** R)
{
    og_residual2(g, bc, ph, q, m, df, R, NULL, NULL);
}

/* Residual.cpp:272-304 implicit_rows: the closure's diffusivity and the
 * Patankar diagonal of k (tc->cf), the first cells' wall rows (tc->ss) for
 * every equation but w, then the boundary folds. */
static void implicit_rows_t(const og_grid* g, const gb_bc* bc, const gb_physics* ph, int eq, const double* F0,
                            const double* F1, const double* F2, const double* z, const double* J,
                            const gb_diffusivities* df, const og_turb* tc, double* A)
{
    const int closure = ph->closure && tc && tc->cf;
    const double* gm;
    if (closure) {
        gm = (eq <= F_W) ? tc->cf[CF_NU] : (eq == F_THETA) ? tc->cf[CF_GTH] : tc->cf[CF_GK];
    } else {
        gm = (eq <= F_W) ? df->nu : (eq == F_THETA) ? df->gamma_theta : df->gamma_tke;
    }
    const int C = (eq <= F_W) ? eq : -1;
    const int t = (eq <= F_W) ? (1 << eq) : CC;
    og_implicit_coefficients(g, C, F0, F1, F2, gm, z, J, ph->log_mean, A);
    if (closure && eq == F_TKE) {
        const int64_t cs = VOL(g);
        for (int k = 0; k < g->nz; ++k) {
            for (int j = 0; j < g->ny; ++j) {
                for (int i = 0; i < g->nx; ++i) { A[COEF_P * cs + IX(g, i, j, k)] += tc->cf[CF_DSDK][IX(g, i, j, k)]; }
            }
        }
    }
    if (bc->face[2] == GB_FACE_SURFACE_LAYER && eq != F_W && tc && tc->ss) {
        og_apply_wall_to_implicit(g, (const double* const*)tc->ss, t, J, A);
        if (eq == F_TKE) { og_apply_wall_k_to_implicit(g, bc, (const double* const*)tc->ss, A); }
    }
    apply_to_implicit(g, bc, z, eq, t, A);
}

void og_implicit_rows(const og_grid* g, const gb_bc* bc, const gb_physics* ph, int eq, const double* F0,
                      const double* F1, const double* F2, const double* z, const double* J, const gb_diffusivities* df,
                      double* A)
{
    implicit_rows_t(g, bc, ph, eq, F0, F1, F2, z, J, df, NULL, A);
}

/* implicit_rows with the closure's fields (N_CF volumes) and the surface
 * state (N_SS planes) of an evaluation (either null: none). */
void og_implicit_rows2(const og_grid* g, const gb_bc* bc, const gb_physics* ph, int eq, const double* F0,
                       const double* F1, const double* F2, const double* z, const double* J,
                       const gb_diffusivities* df, double** cf, double** ss, double* A)
{
    const og_turb t = {cf, ss};
    implicit_rows_t(g, bc, ph, eq, F0, F1, F2, z, J, df, &t, A);
}

/* ------------------------------------------------------------------ */
/* momentum predictor                                                  */
/* ------------------------------------------------------------------ */

/* Predictor.cpp:129-405 momentum_predictor (zjacobi sweeps). ap/d: the
 * predictor fields a_P, d per component (face arrays). */
/* The line solver of the sweeps (steady.sweep, Source/Predictor.H:257-259
 * line_sweeps): z-line Jacobi, or line LU-SGS (lagged ghosts, sequential
 * order) with steady.line_alternate. */
static double line_solve(const og_grid* g, const gb_simplec_opts* so, int loc, const double* A, const double* ap,
                         const double* rhs, double* delta)
{
    if (so->line_sweep == 1) { return og_zline_lusgs(g, loc, A, ap, rhs, so->zline_sweeps, 0, so->line_alternate, delta); }
    return og_zline_jacobi(g, loc, A, ap, rhs, so->zline_sweeps, delta);
}

void og_momentum_predictor(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const gb_simplec_opts* so,
                           gb_state* q, double** R, const double* F0, const double* F1, const double* F2,
                           double** dtau_f, const gb_mesh_fields* m, const gb_diffusivities* df, const og_turb* tc,
                           double** ap, double** dd, double* info)
{
    const int64_t vol = VOL(g), cs = vol;
    double* comps[3] = {q->u, q->v, q->w};
    const double dxinv[3] = {1.0 / g->dx, 1.0 / g->dy, 1.0 / g->dzeta};
    double* A = (double*)calloc(N_COEFS * vol, sizeof(double));
    double* mask = zalloc(g);
    double* rhs = zalloc(g);
    double* delta = zalloc(g);
    const double fs = coriolis_parameter(ph);
    for (int c = 0; c < 3; ++c) {
        const int t = 1 << c;
        implicit_rows_t(g, bc, ph, c, F0, F1, F2, q->z_nd, m->detJ, df, tc, A);
        dirichlet_rows(g, bc, c, t, mask);
        const int ni = ext(g, t, 0), nj = ext(g, t, 1), nk = ext(g, t, 2);
        for (int k = 0; k < nk; ++k) {
            for (int j = 0; j < nj; ++j) {
                for (int i = 0; i < ni; ++i) {
                    const int64_t o = IX(g, i, j, k);
                    const double keep = 1.0 - mask[o];
                    ap[c][o] = keep / dtau_f[c][o] + A[COEF_P * cs + o];
                    const double nb = A[COEF_XM * cs + o] + A[COEF_XP * cs + o] + A[COEF_YM * cs + o] + A[COEF_YP * cs + o]
                                    + A[COEF_ZM * cs + o] + A[COEF_ZP * cs + o];
                    dd[c][o] = keep * (ap[c][o] - nb);
                }
            }
        }
        if (c == 2 && so->w_vnn_cap > 0) {
            const double inv_cap = 1.0 / so->w_vnn_cap;
            const double s = so->w_vnn_cap_slope_margin;
            for (int k = 0; k < nk; ++k) {
                for (int j = 0; j < nj; ++j) {
                    for (int i = 0; i < ni; ++i) {
                        const int64_t o = IX(g, i, j, k);
                        const double keep = 1.0 - mask[o];
                        double term = inv_cap * (A[COEF_ZM * cs + o] + A[COEF_ZP * cs + o]);
                        if (s > 0) {
                            const double* zp = q->z_nd;
                            const double hx = 0.5 * (zp[IX(g, i + 1, j + 1, k)] + zp[IX(g, i + 1, j, k)] - zp[IX(g, i, j + 1, k)] - zp[IX(g, i, j, k)]) * dxinv[0];
                            const double hy = 0.5 * (zp[IX(g, i + 1, j + 1, k)] + zp[IX(g, i, j + 1, k)] - zp[IX(g, i + 1, j, k)] - zp[IX(g, i, j, k)]) * dxinv[1];
                            const double slope2 = hx * hx + hy * hy;
                            if (slope2 > 0) {
                                const double root = sqrt(1.0 + slope2) + 1.0;
                                const double rc = slope2 / (root * root);
                                const double lim = fmax(0.0, 1.0 / (s * rc) - 1.0) / dtau_f[c][o];
                                term = fmin(term, lim);
                            }
                        }
                        const double cap = keep * term;
                        ap[c][o] += cap;
                        dd[c][o] += cap;
                    }
                }
            }
        }
        for (int k = 0; k < nk; ++k) {
            for (int j = 0; j < nj; ++j) {
                for (int i = 0; i < ni; ++i) { rhs[IX(g, i, j, k)] = -R[c][IX(g, i, j, k)]; }
            }
        }
        if (c < 2 && ph->coriolis && fs != 0) {
            /* the other component's residual with its periodic images */
            const double* other = (c == 0) ? R[1] : R[0];
            const int to = (c == 0) ? YF : XF;
            double* og = zalloc(g);
            for (int k = 0; k < ext(g, to, 2); ++k) {
                for (int j = 0; j < ext(g, to, 1); ++j) {
                    for (int i = 0; i < ext(g, to, 0); ++i) { og[IX(g, i, j, k)] = other[IX(g, i, j, k)]; }
                }
            }
            og_fill_periodic(g, to, og, 1);
            /* the horizontal mean per level, every face once */
            const int d_o = 1 - c;
            const int per_o = is_per(g, d_o);
            const int nz = g->nz;
            double* sum = (double*)calloc(nz, sizeof(double));
            const int ilo_hi = ext(g, to, 0) - ((d_o == 0 && per_o) ? 1 : 0);
            const int jlo_hi = ext(g, to, 1) - ((d_o == 1 && per_o) ? 1 : 0);
            for (int k = 0; k < nz; ++k) {
                for (int j = 0; j < jlo_hi; ++j) {
                    for (int i = 0; i < ilo_hi; ++i) { sum[k] += other[IX(g, i, j, k)]; }
                }
            }
            const int n_o = (d_o == 0) ? g->nx : g->ny, n_c = (c == 0) ? g->nx : g->ny;
            const double npts_level = (double)(n_o + (per_o ? 0 : 1)) * (double)n_c;
            for (int k = 0; k < nz; ++k) { sum[k] /= npts_level; }
            const int per_c = is_per(g, c);
            const int lo_edge = 0, hi_edge = (c == 0) ? g->nx : g->ny;
            for (int k = 0; k < nk; ++k) {
                for (int j = 0; j < nj; ++j) {
                    for (int i = 0; i < ni; ++i) {
                        const int64_t o = IX(g, i, j, k);
                        const double keep = 1.0 - mask[o];
                        if (keep == 0) { continue; }
                        const int n = (c == 0) ? i : j;
                        if (!per_c && (n == lo_edge || n == hi_edge)) { continue; }
                        const double nb = A[COEF_XM * cs + o] + A[COEF_XP * cs + o] + A[COEF_YM * cs + o] + A[COEF_YP * cs + o]
                                        + A[COEF_ZM * cs + o] + A[COEF_ZP * cs + o];
                        const double net = fmax(A[COEF_P * cs + o] - nb, 0.0);
                        const double tau_c = 1.0 / fmax(fabs(fs) / so->rotation_relax, net);
                        const double tau_own = 1.0 / (1.0 / dtau_f[c][o] + net);
                        const double stiff = fs * fs * fmax(tau_c, tau_own);
                        ap[c][o] += stiff;
                        dd[c][o] += stiff;
                        const double avg = (c == 0) ? og_interp(g, og, YF, XF, i, j, k) : og_interp(g, og, XF, YF, i, j, k);
                        const double mean = sum[k];
                        rhs[o] += ((c == 0) ? -fs : fs) * (tau_c * mean + tau_own * (avg - mean));
                    }
                }
            }
            free(sum);
            free(og);
        }
        if (c == 2 && ph->gravity > 0) {
            const double gt = ph->gravity / ph->theta0;
            double* At = (double*)calloc(N_COEFS * vol, sizeof(double));
            implicit_rows_t(g, bc, ph, F_THETA, F0, F1, F2, q->z_nd, m->detJ, df, tc, At);
            const double* z = q->z_nd;
            for (int k = 0; k < nk; ++k) {
                for (int j = 0; j < nj; ++j) {
                    for (int i = 0; i < ni; ++i) {
                        const int64_t o = IX(g, i, j, k);
                        const double keep = 1.0 - mask[o];
                        if (keep == 0) { continue; }
#define ZC(kk) (0.125 * (z[IX(g, i, j, kk)] + z[IX(g, i + 1, j, kk)] + z[IX(g, i, j + 1, kk)] + z[IX(g, i + 1, j + 1, kk)] \
                        + z[IX(g, i, j, kk + 1)] + z[IX(g, i + 1, j, kk + 1)] + z[IX(g, i, j + 1, kk + 1)] + z[IX(g, i + 1, j + 1, kk + 1)]))
                        const double gamma = (q->theta[IX(g, i, j, k)] - q->theta[IX(g, i, j, k - 1)]) / (ZC(k) - ZC(k - 1));
#undef ZC
                        const double ap_theta = 0.5 * (At[COEF_P * cs + IX(g, i, j, k - 1)] + At[COEF_P * cs + o]);
                        const double tau = 1.0 / (1.0 / dtau_f[c][o] + ap_theta);
                        const double stiff = gt * fmax(gamma, 0.0) * tau;
                        ap[c][o] += stiff;
                        dd[c][o] += stiff;
                        rhs[o] -= gt * tau * 0.5 * (R[4][IX(g, i, j, k - 1)] + R[4][o]);
                    }
                }
            }
            free(At);
        }
        info[3 + c] = line_solve(g, so, t, A, ap[c], rhs, delta);
        double mx = 0;
        for (int k = 0; k < nk; ++k) {
            for (int j = 0; j < nj; ++j) {
                for (int i = 0; i < ni; ++i) {
                    const double d = fabs(delta[IX(g, i, j, k)]);
                    if (d > mx || d != d) { mx = d; }
                    comps[c][IX(g, i, j, k)] += delta[IX(g, i, j, k)];
                }
            }
        }
        info[c] = mx;
    }
    free(A);
    free(mask);
    free(rhs);
    free(delta);
}

/* ------------------------------------------------------------------ */
/* pressure correction                                                 */
/* ------------------------------------------------------------------ */

static double max_abs_valid(const og_grid* g, int t, const double* f, const double* keep)
{
    double m = 0;
    for (int k = 0; k < ext(g, t, 2); ++k) {
        for (int j = 0; j < ext(g, t, 1); ++j) {
            for (int i = 0; i < ext(g, t, 0); ++i) {
                const int64_t o = IX(g, i, j, k);
                const double v = fabs(keep ? f[o] * keep[o] : f[o]);
                if (v > m || v != v) { m = v; }
            }
        }
    }
    return m;
}

/* poisson_bc_from_faces (BoundaryConditions.cpp:362-380): periodic where the
 * geometry is, Dirichlet (odd) for outflow, Neumann for every other type. */
void og_poisson_bc_from_faces(const og_grid* g, const gb_bc* bc, int* pbc)
{
    for (int f = 0; f < 6; ++f) {
        const int d = f % 3;
        if (is_per(g, d)) { pbc[f] = 0; }
        else { pbc[f] = (bc->face[f] == GB_FACE_OUTFLOW) ? 2 : 1; }
    }
}

/* Simplec.cpp:134-220 pressure_correction. info: [div_before, div_after,
 * max_dp, max_du, max_dv, max_dw, removed_mean, iterations]. Returns 0, or
 * -1 on a net source the boundaries cannot carry, -2 on a Poisson failure. */
int og_pressure_correction(const og_grid* g, const gb_bc* bc, const gb_simplec_opts* so, gb_state* q, double** dd,
                           const gb_mesh_fields* m, double* info)
{
    const int64_t vol = VOL(g);
    double *beta[3], *keep[3];
    const int tt[3] = {XF, YF, ZF};
    for (int c = 0; c < 3; ++c) {
        beta[c] = zalloc(g);
        keep[c] = zalloc(g);
        for (int k = 0; k < ext(g, tt[c], 2); ++k) {
            for (int j = 0; j < ext(g, tt[c], 1); ++j) {
                for (int i = 0; i < ext(g, tt[c], 0); ++i) {
                    const int64_t o = IX(g, i, j, k);
                    const int on = dd[c][o] > 0;
                    beta[c][o] = on ? 1.0 / dd[c][o] : 1.0;
                    keep[c][o] = on ? 1.0 : 0.0;
                }
            }
        }
    }
    double* rhs = zalloc(g);
    og_velocity_divergence(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, m->az, m->detJ, rhs);
    info[0] = max_abs_valid(g, CC, rhs, NULL);
    double speed = fmax(fmax(max_abs_valid(g, XF, q->u, NULL), max_abs_valid(g, YF, q->v, NULL)), max_abs_valid(g, ZF, q->w, NULL));
    double jmin = 1e300;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) { jmin = fmin(jmin, m->detJ[IX(g, i, j, k)]); }
        }
    }
    const double inv_h = 1.0 / g->dx + 1.0 / g->dy + 1.0 / (jmin * g->dzeta);
    int pbc[6];
    og_poisson_bc_from_faces(g, bc, pbc);
    double* AX = zalloc(g);
    double* AY = zalloc(g);
    double* AZ = zalloc(g);
    for (int64_t n = 0; n < vol; ++n) {
        AX[n] = m->ax[n] * beta[0][n];
        AY[n] = m->ay[n] * beta[1][n];
        AZ[n] = m->az[n] * beta[2][n];
    }
    const gb_poisson_opts* po = &so->poisson;
    og_mg* mg = og_mg_create(g, pbc, q->z_nd, m->detJ, AX, AY, AZ, po->max_levels, po->min_coarse, po->nu1, po->nu2,
                             po->nu_coarse);
    double* phi = zalloc(g);
    double res[3];
    const int it = og_poisson_solve(mg, rhs, phi, so->pressure_reltol, po->abstol, po->max_iter, po->restart, 1, res);
    og_mg_destroy(mg);
    int singular = 1;
    for (int f = 0; f < 6; ++f) {
        if (pbc[f] == 2) { singular = 0; }
    }
    info[6] = res[2];
    info[7] = it;
    int status = 0;
    if (it < 0) { status = -2; }
    if (singular && fabs(res[2]) > 1.0e-8 * speed * inv_h) { status = -1; }
    double* F[3] = {zalloc(g), zalloc(g), zalloc(g)};
    og_poisson_fluxes(g, pbc, q->z_nd, phi, beta[0], beta[1], beta[2], F[0], F[1], F[2]);
    double mxp = 0;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const int64_t o = IX(g, i, j, k);
                q->p[o] += so->alpha_p * phi[o];
                mxp = fmax(mxp, fabs(phi[o]));
            }
        }
    }
    info[2] = so->alpha_p * mxp;
    for (int c = 0; c < 3; ++c) { info[3 + c] = max_abs_valid(g, tt[c], F[c], keep[c]); }
    double* om = zalloc(g);
    og_omega_from_w(g, q->u, q->v, q->w, q->z_nd, om, 0);
    double* tgt[3] = {q->u, q->v, om};
    for (int c = 0; c < 3; ++c) {
        for (int k = 0; k < ext(g, tt[c], 2); ++k) {
            for (int j = 0; j < ext(g, tt[c], 1); ++j) {
                for (int i = 0; i < ext(g, tt[c], 0); ++i) {
                    const int64_t o = IX(g, i, j, k);
                    tgt[c][o] += F[c][o] * keep[c][o];
                }
            }
        }
    }
    og_override_sync(g, XF, q->u);
    og_override_sync(g, YF, q->v);
    og_override_sync(g, ZF, om);
    fill_periodic2(g, XF, q->u);
    fill_periodic2(g, YF, q->v);
    og_w_from_omega(g, q->u, q->v, om, q->z_nd, q->w);
    og_override_sync(g, ZF, q->w);
    fill_periodic2(g, ZF, q->w);
    og_velocity_divergence(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, m->az, m->detJ, rhs);
    info[1] = max_abs_valid(g, CC, rhs, NULL);
    for (int c = 0; c < 3; ++c) {
        free(beta[c]);
        free(keep[c]);
        free(F[c]);
    }
    free(rhs);
    free(AX);
    free(AY);
    free(AZ);
    free(phi);
    free(om);
    return status;
}

/* ------------------------------------------------------------------ */
/* scalar sweep, stage                                                 */
/* ------------------------------------------------------------------ */

/* Simplec.cpp:222-281 scalar_sweep. Returns max |dq|; *clipped the k floor count. */
double og_scalar_sweep(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const gb_simplec_opts* so, int eq,
                       double* field, const double* Req, const double* F0, const double* F1, const double* F2,
                       const double* z, const double* J, const gb_diffusivities* df, const og_turb* tc,
                       const double* dtau, double floor, int clip, double* last, int64_t* clipped)
{
    const int64_t vol = VOL(g), cs = vol;
    double* A = (double*)calloc(N_COEFS * vol, sizeof(double));
    implicit_rows_t(g, bc, ph, eq, F0, F1, F2, z, J, df, tc, A);
    double* rhs = zalloc(g);
    double* ap = zalloc(g);
    double* delta = zalloc(g);
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const int64_t o = IX(g, i, j, k);
                rhs[o] = -Req[o];
                ap[o] = 1.0 / dtau[o] + A[COEF_P * cs + o];
            }
        }
    }
    *last = line_solve(g, so, CC, A, ap, rhs, delta);
    double mx = 0;
    int64_t n = 0;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const int64_t o = IX(g, i, j, k);
                const double d = fabs(delta[o]);
                if (d > mx || d != d) { mx = d; }
                field[o] += delta[o];
                if (eq == F_TKE && clip && field[o] < floor) {
                    field[o] = floor;
                    ++n;
                }
            }
        }
    }
    *clipped = n;
    free(A);
    free(rhs);
    free(ap);
    free(delta);
    return mx;
}

/* Simplec.cpp:373-409 stage_norms (scaled RMS of the six residuals; every
 * valid point, both copies of a seam face) and the max-speed and mean-k monitors. */
void og_stage_norms(const og_grid* g, const gb_physics* ph, double** R, const gb_state* q, double* res, double* mon)
{
    const int tt[6] = {XF, YF, ZF, CC, CC, CC};
    const double U = ph->scale_velocity, H = ph->scale_height;
    const double scale[6] = {U * U / H, U * U / H, U * U / H, U / H, U * ph->scale_theta / H, U * ph->scale_tke / H};
    for (int n = 0; n < 6; ++n) {
        double s = 0;
        const int64_t npts = (int64_t)ext(g, tt[n], 0) * ext(g, tt[n], 1) * ext(g, tt[n], 2);
        for (int k = 0; k < ext(g, tt[n], 2); ++k) {
            for (int j = 0; j < ext(g, tt[n], 1); ++j) {
                for (int i = 0; i < ext(g, tt[n], 0); ++i) {
                    const double v = R[n][IX(g, i, j, k)];
                    s += v * v;
                }
            }
        }
        res[n] = sqrt(s) / sqrt((double)npts) / scale[n];
    }
    mon[0] = fmax(fmax(max_abs_valid(g, XF, q->u, NULL), max_abs_valid(g, YF, q->v, NULL)), max_abs_valid(g, ZF, q->w, NULL));
    double s = 0;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) { s += q->tke[IX(g, i, j, k)]; }
        }
    }
    mon[1] = s / ((double)g->nx * g->ny * g->nz);
}

/* SimplecStage::iterate (Simplec.cpp:452-506) without a closure, a wall model
 * and the hybrid blend. R[6] receives the residual at the start. Returns 0 or
 * the pressure correction's status. */
/* SimplecStage::iterate (Simplec.cpp:452-506). With the closure its fields
 * at q (N_CF volumes, nu first: the next step's local dtau reads it) go to
 * cf_out, the surface state of step 1 to ss_out (N_SS planes), when given. */
int og_simplec_iterate2(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const gb_simplec_opts* so, gb_state* q,
                        const gb_mesh_fields* m, const gb_diffusivities* df, const double* dtau, double** R,
                        gb_iter_info* out, double** cf_out, double** ss_out)
{
    const int64_t vol = VOL(g);
    memset(out, 0, sizeof(*out));
    double* cfl[N_CF] = {0};
    double* ssl[N_SS] = {0};
    og_turb tcv = {cf_out, ss_out};
    if (ph->closure && !cf_out) {
        for (int n = 0; n < N_CF; ++n) { cfl[n] = zalloc(g); }
        tcv.cf = cfl;
    }
    if (bc->face[2] == GB_FACE_SURFACE_LAYER && !ss_out) {
        for (int n = 0; n < N_SS; ++n) { ssl[n] = palloc(g); }
        tcv.ss = ssl;
    }
    const og_turb* tc = &tcv;
    /* 1. ghosts and the wall state at q; 2. the residual (the closure at q) */
    og_fill_ghosts2(g, bc, ph, m->z0, q->u, q->v, q->w, q->p, q->theta, q->tke, q->z_nd, (double**)tc->ss);
    residual_t(g, bc, ph, q, m, df, R, tc);
    double mon[2];
    og_stage_norms(g, ph, R, q, out->residual_norms, mon);
    out->max_speed = mon[0];
    out->mean_tke = mon[1];
    if (tc->ss) {
        /* the third monitor (Simplec.cpp:405-408): the mean u* of the domain columns */
        double su = 0;
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) { su += tc->ss[0][(int64_t)(i + g->ng) + (int64_t)(j + g->ng) * g->sy]; }
        }
        out->mean_ustar = su / ((double)g->nx * g->ny);
    }
    double* F[3] = {zalloc(g), zalloc(g), zalloc(g)};
    og_transport_fluxes(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, F[0], F[1], F[2]);
    double* dcc = zalloc(g);
    memcpy(dcc, dtau, sizeof(double) * vol);
    double* dtf[3] = {zalloc(g), zalloc(g), zalloc(g)};
    og_face_dtau(g, dcc, dtf[0], dtf[1], dtf[2]);
    double* ap[3] = {zalloc(g), zalloc(g), zalloc(g)};
    double* dd[3] = {zalloc(g), zalloc(g), zalloc(g)};
    double pinfo[8];
    og_momentum_predictor(g, bc, ph, so, q, R, F[0], F[1], F[2], dtf, m, df, tc, ap, dd, pinfo);
    out->max_du = pinfo[0];
    out->max_dv = pinfo[1];
    out->max_dw = pinfo[2];
    out->last_sweep_du = pinfo[3];
    out->last_sweep_dv = pinfo[4];
    out->last_sweep_dw = pinfo[5];
    og_fill_ghosts2(g, bc, ph, m->z0, q->u, q->v, q->w, q->p, q->theta, q->tke, q->z_nd, NULL);
    double cinfo[8];
    const int st = og_pressure_correction(g, bc, so, q, dd, m, cinfo);
    out->divergence_before = cinfo[0];
    out->divergence_after = cinfo[1];
    out->max_dp = cinfo[2];
    out->poisson_removed_mean = cinfo[6];
    out->poisson_iterations = (int32_t)cinfo[7];
    /* theta's convection with the corrected transport */
    double* conv0 = zalloc(g);
    double* conv1 = zalloc(g);
    og_convection(g, CC, q->theta, F[0], F[1], F[2], m->detJ, ph->limiter, ph->smooth_eps_theta, 0, conv0);
    og_fill_ghosts2(g, bc, ph, m->z0, q->u, q->v, q->w, q->p, q->theta, q->tke, q->z_nd, NULL);
    og_transport_fluxes(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, F[0], F[1], F[2]);
    og_convection(g, CC, q->theta, F[0], F[1], F[2], m->detJ, ph->limiter, ph->smooth_eps_theta, 0, conv1);
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) {
                const int64_t o = IX(g, i, j, k);
                R[4][o] += conv1[o] - conv0[o];
            }
        }
    }
    double last;
    int64_t clipped = 0;
    out->max_dtheta = og_scalar_sweep(g, bc, ph, so, F_THETA, q->theta, R[4], F[0], F[1], F[2], q->z_nd, m->detJ, df,
                                      tc, dtau, 0, 0, &last, &clipped);
    out->max_dtke = og_scalar_sweep(g, bc, ph, so, F_TKE, q->tke, R[5], F[0], F[1], F[2], q->z_nd, m->detJ, df, tc,
                                    dtau, so->tke_floor, 1, &last, &clipped);
    out->tke_clipped = clipped;
    for (int c = 0; c < 3; ++c) {
        free(F[c]);
        free(dtf[c]);
        free(ap[c]);
        free(dd[c]);
    }
    free(dcc);
    free(conv0);
    free(conv1);
    for (int n = 0; n < N_CF; ++n) { free(cfl[n]); }
    for (int n = 0; n < N_SS; ++n) { free(ssl[n]); }
    return st;
}

int og_simplec_iterate(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const gb_simplec_opts* so, gb_state* q,
                       const gb_mesh_fields* m, const gb_diffusivities* df, const double* dtau, double** R,
                       gb_iter_info* out)
{
    return og_simplec_iterate2(g, bc, ph, so, q, m, df, dtau, R, out, NULL, NULL);
}

/* ------------------------------------------------------------------ */
/* mass-consistent initializer                                         */
/* ------------------------------------------------------------------ */

/* A profile component at every point of a field of type t (the valid box
 * grown by the state's two ghost layers) at the point's height above its
 * column's ground floored at h_min; k decays as exp(-(h - zi)/zi) above zi
 * (Source/Initializer.cpp:14-40 fill_from_profile). */
static void fill_from_profile(const og_grid* g, const gb_bc* bc, int t, int f, double h_min, double zi, const double* z,
                              double* a)
{
    const double zinv = 1.0 / fmax(zi, 2.2250738585072014e-308);
    for (int k = -2; k <= ext(g, t, 2) + 1; ++k) {
        for (int j = -2; j <= ext(g, t, 1) + 1; ++j) {
            for (int i = -2; i <= ext(g, t, 0) + 1; ++i) {
                const double h = fmax(height_above_ground(g, z, t, i, j, k), h_min);
                double val = profile_value(bc, f, h);
                if (f == F_TKE && zi > 0) { val *= exp(-(fmax(h - zi, 0.0) * zinv)); }
                a[IX(g, i, j, k)] = val;
            }
        }
    }
}

static double norm2_valid(const og_grid* g, const double* f)
{
    double s = 0;
    for (int k = 0; k < g->nz; ++k) {
        for (int j = 0; j < g->ny; ++j) {
            for (int i = 0; i < g->nx; ++i) { s += f[IX(g, i, j, k)] * f[IX(g, i, j, k)]; }
        }
    }
    return sqrt(s);
}

/* initializer_poisson_bc (Source/Initializer.cpp:181-195): periodic where
 * the geometry is; lambda = 0 (Dirichlet) on the inflow and outflow faces;
 * zero flux elsewhere. */
static void init_poisson_bc(const og_grid* g, const gb_bc* bc, int* pbc)
{
    for (int f = 0; f < 6; ++f) {
        const int d = f % 3;
        if (is_per(g, d)) { pbc[f] = 0; }
        else { pbc[f] = (bc->face[f] == GB_FACE_INFLOW || bc->face[f] == GB_FACE_OUTFLOW) ? 2 : 1; }
    }
}

/* gust::initialize_state with init.first_guess = profile and no O'Brien
 * correction (Source/Initializer.cpp:281-332 first_guess_state, 344-430):
 * the first guess, then with projection the mass-consistent correction
 * with Sigma = alpha^2 I (alpha_h = alpha_v). info: [divergence before,
 * divergence after, Poisson iterations, final Poisson residual]. Returns 0,
 * or -2 on a Poisson failure. */
/* obrien_omega (Source/Initializer.cpp:197-274): Omega on the z-faces from the
 * column continuity of (a_x u, a_y v) from Omega = 0 at the ground,
 * a_z Omega_{k+1/2} = a_z Omega_{k-1/2} - J_k Dh_k dzeta with Dh the horizontal
 * part of face_divergence, then the column's top value E removed with the
 * weight ((z_f - z_ground) / depth)^2 of the face's node-mean height, the top
 * face set to 0 exactly. Returns max |E| over the columns. */
double og_obrien_omega(const og_grid* g, const double* u, const double* v, const double* z, const double* ax,
                       const double* ay, const double* az, const double* J, double* om)
{
    double* zero = zalloc(g);
    double* dh = zalloc(g);
    og_face_divergence(g, ax, ay, az, J, u, v, zero, dh);
    const double dzeta = g->dzeta;
    double worst = 0;
    for (int j = 0; j < g->ny; ++j) {
        for (int i = 0; i < g->nx; ++i) {
            om[IX(g, i, j, 0)] = 0;
            for (int k = 0; k < g->nz; ++k) {
                om[IX(g, i, j, k + 1)] = (az[IX(g, i, j, k)] * om[IX(g, i, j, k)]
                                          - J[IX(g, i, j, k)] * dh[IX(g, i, j, k)] * dzeta)
                                         / az[IX(g, i, j, k + 1)];
            }
            const double E = om[IX(g, i, j, g->nz)];
            worst = fmax(worst, fabs(E));
            const double zg = 0.25 * (z[IX(g, i, j, 0)] + z[IX(g, i + 1, j, 0)] + z[IX(g, i, j + 1, 0)]
                                      + z[IX(g, i + 1, j + 1, 0)]);
            const double depth = 0.25 * (z[IX(g, i, j, g->nz)] + z[IX(g, i + 1, j, g->nz)] + z[IX(g, i, j + 1, g->nz)]
                                         + z[IX(g, i + 1, j + 1, g->nz)]) - zg;
            for (int k = 1; k <= g->nz; ++k) {
                const double zf = 0.25 * (z[IX(g, i, j, k)] + z[IX(g, i + 1, j, k)] + z[IX(g, i, j + 1, k)]
                                          + z[IX(g, i + 1, j + 1, k)]);
                const double frac = (zf - zg) / depth;
                om[IX(g, i, j, k)] -= frac * frac * E;
            }
            om[IX(g, i, j, g->nz)] = 0;
        }
    }
    free(zero);
    free(dh);
    return worst;
}

int og_initialize(const og_grid* g, const gb_bc* bc, const gb_init_opts* io, gb_state* q, const gb_mesh_fields* m,
                  double* info)
{
    const int64_t vol = VOL(g);
    const double* z = q->z_nd;
    /* 1. u, v at every point; w = 0 but the ground faces, which carry no flux */
    fill_from_profile(g, bc, XF, F_U, io->z_agl_min, 0.0, z, q->u);
    fill_from_profile(g, bc, YF, F_V, io->z_agl_min, 0.0, z, q->v);
    memset(q->w, 0, sizeof(double) * (size_t)vol);
    double* om = zalloc(g);
    og_omega_from_w(g, q->u, q->v, q->w, z, om, 0);
    for (int j = 0; j < g->ny; ++j) {
        for (int i = 0; i < g->nx; ++i) { om[IX(g, i, j, 0)] = 0; }
    }
    og_w_from_omega(g, q->u, q->v, om, z, q->w);
    /* 2. k from the profile, theta the sounding (one ghost layer), p' = 0 */
    fill_from_profile(g, bc, CC, F_TKE, io->z_agl_min, io->k_decay_height, z, q->tke);
    memset(q->theta, 0, sizeof(double) * (size_t)vol);
    fill_theta_ref(g, bc, z, q->theta);
    memset(q->p, 0, sizeof(double) * (size_t)vol);
    info[0] = info[1] = info[2] = info[3] = info[4] = 0;
    /* 3. O'Brien: w0 from the column continuity, the top residual removed
     * (Source/Initializer.cpp:326-333) */
    if (io->obrien) {
        double* om0 = zalloc(g);
        info[4] = og_obrien_omega(g, q->u, q->v, z, m->ax, m->ay, m->az, m->detJ, om0);
        og_w_from_omega(g, q->u, q->v, om0, z, q->w);
        free(om0);
    }
    int status = 0;
    double* rhs = zalloc(g);
    og_velocity_divergence(g, q->u, q->v, q->w, z, m->ax, m->ay, m->az, m->detJ, rhs);
    info[0] = info[1] = norm2_valid(g, rhs);
    if (io->projection) {
        int pbc[6];
        init_poisson_bc(g, bc, pbc);
        /* Sigma = diag(alpha_h^2, alpha_h^2, alpha_v^2): x, y and the cross part
         * of the z-faces carry alpha_h^2, the z part alpha_v^2; the split only
         * when alpha_v != alpha_h (Source/Initializer.cpp:380-403) */
        const double ah2 = io->alpha_h * io->alpha_h, av2 = io->alpha_v * io->alpha_v;
        const int unit = (io->alpha_h == 1 && io->alpha_v == 1);
        const int split = (io->alpha_v != io->alpha_h);
        double* bh = zalloc(g);
        double* bv = zalloc(g);
        for (int64_t n = 0; n < vol; ++n) {
            bh[n] = ah2;
            bv[n] = av2;
        }
        double* AX = zalloc(g);
        double* AY = zalloc(g);
        double* AZ = zalloc(g);
        for (int64_t n = 0; n < vol; ++n) {
            AX[n] = unit ? m->ax[n] : m->ax[n] * ah2;
            AY[n] = unit ? m->ay[n] : m->ay[n] * ah2;
            AZ[n] = unit ? m->az[n] : m->az[n] * av2;
        }
        const gb_poisson_opts* po = &io->poisson;
        og_mg* mg = og_mg_create(g, pbc, z, m->detJ, AX, AY, AZ, po->max_levels, po->min_coarse, po->nu1, po->nu2,
                                 po->nu_coarse);
        if (split) { og_mg_set_cross(mg, m->az, bv, bh); }
        double* lam = zalloc(g);
        double res[3];
        const int it = og_poisson_solve(mg, rhs, lam, po->reltol, po->abstol, po->max_iter, po->restart, 1, res);
        og_mg_destroy(mg);
        if (it < 0) { status = -2; }
        info[2] = it;
        info[3] = res[1];
        double* F[3] = {zalloc(g), zalloc(g), zalloc(g)};
        og_poisson_fluxes(g, pbc, z, lam, unit ? NULL : bh, unit ? NULL : bh, unit ? NULL : bv, F[0], F[1], F[2]);
        if (split) {
            double* d = zalloc(g);
            for (int64_t n = 0; n < vol; ++n) { d[n] = bv[n] - bh[n]; }
            og_poisson_cross_flux(g, pbc, d, z, lam, F[2]);
            free(d);
        }
        og_omega_from_w(g, q->u, q->v, q->w, z, om, 0);
        double* tgt[3] = {q->u, q->v, om};
        const int tt[3] = {XF, YF, ZF};
        for (int c = 0; c < 3; ++c) {
            for (int k = 0; k < ext(g, tt[c], 2); ++k) {
                for (int j = 0; j < ext(g, tt[c], 1); ++j) {
                    for (int i = 0; i < ext(g, tt[c], 0); ++i) { tgt[c][IX(g, i, j, k)] += F[c][IX(g, i, j, k)]; }
                }
            }
        }
        fill_periodic2(g, XF, q->u);
        fill_periodic2(g, YF, q->v);
        og_w_from_omega(g, q->u, q->v, om, z, q->w);
        og_velocity_divergence(g, q->u, q->v, q->w, z, m->ax, m->ay, m->az, m->detJ, rhs);
        info[1] = norm2_valid(g, rhs);
        for (int c = 0; c < 3; ++c) { free(F[c]); }
        free(bh);
        free(bv);
        free(AX);
        free(AY);
        free(AZ);
        free(lam);
    }
    free(rhs);
    free(om);
    return status;
}

/* The first steps of SimplecStage::iterate (Simplec.cpp:452-506) one at a
 * time, for the tests of the stage's stand-alone entry points
 * (momentum_predictor, pressure_correction, scalar_sweep): the ghost fill
 * with the wall state and the residual at q (into R), the momentum predictor
 * (Predictor.cpp:129-405; pinfo[6], ap[3], dd[3]), the ghost fill and the
 * pressure correction with the predictor's denominators (Simplec.cpp:134-220;
 * cinfo[8]), then the scalar sweeps (Simplec.cpp:222-281) of theta with
 * R_theta as the residual left it and of k, each after a ghost fill, with the
 * transport fluxes of the corrected state (sinfo: max |dtheta|, its last
 * sweep, max |dk|, its last sweep, cells clipped). snap (7 arrays, or NULL)
 * receives u, v, w after the predictor and u, v, w, p after the correction. */
int og_stage_steps(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const gb_simplec_opts* so, gb_state* q,
                   const gb_mesh_fields* m, const gb_diffusivities* df, const double* dtau, double** R, double** ap,
                   double** dd, double** snap, double* pinfo, double* cinfo, double* sinfo)
{
    const int64_t vol = VOL(g);
    double* cfl[N_CF] = {0};
    double* ssl[N_SS] = {0};
    og_turb tcv = {NULL, NULL};
    if (ph->closure) {
        for (int n = 0; n < N_CF; ++n) { cfl[n] = zalloc(g); }
        tcv.cf = cfl;
    }
    if (bc->face[2] == GB_FACE_SURFACE_LAYER) {
        for (int n = 0; n < N_SS; ++n) { ssl[n] = palloc(g); }
        tcv.ss = ssl;
    }
    const og_turb* tc = &tcv;
    og_fill_ghosts2(g, bc, ph, m->z0, q->u, q->v, q->w, q->p, q->theta, q->tke, q->z_nd, (double**)tc->ss);
    residual_t(g, bc, ph, q, m, df, R, tc);
    double* F[3] = {zalloc(g), zalloc(g), zalloc(g)};
    og_transport_fluxes(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, F[0], F[1], F[2]);
    double* dcc = zalloc(g);
    memcpy(dcc, dtau, sizeof(double) * vol);
    double* dtf[3] = {zalloc(g), zalloc(g), zalloc(g)};
    og_face_dtau(g, dcc, dtf[0], dtf[1], dtf[2]);
    og_momentum_predictor(g, bc, ph, so, q, R, F[0], F[1], F[2], dtf, m, df, tc, ap, dd, pinfo);
    if (snap) {
        memcpy(snap[0], q->u, sizeof(double) * vol);
        memcpy(snap[1], q->v, sizeof(double) * vol);
        memcpy(snap[2], q->w, sizeof(double) * vol);
    }
    og_fill_ghosts2(g, bc, ph, m->z0, q->u, q->v, q->w, q->p, q->theta, q->tke, q->z_nd, NULL);
    const int st = og_pressure_correction(g, bc, so, q, dd, m, cinfo);
    if (snap) {
        memcpy(snap[3], q->u, sizeof(double) * vol);
        memcpy(snap[4], q->v, sizeof(double) * vol);
        memcpy(snap[5], q->w, sizeof(double) * vol);
        memcpy(snap[6], q->p, sizeof(double) * vol);
    }
    og_fill_ghosts2(g, bc, ph, m->z0, q->u, q->v, q->w, q->p, q->theta, q->tke, q->z_nd, NULL);
    og_transport_fluxes(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, F[0], F[1], F[2]);
    double last;
    int64_t clipped = 0;
    sinfo[0] = og_scalar_sweep(g, bc, ph, so, F_THETA, q->theta, R[4], F[0], F[1], F[2], q->z_nd, m->detJ, df, tc,
                               dtau, 0, 0, &last, &clipped);
    sinfo[1] = last;
    og_fill_ghosts2(g, bc, ph, m->z0, q->u, q->v, q->w, q->p, q->theta, q->tke, q->z_nd, NULL);
    og_transport_fluxes(g, q->u, q->v, q->w, q->z_nd, m->ax, m->ay, F[0], F[1], F[2]);
    sinfo[2] = og_scalar_sweep(g, bc, ph, so, F_TKE, q->tke, R[5], F[0], F[1], F[2], q->z_nd, m->detJ, df, tc, dtau,
                               so->tke_floor, 1, &last, &clipped);
    sinfo[3] = last;
    sinfo[4] = (double)clipped;
    for (int c = 0; c < 3; ++c) {
        free(F[c]);
        free(dtf[c]);
    }
    free(dcc);
    for (int n = 0; n < N_CF; ++n) { free(cfl[n]); }
    for (int n = 0; n < N_SS; ++n) { free(ssl[n]); }
    return st;
}
