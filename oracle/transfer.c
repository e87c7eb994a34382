/*
 * ORACLE -- test infrastructure, not product code. FP64 C restatement of the
 * transfers of grid sequencing (Source/Transfer.cpp): the restriction
 * (restrict_state, :150-286), and for the prolongation the locate/axis
 * arithmetic (:20-84), the bilinear interpolation per zeta-level (:86-108),
 * prolong_fields (:290-320) and prolong_state (:322-385): k clipped at the
 * floor, the fine level's ghost fill, the projection by the pressure
 * correction with d = 1 off the Dirichlet rows, p' restored. Only tests/, the
 * smoke check and the benchmark's CPU legs use it.
 */
#include "og.h"

#include "../include/gust_b200.h"

enum { CC = 0, XF = 1, YF = 2, ZF = 4 };

void og_fill_ghosts2(const og_grid* g, const gb_bc* bc, const gb_physics* ph, const double* z0map, double* u, double* v,
                     double* w, double* p, double* th, double* tk, const double* z, double** ss_out);
int og_pressure_correction(const og_grid* g, const gb_bc* bc, const gb_simplec_opts* so, gb_state* q, double** dd,
                           const gb_mesh_fields* m, double* info);
void og_dirichlet_rows(const og_grid* g, const gb_bc* bc, int f, int t, double* mask);

/* Axis (Transfer.cpp:20-62): where a fine point sits among the coarse ones. */
typedef struct {
    int r, imin, imax, step;
    double lin, inv;
} axis_t;

static axis_t make_axis(int N, int periodic, int r, int nodal)
{
    axis_t a;
    a.r = r;
    a.step = 1;
    a.lin = 1;
    if (nodal) {
        a.imin = 0;
        a.imax = N - 1;
        a.inv = 1.0 / (double)r;
    } else {
        a.inv = 1.0 / (double)(2 * r);
        if (periodic) {
            a.imin = -1;
            a.imax = N - 1;
        } else if (N >= 2) {
            a.imin = 0;
            a.imax = N - 2;
        } else {
            a.imin = 0;
            a.imax = 0;
            a.step = 0;
            a.lin = 0;
        }
    }
    return a;
}

static int floor_div(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

/* locate<Nodal> (Transfer.cpp:70-80), the domains starting at 0. */
static void locate(const axis_t* a, int nodal, int i, int* ic, double* t)
{
    const int den = nodal ? a->r : 2 * a->r;
    const int m = nodal ? i : (2 * i + 1 - a->r);
    int c = floor_div(nodal ? m - 1 : m, den);
    c = c < a->imin ? a->imin : (c > a->imax ? a->imax : c);
    *t = a->lin * (double)(m - den * c) * a->inv;
    *ic = c;
}

static void interpolate(const og_grid* gf, const og_grid* gc, int t, const double* q, double* f, int r)
{
    const int nxn = nodal(t, 0), nyn = nodal(t, 1);
    const axis_t ax = make_axis(gc->nx, gc->periodic_x, r, nxn);
    const axis_t ay = make_axis(gc->ny, gc->periodic_y, r, nyn);
    const int ni = gf->nx + nxn, nj = gf->ny + nyn, nk = gf->nz + nodal(t, 2);
    for (int k = 0; k < nk; ++k) {
        for (int j = 0; j < nj; ++j) {
            for (int i = 0; i < ni; ++i) {
                int I, J;
                double tx, ty;
                locate(&ax, nxn, i, &I, &tx);
                locate(&ay, nyn, j, &J, &ty);
                int I1 = I + ax.step, J1 = J + ay.step;
                /* the coarse image's periodic copies (Transfer.cpp:316-320):
                 * only the coarse valid points are read */
                if (!nxn && gc->periodic_x) {
                    I = (I + gc->nx) % gc->nx;
                    I1 = (I1 + gc->nx) % gc->nx;
                }
                if (!nyn && gc->periodic_y) {
                    J = (J + gc->ny) % gc->ny;
                    J1 = (J1 + gc->ny) % gc->ny;
                }
                const double one = 1;
                f[IX(gf, i, j, k)] = (one - ty) * ((one - tx) * q[IX(gc, I, J, k)] + tx * q[IX(gc, I1, J, k)])
                                   + ty * ((one - tx) * q[IX(gc, I, J1, k)] + tx * q[IX(gc, I1, J1, k)]);
            }
        }
    }
}

/* prolong_fields (Transfer.cpp:290-320): theta, k, p', u, v, w of the fine
 * valid points from the coarse state's valid points, r = the fine-to-coarse
 * ratio. */
void og_prolong_fields(const og_grid* gc, const gb_state* qc, const og_grid* gf, gb_state* qf, int r)
{
    interpolate(gf, gc, CC, qc->theta, qf->theta, r);
    interpolate(gf, gc, CC, qc->tke, qf->tke, r);
    interpolate(gf, gc, CC, qc->p, qf->p, r);
    interpolate(gf, gc, XF, qc->u, qf->u, r);
    interpolate(gf, gc, YF, qc->v, qf->v, r);
    interpolate(gf, gc, ZF, qc->w, qf->w, r);
}

/* prolong_state (Transfer.cpp:322-385): prolong_fields, k raised to
 * tke_floor, the fine ghost fill, the projection (the pressure correction
 * with d = 1 - the Dirichlet mask, alpha_p 1, the Poisson solve to reltol),
 * p' restored. info: [divergence before, after (max norms), Poisson
 * iterations, k cells raised]. Returns the pressure correction's status. */
int og_prolong_state(const og_grid* gc, const gb_state* qc, const og_grid* gf, gb_state* qf, int r, const gb_bc* bc,
                     const gb_physics* ph, const gb_simplec_opts* so, const gb_mesh_fields* m, double reltol,
                     double* info)
{
    og_prolong_fields(gc, qc, gf, qf, r);
    int64_t clipped = 0;
    for (int k = 0; k < gf->nz; ++k) {
        for (int j = 0; j < gf->ny; ++j) {
            for (int i = 0; i < gf->nx; ++i) {
                double* x = &qf->tke[IX(gf, i, j, k)];
                if (*x < so->tke_floor) {
                    *x = so->tke_floor;
                    ++clipped;
                }
            }
        }
    }
    og_fill_ghosts2(gf, bc, ph, m->z0, qf->u, qf->v, qf->w, qf->p, qf->theta, qf->tke, qf->z_nd, NULL);
    const int64_t vol = VOL(gf);
    double* dd[3];
    const int tt[3] = {XF, YF, ZF};
    for (int c = 0; c < 3; ++c) {
        dd[c] = (double*)calloc(vol, sizeof(double));
        og_dirichlet_rows(gf, bc, c, tt[c], dd[c]);
        for (int64_t n = 0; n < vol; ++n) { dd[c][n] = dd[c][n] * -1.0 + 1.0; }
    }
    double* pkeep = (double*)malloc(sizeof(double) * (size_t)vol);
    memcpy(pkeep, qf->p, sizeof(double) * (size_t)vol);
    gb_simplec_opts sp = *so;
    sp.pressure_reltol = reltol;
    sp.alpha_p = 1.0;
    double cinfo[8];
    const int st = og_pressure_correction(gf, bc, &sp, qf, dd, m, cinfo);
    memcpy(qf->p, pkeep, sizeof(double) * (size_t)vol);
    info[0] = cinfo[0];
    info[1] = cinfo[1];
    info[2] = cinfo[7];
    info[3] = (double)clipped;
    for (int c = 0; c < 3; ++c) { free(dd[c]); }
    free(pkeep);
    return st;
}

void og_omega_from_w(const og_grid* g, const double* u, const double* v, const double* w, const double* z, double* om,
                     int ngrow);
void og_w_from_omega(const og_grid* g, const double* u, const double* v, const double* om, const double* z, double* w);

/* restrict_state (Transfer.cpp:199-286): the fine state onto the coarse
 * level r times coarser in x and y. Cell fields: the detJ-weighted means
 * (restrict_cells, :112-132); u, v: the r fine face fluxes summed over r,
 * over the coarse area (restrict_faces, :134-155); Omega: the r x r fine
 * z-face fluxes over r^2, over the coarse a_z (restrict_zfaces, :157-175);
 * w from it with the coarse u and v read with zero-gradient rows
 * (zero_gradient_rows, :177-197). omega_c (may be NULL) receives the coarse
 * Omega. */
void og_restrict_state(const og_grid* gf, const gb_state* qf, const gb_mesh_fields* mf, const og_grid* gc, gb_state* qc,
                       const gb_mesh_fields* mc, int r, double* omega_c)
{
    const double* src[3] = {qf->theta, qf->tke, qf->p};
    double* dst[3] = {qc->theta, qc->tke, qc->p};
    for (int n = 0; n < 3; ++n) {
        for (int k = 0; k < gc->nz; ++k) {
            for (int J = 0; J < gc->ny; ++J) {
                for (int I = 0; I < gc->nx; ++I) {
                    double sjq = 0, sj = 0;
                    for (int b = 0; b < r; ++b) {
                        for (int a = 0; a < r; ++a) {
                            const double w = mf->detJ[IX(gf, r * I + a, r * J + b, k)];
                            sjq += w * src[n][IX(gf, r * I + a, r * J + b, k)];
                            sj += w;
                        }
                    }
                    dst[n][IX(gc, I, J, k)] = sjq / sj;
                }
            }
        }
    }
    const double rinv = 1.0 / (double)r;
    for (int k = 0; k < gc->nz; ++k) {
        for (int J = 0; J < gc->ny; ++J) {
            for (int I = 0; I <= gc->nx; ++I) {
                double s = 0;
                for (int b = 0; b < r; ++b) { s += mf->ax[IX(gf, r * I, r * J + b, k)] * qf->u[IX(gf, r * I, r * J + b, k)]; }
                const double c = s * rinv;
                qc->u[IX(gc, I, J, k)] = c / mc->ax[IX(gc, I, J, k)];
            }
        }
        for (int J = 0; J <= gc->ny; ++J) {
            for (int I = 0; I < gc->nx; ++I) {
                double s = 0;
                for (int b = 0; b < r; ++b) { s += mf->ay[IX(gf, r * I + b, r * J, k)] * qf->v[IX(gf, r * I + b, r * J, k)]; }
                const double c = s * rinv;
                qc->v[IX(gc, I, J, k)] = c / mc->ay[IX(gc, I, J, k)];
            }
        }
    }
    const int64_t vf = VOL(gf), vc = VOL(gc);
    double* omf = (double*)calloc(vf, sizeof(double));
    og_omega_from_w(gf, qf->u, qf->v, qf->w, qf->z_nd, omf, 0);
    double* omc = (double*)calloc(vc, sizeof(double));
    const double r2inv = 1.0 / (double)(r * r);
    for (int k = 0; k <= gc->nz; ++k) {
        for (int J = 0; J < gc->ny; ++J) {
            for (int I = 0; I < gc->nx; ++I) {
                double s = 0;
                for (int b = 0; b < r; ++b) {
                    for (int a = 0; a < r; ++a) {
                        s += mf->az[IX(gf, r * I + a, r * J + b, k)] * omf[IX(gf, r * I + a, r * J + b, k)];
                    }
                }
                const double c = s * r2inv;
                omc[IX(gc, I, J, k)] = c / mc->az[IX(gc, I, J, k)];
            }
        }
    }
    double* u1 = (double*)malloc(sizeof(double) * (size_t)vc);
    double* v1 = (double*)malloc(sizeof(double) * (size_t)vc);
    memcpy(u1, qc->u, sizeof(double) * (size_t)vc);
    memcpy(v1, qc->v, sizeof(double) * (size_t)vc);
    for (int j = 0; j < gc->ny; ++j) {
        for (int i = 0; i <= gc->nx; ++i) {
            u1[IX(gc, i, j, -1)] = u1[IX(gc, i, j, 0)];
            u1[IX(gc, i, j, gc->nz)] = u1[IX(gc, i, j, gc->nz - 1)];
        }
    }
    for (int j = 0; j <= gc->ny; ++j) {
        for (int i = 0; i < gc->nx; ++i) {
            v1[IX(gc, i, j, -1)] = v1[IX(gc, i, j, 0)];
            v1[IX(gc, i, j, gc->nz)] = v1[IX(gc, i, j, gc->nz - 1)];
        }
    }
    og_w_from_omega(gc, u1, v1, omc, qc->z_nd, qc->w);
    if (omega_c) { memcpy(omega_c, omc, sizeof(double) * (size_t)vc); }
    free(omf);
    free(omc);
    free(u1);
    free(v1);
}
