/*
 * ORACLE -- test infrastructure, not product code.
 *
 * A plain-C FP64 CPU restatement of the reference's (hgopalan/ablsteadyrans,
 * "GUST") SIMPLEC hot path, written from the reference's sources and used only
 * as the checker of the CUDA path (tests/, __graft_entry__.smoke()) and as the
 * timed CPU baseline of bench.py. Each function cites the reference file:line
 * it restates. Compiled with -O2 -ffp-contract=off so the arithmetic is the
 * reference's operation order without fused multiply-adds.
 *
 * Layout: the same index space as include/gust_b200.h (every array of a grid
 * has ng ghost layers around the node box, i fastest), so the tests hand the
 * same host arrays to the oracle and, copied, to the GPU. The restatement
 * keeps AMReX's semantics explicit where the CUDA path folds them into index
 * arithmetic: FillBoundary is a ghost copy of periodic images, OverrideSync a
 * copy of the low seam copy onto the high one.
 */
#include "og.h"

void og_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}

int og_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* AMReX semantics used by the reference                               */
/* ------------------------------------------------------------------ */

/* FillBoundary of one ghost layer (the periodic images in x and y) of a field
 * at location t. Ghosts outside a non-periodic face are left alone. x first,
 * then y over the x ghosts (so the corner ghosts are images too). */
static void fill_periodic(const og_grid* g, int t, double* f, int layers)
{
    const int nvx = g->nx + nodal(t, 0), nvy = g->ny + nodal(t, 1), nvz = g->nz + nodal(t, 2);
    for (int k = -layers; k < nvz + layers; ++k) {
        if (k < -g->ng || k > g->nz + g->ng) { continue; }
        if (g->periodic_x) {
            for (int j = 0; j < nvy; ++j) {
                for (int l = 1; l <= layers; ++l) {
                    f[IX(g, -l, j, k)] = f[IX(g, g->nx - l, j, k)];
                    f[IX(g, nvx - 1 + l, j, k)] = f[IX(g, nvx - 1 + l - g->nx, j, k)];
                }
            }
        }
        if (g->periodic_y) {
            for (int i = -layers; i < nvx + layers; ++i) {
                for (int l = 1; l <= layers; ++l) {
                    f[IX(g, i, -l, k)] = f[IX(g, i, g->ny - l, k)];
                    f[IX(g, i, nvy - 1 + l, k)] = f[IX(g, i, nvy - 1 + l - g->ny, k)];
                }
            }
        }
    }
}

/* OverrideSync: the high copy of a periodic seam takes the low copy. */
static void override_sync(const og_grid* g, int t, double* f)
{
    const int nvx = g->nx + nodal(t, 0), nvy = g->ny + nodal(t, 1), nvz = g->nz + nodal(t, 2);
    if (nodal(t, 0) && g->periodic_x) {
        for (int k = 0; k < nvz; ++k) {
            for (int j = 0; j < nvy; ++j) { f[IX(g, g->nx, j, k)] = f[IX(g, 0, j, k)]; }
        }
    }
    if (nodal(t, 1) && g->periodic_y) {
        for (int k = 0; k < nvz; ++k) {
            for (int i = 0; i < nvx; ++i) { f[IX(g, i, g->ny, k)] = f[IX(g, i, 0, k)]; }
        }
    }
}

void og_fill_periodic(const og_grid* g, int t, double* f, int layers) { fill_periodic(g, t, f, layers); }
void og_override_sync(const og_grid* g, int t, double* f) { override_sync(g, t, f); }

/* ------------------------------------------------------------------ */
/* z-line relaxation                                                   */
/* ------------------------------------------------------------------ */

/* Source/LineSolve_K.H:22-45 (solve_column): Thomas forward elimination of
 * (-a_zm, dg, -a_zp) with the x/y neighbour terms of d on the right-hand side,
 * then back substitution into out. */
static void solve_column(const og_grid* g, const double* a, int64_t cs, const double* dg, const double* r,
                         const double* d, double* c, double* e, double* out, int i, int j, int klo, int khi)
{
    for (int k = klo; k <= khi; ++k) {
        const int64_t o = IX(g, i, j, k);
        const double rk = r[o] + a[COEF_XM * cs + o] * d[IX(g, i - 1, j, k)] + a[COEF_XP * cs + o] * d[IX(g, i + 1, j, k)]
                        + a[COEF_YM * cs + o] * d[IX(g, i, j - 1, k)] + a[COEF_YP * cs + o] * d[IX(g, i, j + 1, k)];
        const double lower = -a[COEF_ZM * cs + o], upper = -a[COEF_ZP * cs + o];
        if (k == klo) {
            const double m = dg[o];
            c[o] = upper / m;
            e[o] = rk / m;
        } else {
            const int64_t om = IX(g, i, j, k - 1);
            const double m = dg[o] - lower * c[om];
            c[o] = upper / m;
            e[o] = (rk - lower * e[om]) / m;
        }
    }
    out[IX(g, i, j, khi)] = e[IX(g, i, j, khi)];
    for (int k = khi - 1; k >= klo; --k) { out[IX(g, i, j, k)] = e[IX(g, i, j, k)] - c[IX(g, i, j, k)] * out[IX(g, i, j, k + 1)]; }
}

/* Source/Predictor.cpp:87-127 (zline_jacobi) with check_line_system's
 * delta.setVal(0) (Source/LineSweeps.cpp:391-413): sweeps of column solves with
 * the lagged neighbours (FillBoundary before each sweep), the change of the last
 * sweep, next -> delta, and OverrideSync at the end. Returns the change. */
double og_zline_jacobi(const og_grid* g, int loc, const double* A, const double* ap, const double* rhs, int sweeps,
                       double* delta)
{
    const int64_t vol = VOL(g);
    double* c = (double*)calloc((size_t)vol, sizeof(double));
    double* e = (double*)calloc((size_t)vol, sizeof(double));
    double* next = (double*)calloc((size_t)vol, sizeof(double));
    const int ni = g->nx + nodal(loc, 0), nj = g->ny + nodal(loc, 1), nk = g->nz + nodal(loc, 2);
    memset(delta, 0, sizeof(double) * (size_t)vol);
    double change = 0;
    for (int s = 0; s < sweeps; ++s) {
        fill_periodic(g, loc, delta, 1);
#pragma omp parallel for collapse(2) schedule(static)
        for (int j = 0; j < nj; ++j) {
            for (int i = 0; i < ni; ++i) { solve_column(g, A, vol, ap, rhs, delta, c, e, next, i, j, 0, nk - 1); }
        }
        if (s == sweeps - 1) {
            change = 0;
            for (int k = 0; k < nk; ++k) {
                for (int j = 0; j < nj; ++j) {
                    for (int i = 0; i < ni; ++i) {
                        const double dd = fabs(next[IX(g, i, j, k)] - delta[IX(g, i, j, k)]);
                        if (dd > change || dd != dd) { change = dd; }
                    }
                }
            }
        }
        for (int k = 0; k < nk; ++k) {
            for (int j = 0; j < nj; ++j) {
                for (int i = 0; i < ni; ++i) { delta[IX(g, i, j, k)] = next[IX(g, i, j, k)]; }
            }
        }
    }
    override_sync(g, loc, delta);
    free(c);
    free(e);
    free(next);
    return change;
}

/* ------------------------------------------------------------------ */
/* line LU-SGS                                                         */
/* ------------------------------------------------------------------ */

/* One pass of the line LU-SGS sweep over the columns of the valid box, in
 * place (Source/LineSweeps.cpp:38-171): forward = (+i, +j) or, j-reversed,
 * (+i, -j); backward the opposite pair. order 0 walks the columns
 * sequentially (j outer, i inner), order 1 the wavefront planes
 * (i - ilo) + (j - jlo) = s (or (i - ilo) + (jhi - j) = s reversed), one
 * column after another inside a plane: the two orders give the same values. */
static void lusgs_pass(const og_grid* g, int ni, int nj, int nk, const double* A, int64_t cs, const double* ap,
                       const double* rhs, double* d, double* c, double* e, int forward, int jrev, int order)
{
    if (order == 0) {
        if (forward) {
            for (int jj = 0; jj < nj; ++jj) {
                const int j = jrev ? nj - 1 - jj : jj;
                for (int i = 0; i < ni; ++i) { solve_column(g, A, cs, ap, rhs, d, c, e, d, i, j, 0, nk - 1); }
            }
        } else {
            for (int jj = nj - 1; jj >= 0; --jj) {
                const int j = jrev ? nj - 1 - jj : jj;
                for (int i = ni - 1; i >= 0; --i) { solve_column(g, A, cs, ap, rhs, d, c, e, d, i, j, 0, nk - 1); }
            }
        }
        return;
    }
    const int last = ni + nj - 2;
    for (int q = 0; q <= last; ++q) {
        const int s = forward ? q : last - q;
        const int amin = (s - (nj - 1) > 0) ? s - (nj - 1) : 0;
        const int amax = (s < ni - 1) ? s : ni - 1;
        for (int ia = amin; ia <= amax; ++ia) {
            const int jb = s - ia;
            const int j = jrev ? nj - 1 - jb : jb;
            solve_column(g, A, cs, ap, rhs, d, c, e, d, ia, j, 0, nk - 1);
        }
    }
}

/* Source/LineSweeps.cpp:183-210 (lusgs_lagged) with check_line_system's
 * delta.setVal(0) and zline_lusgs's dispatch (:415-428): `sweeps` symmetric
 * passes; before every pass FillBoundary copies the periodic images of the
 * pass's starting values into the ghosts; with alternate the odd sweeps take
 * the j-reversed pair; the change is max |delta| change over the last
 * backward pass (valid points); OverrideSync at the end. */
double og_zline_lusgs(const og_grid* g, int loc, const double* A, const double* ap, const double* rhs, int sweeps,
                      int order, int alternate, double* delta)
{
    const int64_t vol = VOL(g);
    double* c = (double*)calloc((size_t)vol, sizeof(double));
    double* e = (double*)calloc((size_t)vol, sizeof(double));
    double* before = (double*)calloc((size_t)vol, sizeof(double));
    const int ni = g->nx + nodal(loc, 0), nj = g->ny + nodal(loc, 1), nk = g->nz + nodal(loc, 2);
    memset(delta, 0, sizeof(double) * (size_t)vol);
    double change = 0;
    for (int s = 0; s < sweeps; ++s) {
        for (int forward = 1; forward >= 0; --forward) {
            if (s == sweeps - 1 && !forward) { memcpy(before, delta, sizeof(double) * (size_t)vol); }
            fill_periodic(g, loc, delta, 1);
            lusgs_pass(g, ni, nj, nk, A, vol, ap, rhs, delta, c, e, forward, alternate && (s % 2 == 1), order);
        }
        if (s == sweeps - 1) {
            change = 0;
            for (int k = 0; k < nk; ++k) {
                for (int j = 0; j < nj; ++j) {
                    for (int i = 0; i < ni; ++i) {
                        const double dd = fabs(before[IX(g, i, j, k)] - delta[IX(g, i, j, k)]);
                        if (dd > change || dd != dd) { change = dd; }
                    }
                }
            }
        }
    }
    override_sync(g, loc, delta);
    free(c);
    free(e);
    free(before);
    return change;
}
