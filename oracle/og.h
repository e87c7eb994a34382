/*
 * ORACLE -- test infrastructure, not product code. Shared declarations of the
 * FP64 C restatement of the reference's SIMPLEC hot path (see gust_oracle.c).
 */
#ifndef GUST_ORACLE_OG_H_
#define GUST_ORACLE_OG_H_

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct og_grid {
    int32_t nx, ny, nz, ng, periodic_x, periodic_y;
    int64_t sy, sz;
    double dx, dy, dzeta;
} og_grid;

enum { COEF_P = 0, COEF_XM, COEF_XP, COEF_YM, COEF_YP, COEF_ZM, COEF_ZP, N_COEFS };

static inline int64_t IX(const og_grid* g, int i, int j, int k)
{
    return (int64_t)(i + g->ng) + (int64_t)(j + g->ng) * g->sy + (int64_t)(k + g->ng) * g->sz;
}

static inline int64_t VOL(const og_grid* g) { return g->sz * (int64_t)(g->nz + 1 + 2 * g->ng); }

static inline int nodal(int t, int d) { return (t >> d) & 1; }


/* AMReX semantics (gust_oracle.c). */
void og_fill_periodic(const og_grid* g, int t, double* f, int layers);
void og_override_sync(const og_grid* g, int t, double* f);

#endif
