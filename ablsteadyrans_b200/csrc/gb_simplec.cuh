// The SIMPLEC stage's internal entry points (the C ABI wraps them).
#pragma once

#include "gb_common.cuh"

struct gb_simplec;

namespace gb {

gb_status simplec_build(gb_simplec* S);
gb_status simplec_set_wall_distance(gb_simplec* S, const double* dist);
void simplec_delete(gb_simplec* S);
void simplec_fill_ghosts(gb_simplec* S, const gb_state& q);
void simplec_residual(gb_simplec* S, const gb_state& q, double** R);
void simplec_implicit_rows(gb_simplec* S, int eq, double* const* F, double* A);
void simplec_implicit_rows_at(gb_simplec* S, const gb_state& q, int eq, double* A);
gb_status simplec_iterate(gb_simplec* S, const gb_state& q, const double* dtau, gb_iter_info* info);
gb_status simplec_norms(gb_simplec* S, const gb_state& q, double* res, double* mon);
gb_status simplec_predictor_step(gb_simplec* S, const gb_state& q, double* const* R, const double* dtau,
                                 double* const* ap_out, double* const* d_out, gb_predictor_result* res);
gb_status simplec_pressure_step(gb_simplec* S, const gb_state& q, const double* const* d, gb_pressure_result* res);
gb_status simplec_scalar_step(gb_simplec* S, const gb_state& q, int eq, const double* R_eq, const double* dtau,
                              int clip, gb_scalar_result* res);
gb_status simplec_linear_setup(gb_simplec* S, const gb_state& q, const double* dtau, double inf_cfl);
gb_status simplec_linear_apply(gb_simplec* S, const gb_state& q, const double* const* r, double* const* dq,
                               bool diagonal);
gb_status implicit_coefficients_at(gb_ctx* ctx, const gb_grid& g, int loc, double* const* F, const double* gamma,
                                   const double* z, const double* J, int logz, double* A);
gb_status simplec_confidence(gb_simplec* S, const double* thresholds, double* share, double* height);
gb_status simplec_local_dtau(gb_simplec* S, const gb_state& q, double cfl, double* dtau);
gb_status simplec_initialize(gb_simplec* S, const gb_state& q, const gb_init_opts& o, gb_init_result* r);
gb_status simplec_turbulence(gb_simplec* S, double* const* closure, double* const* surface);
gb_status simplec_prolong(gb_simplec* S, const gb_state& q, const gb_grid& gc, const gb_state& qc, double reltol,
                          gb_prolong_result* r);
const gb_grid& simplec_grid(const gb_simplec* S);
gb_ctx* simplec_ctx(const gb_simplec* S);
const gb_physics& simplec_physics(const gb_simplec* S);
//! Whether the ground is a surface-layer face (the wall model's state).
bool simplec_has_wall(const gb_simplec* S);
const gb_simplec_opts& simplec_options(const gb_simplec* S);
//! The convection limiter of the stage's momentum and theta residuals, and
//! its replacement for a while (the Newton stage's smooth counterpart); the
//! stage's graphs never run while it is replaced.
int simplec_limiter(const gb_simplec* S);
void simplec_set_limiter(gb_simplec* S, int limiter);
//! theta_ref at the cell centres (the stage's reference profile).
const double* simplec_theta_ref(const gb_simplec* S);
//! The Dirichlet rows (1, else 0) of velocity component c on its valid faces.
void simplec_dirichlet_rows(gb_simplec* S, int c, double* mask);
//! dtau on the x-, y- and z-faces from the cell dtau (face_dtau, Predictor.H).
void simplec_face_dtau(gb_simplec* S, const double* dtau, double** faces);

}  // namespace gb
