// The k-L closure and the surface layer on the GPU (gust::Closure,
// Source/Closure.cpp; gust::compute_surface_state and the wall rows,
// Source/SurfaceLayer.cpp): the SIMPLEC stage calls these when the closure
// is on (gb_physics.closure) or the ground is a surface_layer face.
//
// The closure's fields are ten volumes in the order of kClosure*; the
// surface state is eleven planes (one value per column, column (i, j) at
// (j + ng) sy + i + ng, on the columns -1..nx, -1..ny) in the order of kSs*;
// the wall law's ground gradient is three planes (u, v, theta) on the
// columns -2..nx+1, -2..ny+1.
#pragma once

#include "gb_stencil.cuh"

namespace gb {

enum {
    kClosureNu = 0,
    kClosureGammaTheta,
    kClosureGammaTke,
    kClosureNut,
    kClosureLength,
    kClosureRt,
    kClosurePs,
    kClosurePb,
    kClosureEps,
    kClosureDSdk,
    kClosureFields
};
enum {
    kSsUstar = 0,
    kSsSpeed,
    kSsZref,
    kSsD0,
    kSsInvL,
    kSsTauX,
    kSsTauY,
    kSsTauZ,
    kSsDrag,
    kSsKwall,
    kSsArea,
    kSsPlanes
};

//! One plane of per-column values: the number of doubles.
inline int64_t plane_size(const gb_grid& g) { return g.sy * static_cast<int64_t>(g.ny + 1 + 2 * g.ng); }

__host__ __device__ __forceinline__ int64_t plane_at(const gb_grid& g, int i, int j)
{
    return static_cast<int64_t>((i + g.ng) + (j + g.ng) * static_cast<int32_t>(g.sy));
}

//! The wall law's gradient of column (i, j) for a point of type t on the
//! ground fill (fill_gradient_z, BoundaryConditions.cpp:495-509): the mean
//! of the two columns beside a nodal face point, clamped to the gradient's
//! columns -2..nx+1, -2..ny+1.
__device__ __forceinline__ double ground_gradient_at(const gb_grid& g, const double* __restrict__ gg, int t, int i, int j)
{
    const int lo = -2, hix = g.nx + 1, hiy = g.ny + 1;
    const int ia = min(max(i, lo), hix), ja = min(max(j, lo), hiy);
    const int ib = min(max(st::nodal(t, 0) ? i - 1 : i, lo), hix);
    const int jb = min(max(st::nodal(t, 1) ? j - 1 : j, lo), hiy);
    return 0.5 * (gg[plane_at(g, ib, jb)] + gg[plane_at(g, ia, ja)]);
}

//! height_above_ground (Closure.cpp:270-300) on the cells -1..nx, -1..ny,
//! the vertical ghosts copied.
void turb_height_above_ground(gb_ctx* ctx, const gb_grid& g, const double* z, double* dist);

//! Closure::evaluate (Closure.cpp:365-460) with the weight 1, no cap and no
//! gate, at the state q (ghosts filled): cf[kClosure*].
//! nut_prev: the nu_t of the last accepted iteration (turb.nut_relax < 1
//! blends with it), or null (no history yet: the weight is 1).
void turb_closure(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const gb_physics& ph, const gb_state& q,
                  const double* z, const double* dist, const double* z0map, double* const* cf,
                  const double* nut_prev = nullptr);

//! compute_surface_state's columns (SurfaceLayer.cpp:97-230) into ss; the
//! columns without a positive, finite u* (or with a non-finite k_w) are
//! counted into *bad (device word, added to).
void turb_surface_state(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const gb_physics& ph, const gb_state& q,
                        const double* z, const double* z0map, double* const* ss, unsigned long long* bad);

//! The wall law's gradient planes (BoundaryConditions.cpp:549-648).
void turb_ground_gradients(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const double* const* ss,
                           const double* z0map, double* const* gg);

//! set_ground_fluxes (SurfaceLayer.cpp:418-450) on the ground faces of one
//! z-flux array: field 0 u (the wall stress, the mean of the two columns),
//! 1 v, 2 theta (-q |A|), 3 k (0).
void turb_ground_flux(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const double* const* ss, int field, double* Gz);

//! R_k -= P_s + P_b - eps on the valid cells (Residual.cpp:240-245).
void turb_k_sources(gb_ctx* ctx, const gb_grid& g, const double* const* cf, double* Rk);

//! apply_wall_k (SurfaceLayer.cpp:452-481).
void turb_apply_wall_k(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const double* const* ss, const double* tke,
                       double* Rk);

//! The Patankar diagonal of k added to a_P on the valid cells (Residual.cpp:287-290).
void turb_patankar(gb_ctx* ctx, const gb_grid& g, const double* dSdk, double* A);

//! apply_wall_to_implicit (SurfaceLayer.cpp:483-518) for the rows at loc.
void turb_wall_rows(gb_ctx* ctx, const gb_grid& g, const double* const* ss, int loc, const double* J, double* A);

//! apply_wall_k_to_implicit (SurfaceLayer.cpp:520-569).
void turb_wall_k_rows(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const double* const* ss, double* A);

}  // namespace gb
