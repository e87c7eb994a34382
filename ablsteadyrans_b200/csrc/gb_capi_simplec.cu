// C ABI of the SIMPLEC stage: argument and inputs checks with the reference's
// messages (Source/Simplec.cpp:25-48 check_simplec_options,
// Source/BoundaryConditions.cpp check_boundary_inputs), then gb_simplec.cu.
#include "gb_poisson_api.cuh"
#include "gb_simplec.cuh"

#include <cmath>
#include <limits>
#include <new>

// the handle's layout lives in gb_simplec.cu; only the fields the checks need are read here
namespace gb {
gb_status simplec_create_checked(gb_ctx* ctx, const gb_grid* g, const gb_bc* bc, const gb_physics* ph,
                                 const gb_simplec_opts* opt, const double* z_nd, const gb_mesh_fields* mesh,
                                 const gb_diffusivities* df, gb_simplec** out);
void simplec_delete(gb_simplec* S);
}  // namespace gb

namespace {

gb_status check_simplec_options(const gb_simplec_opts& o)
{
    const double eps10 = 10 * std::numeric_limits<double>::epsilon();
    if (std::isnan(o.pressure_reltol) || !(o.pressure_reltol >= eps10 && o.pressure_reltol < 1)) {
        gb::set_error("gust: invalid inputs:\n  simplec.pressure_reltol = %g: must be >= 10 machine epsilon and < 1 "
                      "(the Poisson solver's own bound)", o.pressure_reltol);
        return GB_BAD_ARG;
    }
    if (std::isnan(o.alpha_p) || !(o.alpha_p > 0 && o.alpha_p <= 1)) {
        gb::set_error("gust: invalid inputs:\n  simplec.alpha_p = %g: must be > 0 and <= 1", o.alpha_p);
        return GB_BAD_ARG;
    }
    if (std::isnan(o.rotation_relax) || !(o.rotation_relax > 0 && o.rotation_relax <= 1)) {
        gb::set_error("gust: invalid inputs:\n  simplec.rotation_relax = %g: must be > 0 and <= 1", o.rotation_relax);
        return GB_BAD_ARG;
    }
    if (std::isnan(o.w_vnn_cap) || !(o.w_vnn_cap == 0 || (o.w_vnn_cap >= 16 && std::isfinite(o.w_vnn_cap)))) {
        gb::set_error("gust: invalid inputs:\n  simplec.w_vnn_cap = %g: must be 0 (off), or finite and >= 16", o.w_vnn_cap);
        return GB_BAD_ARG;
    }
    if (std::isnan(o.w_vnn_cap_slope_margin)
        || !(o.w_vnn_cap_slope_margin == 0 || (o.w_vnn_cap_slope_margin >= 1 && std::isfinite(o.w_vnn_cap_slope_margin)))) {
        gb::set_error("gust: invalid inputs:\n  simplec.w_vnn_cap_slope_margin = %g: must be 0 (off), or finite and >= 1",
                      o.w_vnn_cap_slope_margin);
        return GB_BAD_ARG;
    }
    if (o.zline_sweeps < 1 || o.zline_sweeps > 100) {
        gb::set_error("gust: SimplecStage: sweeps must be >= 1 (steady.zline_sweeps; 2..100 for zjacobi)");
        return GB_BAD_ARG;
    }
    if (o.line_sweep != 0 && o.line_sweep != 1) {
        gb::set_error("gust: invalid inputs:\n  steady.sweep = %d: must be zjacobi (0) or lusgs (1)", o.line_sweep);
        return GB_BAD_ARG;
    }
    if (o.line_alternate != 0 && o.line_alternate != 1) {
        gb::set_error("gust: invalid inputs:\n  steady.line_alternate = %d: must be 0 or 1", o.line_alternate);
        return GB_BAD_ARG;
    }
    if (o.line_alternate == 1 && o.line_sweep != 1) {
        gb::set_error("gust: invalid inputs:\n  steady.line_alternate has no effect unless steady.sweep = lusgs");
        return GB_BAD_ARG;
    }
    if (o.line_alternate == 1 && o.zline_sweeps < 2) {
        gb::set_error("gust: invalid inputs:\n  steady.line_alternate = 1 needs steady.zline_sweeps >= 2 (only the odd "
                      "sweeps are reversed)");
        return GB_BAD_ARG;
    }
    if (std::isnan(o.tke_floor) || !(o.tke_floor >= 0)) {
        gb::set_error("gust: SimplecStage: tke_floor must be >= 0 (turb.tke_floor)");
        return GB_BAD_ARG;
    }
    if (o.precision != 0 && o.precision != 1) {
        gb::set_error("gust: SimplecStage: precision must be 0 (plain FP64) or 1 (FP32 inner solves)");
        return GB_BAD_ARG;
    }
    return GB_OK;
}

gb_status check_bc(const gb_grid& g, const gb_bc& bc)
{
    const char* keys[6] = {"bc.xlo", "bc.ylo", "bc.zlo", "bc.xhi", "bc.yhi", "bc.zhi"};
    const int per[3] = {g.periodic_x, g.periodic_y, 0};
    for (int f = 0; f < 6; ++f) {
        const int d = f % 3;
        const int t = bc.face[f];
        if (t < GB_FACE_PERIODIC || t > GB_FACE_SURFACE_LAYER) {
            gb::set_error("gust: invalid inputs:\n  %s: unknown face type %d", keys[f], t);
            return GB_BAD_ARG;
        }
        if (t == GB_FACE_SURFACE_LAYER && f != 2) {
            gb::set_error("gust: invalid inputs:\n  %s = surface_layer: the surface layer is the ground's only "
                          "(bc.zlo)", keys[f]);
            return GB_BAD_ARG;
        }
        if ((per[d] != 0) != (t == GB_FACE_PERIODIC)) {
            gb::set_error("gust: invalid inputs:\n  %s: periodic exactly where the geometry is periodic", keys[f]);
            return GB_BAD_ARG;
        }
        if (d == 2 && (t == GB_FACE_INFLOW || t == GB_FACE_OUTFLOW)) {
            gb::set_error("gust: invalid inputs:\n  %s: inflow and outflow are lateral faces only", keys[f]);
            return GB_BAD_ARG;
        }
    }
    if (bc.theta_ref_n < 1 || bc.theta_ref_n > GB_MAX_PROFILE) {
        gb::set_error("gust: invalid inputs:\n  theta_ref: 1 to %d levels", GB_MAX_PROFILE);
        return GB_BAD_ARG;
    }
    for (int n = 1; n < bc.theta_ref_n; ++n) {
        if (!(bc.theta_ref_z[n] > bc.theta_ref_z[n - 1])) {
            gb::set_error("gust: invalid inputs:\n  theta_ref: heights must increase");
            return GB_BAD_ARG;
        }
    }
    if (bc.face[2] == GB_FACE_SURFACE_LAYER) {
        // check_surface_layer_options (SurfaceLayer.cpp:236-280), the keys bc.surface_*
        auto bad = [](double x) { return std::isnan(x) || !std::isfinite(x); };
        if (bad(bc.surface_z0) || !(bc.surface_z0 > 0)) {
            gb::set_error("gust: invalid inputs:\n  bc.surface_z0 = %g: must be finite and > 0", bc.surface_z0);
            return GB_BAD_ARG;
        }
        if (bad(bc.kappa) || !(bc.kappa > 0) || bad(bc.Cmu0) || !(bc.Cmu0 > 0)) {
            gb::set_error("gust: invalid inputs:\n  the surface layer's kappa and Cmu0 must be finite and > 0");
            return GB_BAD_ARG;
        }
        if (bad(bc.surface_zref)) {
            gb::set_error("gust: invalid inputs:\n  bc.surface_zref = %g: must be finite (<= 0: first cell centre)",
                          bc.surface_zref);
            return GB_BAD_ARG;
        }
        if (bc.surface_stability != GB_SURFACE_NEUTRAL && bc.surface_stability != GB_SURFACE_HEAT_FLUX) {
            gb::set_error("gust: invalid inputs:\n  bc.surface_stability must be neutral or heat_flux");
            return GB_BAD_ARG;
        }
        if (bad(bc.surface_heat_flux)) {
            gb::set_error("gust: invalid inputs:\n  bc.surface_heat_flux = %g: must be finite", bc.surface_heat_flux);
            return GB_BAD_ARG;
        }
        if (bc.surface_stability == GB_SURFACE_NEUTRAL && bc.surface_heat_flux != 0) {
            gb::set_error("gust: invalid inputs:\n  bc.surface_heat_flux is set but the stability is neutral; it would be "
                          "ignored");
            return GB_BAD_ARG;
        }
        if (bc.surface_wall_k != GB_WALL_K_DIRICHLET && bc.surface_wall_k != GB_WALL_K_SOURCE) {
            gb::set_error("gust: invalid inputs:\n  bc.surface_wall_k must be dirichlet or source");
            return GB_BAD_ARG;
        }
        // check_surface_layer_options (SurfaceLayer.cpp:250-292): QNSE's b > 0 and a >= b
        if (bc.surface_qnse != 0 && bc.surface_qnse != 1) {
            gb::set_error("gust: invalid inputs:\n  bc.surface_stable_functions must be businger_dyer or qnse");
            return GB_BAD_ARG;
        }
        if (bc.surface_qnse) {
            const double a[2] = {bc.surface_qnse_am, bc.surface_qnse_ah}, b[2] = {bc.surface_qnse_bm, bc.surface_qnse_bh};
            const char* an[2] = {"qnse_am", "qnse_ah"};
            const char* bn[2] = {"qnse_bm", "qnse_bh"};
            for (int n = 0; n < 2; ++n) {
                if (std::isnan(b[n]) || !(b[n] > 0 && std::isfinite(b[n]))) {
                    gb::set_error("gust: invalid inputs:\n  surface layer %s = %g: must be finite and > 0", bn[n], b[n]);
                    return GB_BAD_ARG;
                }
                if (!(std::isfinite(a[n]) && a[n] >= b[n])) {
                    gb::set_error("gust: invalid inputs:\n  surface layer %s = %g: must be finite and >= %s = %g", an[n], a[n],
                                  bn[n], b[n]);
                    return GB_BAD_ARG;
                }
            }
        } else {
            // With Businger-Dyer a QNSE coefficient other than its default would be
            // ignored, which the reference refuses (SurfaceLayer.cpp:282-288). A zero
            // reads as "not set", so a zero-initialised gb_bc stays valid.
            const double qc[4] = {bc.surface_qnse_am, bc.surface_qnse_bm, bc.surface_qnse_ah, bc.surface_qnse_bh};
            const double qd[4] = {2.5, 0.2, 2.5, 0.2};
            const char* qn[4] = {"qnse_am", "qnse_bm", "qnse_ah", "qnse_bh"};
            for (int n = 0; n < 4; ++n) {
                if (qc[n] != 0.0 && qc[n] != qd[n]) {
                    gb::set_error("gust: invalid inputs:\n  surface layer %s is set but stable_functions is "
                                  "businger_dyer; it would be ignored", qn[n]);
                    return GB_BAD_ARG;
                }
            }
        }
        if (bc.surface_denominator_floor != GB_DENOMINATOR_LOG_LAW && bc.surface_denominator_floor != GB_DENOMINATOR_ONE) {
            gb::set_error("gust: invalid inputs:\n  bc.surface_denominator_floor must be log_law or one");
            return GB_BAD_ARG;
        }
    }
    {
        // the damping checks (BoundaryConditions.cpp:330-357)
        auto bad = [](double x) { return std::isnan(x) || !std::isfinite(x); };
        bool lateral = false;
        for (int f : {0, 1, 3, 4}) { lateral = lateral || bc.face[f] == GB_FACE_INFLOW || bc.face[f] == GB_FACE_OUTFLOW; }
        if (bad(bc.rayleigh_zdamp) || !(bc.rayleigh_zdamp >= 0)) {
            gb::set_error("gust: invalid inputs:\n  bc.rayleigh_zdamp = %g: must be in [0, the top level) (0: off)",
                          bc.rayleigh_zdamp);
            return GB_BAD_ARG;
        }
        if (bad(bc.rayleigh_dampcoef) || !(bc.rayleigh_dampcoef >= 0)) {
            gb::set_error("gust: invalid inputs:\n  bc.rayleigh_dampcoef = %g: must be finite and >= 0 (1/s)",
                          bc.rayleigh_dampcoef);
            return GB_BAD_ARG;
        }
        if (bc.rayleigh_zdamp > 0 && !(bc.rayleigh_dampcoef > 0)) {
            gb::set_error("gust: invalid inputs:\n  bc.rayleigh_zdamp > 0 needs bc.rayleigh_dampcoef > 0");
            return GB_BAD_ARG;
        }
        if (bc.rayleigh_fields < 0 || bc.rayleigh_fields > 31 || bc.rayleigh_above_ground < 0
            || bc.rayleigh_above_ground > 1) {
            gb::set_error("gust: invalid inputs:\n  bc.rayleigh_fields must be among u, v, w, theta, tke and "
                          "bc.rayleigh_height absolute or above_ground");
            return GB_BAD_ARG;
        }
        if (bad(bc.sponge_width) || !(bc.sponge_width >= 0)) {
            gb::set_error("gust: invalid inputs:\n  bc.sponge_width = %g: must be finite and >= 0 (0: off)",
                          bc.sponge_width);
            return GB_BAD_ARG;
        }
        if (bc.sponge_width > 0 && !lateral) {
            gb::set_error("gust: invalid inputs:\n  bc.sponge_width > 0 needs an inflow or outflow face to damp towards");
            return GB_BAD_ARG;
        }
        if (bad(bc.sponge_strength) || !(bc.sponge_strength >= 0)) {
            gb::set_error("gust: invalid inputs:\n  bc.sponge_strength = %g: must be finite and >= 0 (1/s)",
                          bc.sponge_strength);
            return GB_BAD_ARG;
        }
        if (bc.sponge_width > 0 && !(bc.sponge_strength > 0)) {
            gb::set_error("gust: invalid inputs:\n  bc.sponge_width > 0 needs bc.sponge_strength > 0");
            return GB_BAD_ARG;
        }
    }
    bool inflow = false;
    for (int f = 0; f < 6; ++f) { inflow = inflow || bc.face[f] == GB_FACE_INFLOW; }
    // the profile serves the inflow faces and the damping's reference (needs_profile, BoundaryConditions.cpp:287)
    const bool damping = bc.rayleigh_zdamp > 0 || bc.sponge_width > 0;
    if ((inflow || damping) && !(bc.inflow_ustar > 0 && bc.inflow_z0 > 0 && bc.kappa > 0 && bc.Cmu0 > 0)) {
        gb::set_error("gust: invalid inputs:\n  bc.inflow_ustar and bc.inflow_z0 must be > 0 (log law)");
        return GB_BAD_ARG;
    }
    return GB_OK;
}

//! check_closure_options (Closure.cpp:171-210): one message naming the key.
gb_status check_closure(const gb_physics& ph)
{
    if (ph.closure != 0 && ph.closure != 1) {
        gb::set_error("gust: invalid inputs:\n  the closure switch must be 0 (given diffusivities) or 1 (k-L)");
        return GB_BAD_ARG;
    }
    if (!ph.closure) { return GB_OK; }
    auto bad = [](double x) { return std::isnan(x) || !std::isfinite(x); };
    struct Rule {
        const char* key;
        double x;
        bool ok;
        const char* range;
    };
    const double eps = std::numeric_limits<double>::epsilon();
    const Rule rules[] = {
        {"Cmu0", ph.turb_Cmu0, ph.turb_Cmu0 > 0, "finite and > 0"},
        {"Cb", ph.turb_Cb, ph.turb_Cb > 0, "finite and > 0"},
        {"Rt_crit", ph.turb_Rt_crit, ph.turb_Rt_crit <= 0, "finite and <= 0"},
        {"Rt_min", ph.turb_Rt_min, ph.turb_Rt_min < ph.turb_Rt_crit && ph.turb_Rt_min > -3.598,
         "finite, < turb.Rt_crit and > -3.598 (c_mu has its pole at -3.5987)"},
        {"max_geom_lscale", ph.turb_max_geom_lscale, ph.turb_max_geom_lscale > 0, "finite and > 0 (m)"},
        {"tke_floor", ph.turb_tke_floor, ph.turb_tke_floor == 0 || ph.turb_tke_floor >= eps,
         "0 (machine epsilon) or >= machine epsilon (m^2/s^2)"},
        {"sigma_k", ph.turb_sigma_k, ph.turb_sigma_k > 0, "finite and > 0"},
        {"nu_molecular", ph.turb_nu_molecular, ph.turb_nu_molecular >= 0, "finite and >= 0 (m^2/s)"},
        {"alpha_molecular", ph.turb_alpha_molecular, ph.turb_alpha_molecular >= 0, "finite and >= 0 (m^2/s)"},
        {"kappa", ph.turb_kappa, ph.turb_kappa > 0, "finite and > 0"},
        {"ri_gate", ph.turb_ri_gate, ph.turb_ri_gate == 0 || (ph.turb_ri_gate >= 1e-6 && ph.turb_ri_gate <= 1),
         "0 (off) or finite, >= 1e-6 and <= 1"},
        {"nut_relax", ph.turb_nut_relax, ph.turb_nut_relax > 0 && ph.turb_nut_relax <= 1, "finite, > 0 and <= 1"},
        {"realizability", ph.turb_realizability,
         ph.turb_realizability == 0 || (ph.turb_realizability >= 0.01 && ph.turb_realizability <= 10),
         "0 (off) or finite, >= 0.01 and <= 10"},
    };
    for (const Rule& r : rules) {
        if (bad(r.x) || !r.ok) {
            gb::set_error("gust: invalid closure options:\n  turb.%s = %g: must be %s", r.key, r.x, r.range);
            return GB_BAD_ARG;
        }
    }
    return GB_OK;
}

}  // namespace

extern "C" {

gb_status gb_simplec_create(gb_ctx* ctx, const gb_grid* g, const gb_bc* bc, const gb_physics* ph,
                            const gb_simplec_opts* opt, const double* z_nd, const gb_mesh_fields* mesh,
                            const gb_diffusivities* df, gb_simplec** out)
{
    gb::clear_error();
    if (ctx == nullptr || bc == nullptr || ph == nullptr || opt == nullptr || z_nd == nullptr || mesh == nullptr
        || df == nullptr || out == nullptr) {
        gb::set_error("gust: SimplecStage: null argument");
        return GB_BAD_ARG;
    }
    gb_status st = gb::check_grid("SimplecStage", g);
    if (st == GB_OK) { st = check_simplec_options(*opt); }
    if (st == GB_OK) { st = check_bc(*g, *bc); }
    if (st == GB_OK) { st = check_closure(*ph); }
    if (st != GB_OK) { return st; }
    if (!mesh->detJ || !mesh->ax || !mesh->ay || !mesh->az) {
        gb::set_error("gust: SimplecStage: the mesh's detJ, ax, ay and az are needed");
        return GB_BAD_ARG;
    }
    if (!ph->closure && (!df->nu || !df->gamma_theta || !df->gamma_tke)) {
        gb::set_error("gust: SimplecStage: without a closure the residual inputs need the diffusivities");
        return GB_BAD_ARG;
    }
    if (!(ph->scale_velocity > 0 && ph->scale_theta > 0 && ph->scale_tke > 0 && ph->scale_height > 0)) {
        gb::set_error("gust: SimplecStage: the residual scales (jvp_scales) must be finite and > 0");
        return GB_BAD_ARG;
    }
    if (std::isnan(ph->gravity) || !(ph->gravity >= 0) || !(ph->theta0 > 0)) {
        gb::set_error("gust: invalid inputs:\n  forcing.gravity must be >= 0 and forcing.theta0 > 0");
        return GB_BAD_ARG;
    }
    if (ph->coriolis && !(ph->rotation_period > 0 && ph->latitude >= -90 && ph->latitude <= 90)) {
        gb::set_error("gust: invalid inputs:\n  forcing.latitude must be in [-90, 90] and forcing.rotation_period > 0");
        return GB_BAD_ARG;
    }
    if (ph->limiter < GB_LIMITER_VAN_LEER || ph->limiter > GB_LIMITER_UPWIND) {
        gb::set_error("gust: invalid inputs:\n  convection.limiter must be van_leer, van_albada or upwind");
        return GB_BAD_ARG;
    }
    return gb::simplec_create_checked(ctx, g, bc, ph, opt, z_nd, mesh, df, out);
}

gb_status gb_simplec_turbulence(gb_simplec* s, double* const* closure, double* const* surface)
{
    gb::clear_error();
    if (s == nullptr) {
        gb::set_error("gust: SimplecStage: null argument");
        return GB_BAD_ARG;
    }
    return gb::simplec_turbulence(s, closure, surface);
}

gb_status gb_simplec_set_wall_distance(gb_simplec* s, const double* dist)
{
    gb::clear_error();
    if (s == nullptr || dist == nullptr) {
        gb::set_error("gust: SimplecStage::set_wall_distance: null argument");
        return GB_BAD_ARG;
    }
    return gb::simplec_set_wall_distance(s, dist);
}

gb_status gb_simplec_destroy(gb_simplec* s)
{
    gb::clear_error();
    gb::simplec_delete(s);
    return gb::check_cuda("SimplecStage::~SimplecStage");
}

gb_status gb_simplec_fill_ghosts(gb_simplec* s, const gb_state* q)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr) {
        gb::set_error("gust: fill_ghosts: null argument");
        return GB_BAD_ARG;
    }
    gb::simplec_fill_ghosts(s, *q);
    return gb::check_cuda("fill_ghosts");
}

gb_status gb_simplec_prolong(gb_simplec* s, const gb_state* q, const gb_grid* gc, const gb_state* qc, double reltol,
                             gb_prolong_result* r)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || gc == nullptr || qc == nullptr || r == nullptr) {
        gb::set_error("gust: prolong_state: null argument");
        return GB_BAD_ARG;
    }
    gb_status st = gb::check_grid("prolong_state", gc);
    if (st != GB_OK) { return st; }
    const gb_grid& g = gb::simplec_grid(s);
    const int rx = gc->nx > 0 ? g.nx / gc->nx : 0, ry = gc->ny > 0 ? g.ny / gc->ny : 0;
    if (rx < 2 || rx != ry || rx * gc->nx != g.nx || ry * gc->ny != g.ny || (rx & (rx - 1)) != 0 || gc->nz != g.nz
        || gc->periodic_x != g.periodic_x || gc->periodic_y != g.periodic_y) {
        gb::set_error("gust: prolong_state: the levels must satisfy 0 <= fine < coarse: the coarse grid coarser by a "
                      "power of two in x and y, the same layers and periodicity");
        return GB_BAD_ARG;
    }
    if (!std::isfinite(reltol) || !(reltol > 0) || !(reltol < 1)) {
        gb::set_error("gust: invalid inputs:\n  solver.poisson_reltol must be finite, > 0 and < 1");
        return GB_BAD_ARG;
    }
    return gb::simplec_prolong(s, *q, *gc, *qc, reltol, r);
}

gb_status gb_simplec_norms(gb_simplec* s, const gb_state* q, double* residual_norms, double* monitors)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || residual_norms == nullptr || monitors == nullptr) {
        gb::set_error("gust: stage_norms: null argument");
        return GB_BAD_ARG;
    }
    return gb::simplec_norms(s, *q, residual_norms, monitors);
}

gb_status gb_simplec_confidence(gb_simplec* s, const double* thresholds, double* share, double* height)
{
    gb::clear_error();
    if (s == nullptr || thresholds == nullptr || share == nullptr || height == nullptr) {
        gb::set_error("gust: SimplecStage::confidence: null argument");
        return GB_BAD_ARG;
    }
    return gb::simplec_confidence(s, thresholds, share, height);
}

gb_status gb_simplec_implicit_rows(gb_simplec* s, const gb_state* q, int32_t eq, double* A)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || A == nullptr || eq < 0 || eq > 5 || eq == 3) {
        gb::set_error("gust: implicit_rows: the stage, the state, A and an equation among u, v, w, theta, k are needed");
        return GB_BAD_ARG;
    }
    gb::simplec_implicit_rows_at(s, *q, eq, A);
    return gb::check_cuda("implicit_rows");
}

gb_status gb_simplec_residual(gb_simplec* s, const gb_state* q, double* const* R)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || R == nullptr) {
        gb::set_error("gust: residual: null argument");
        return GB_BAD_ARG;
    }
    double* r[6];
    for (int n = 0; n < 6; ++n) {
        if (R[n] == nullptr) {
            gb::set_error("gust: residual: R needs six device arrays (u, v, w, p, theta, tke)");
            return GB_BAD_ARG;
        }
        r[n] = R[n];
    }
    gb::simplec_residual(s, *q, r);
    return gb::check_cuda("residual");
}

gb_status gb_momentum_predictor(gb_simplec* s, const gb_state* q, double* const* R, const double* dtau,
                                double* const* ap, double* const* d, gb_predictor_result* res)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || R == nullptr || dtau == nullptr || res == nullptr) {
        gb::set_error("gust: momentum_predictor: the stage, the state, R, dtau and the result are needed");
        return GB_BAD_ARG;
    }
    for (int n = 0; n < 6; ++n) {
        if (R[n] == nullptr) {
            gb::set_error("gust: momentum_predictor: R needs six device arrays (u, v, w, p, theta, tke)");
            return GB_BAD_ARG;
        }
    }
    return gb::simplec_predictor_step(s, *q, R, dtau, ap, d, res);
}

gb_status gb_pressure_correction(gb_simplec* s, const gb_state* q, const double* const* d, gb_pressure_result* res)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || res == nullptr) {
        gb::set_error("gust: pressure_correction: the stage, the state and the result are needed");
        return GB_BAD_ARG;
    }
    if (d != nullptr && (d[0] == nullptr || d[1] == nullptr || d[2] == nullptr)) {
        gb::set_error("gust: pressure_correction: d needs three device arrays (the u, v, w faces) or none");
        return GB_BAD_ARG;
    }
    return gb::simplec_pressure_step(s, *q, d, res);
}

gb_status gb_scalar_sweep(gb_simplec* s, const gb_state* q, int32_t eq, const double* R_eq, const double* dtau,
                          int32_t clip, gb_scalar_result* res)
{
    gb::clear_error();
    if (eq != 4 && eq != 5) {
        gb::set_error("gust: scalar_sweep: eq must be theta or tke");
        return GB_BAD_ARG;
    }
    if (s == nullptr || q == nullptr || R_eq == nullptr || dtau == nullptr || res == nullptr) {
        gb::set_error("gust: scalar_sweep: the stage, the state, R, dtau and the result are needed");
        return GB_BAD_ARG;
    }
    return gb::simplec_scalar_step(s, *q, eq, R_eq, dtau, clip, res);
}

gb_status gb_simplec_precondition(gb_simplec* s, const gb_state* q, const double* dtau, double inf_cfl,
                                  int32_t denominators, double* const* r, double* const* dq)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || r == nullptr || dq == nullptr) {
        gb::set_error("gust: SimplecPreconditioner: the stage, the state, r and dq are needed");
        return GB_BAD_ARG;
    }
    if (denominators != 1 && denominators != 2) {
        gb::set_error("gust: SimplecPreconditioner: denominators must be 1 (diagonal) or 2 (stage)");
        return GB_BAD_ARG;
    }
    if (dtau == nullptr && (!std::isfinite(inf_cfl) || !(inf_cfl > 0))) {
        gb::set_error("gust: SimplecPreconditioner: inf_cfl = %g: must be finite and > 0 (steady.cfl_max)", inf_cfl);
        return GB_BAD_ARG;
    }
    for (int f = 0; f < 6; ++f) {
        if (r[f] == nullptr || dq[f] == nullptr) {
            gb::set_error("gust: SimplecPreconditioner: r and dq need six device arrays (u, v, w, p, theta, tke)");
            return GB_BAD_ARG;
        }
    }
    gb_status st = gb::simplec_linear_setup(s, *q, dtau, inf_cfl);
    if (st != GB_OK) { return st; }
    const double* rr[6] = {r[0], r[1], r[2], r[3], r[4], r[5]};
    return gb::simplec_linear_apply(s, *q, rr, dq, denominators == 1);
}

gb_status gb_implicit_coefficients(gb_ctx* ctx, const gb_grid* g, int32_t loc, const double* F0, const double* F1,
                                   const double* F2, const double* gamma, const double* z_nd, const double* detJ,
                                   int32_t log_mean, double* A)
{
    gb::clear_error();
    const char* op = "implicit_coefficients";
    if (ctx == nullptr) {
        gb::set_error("gust: %s: ctx is null", op);
        return GB_BAD_ARG;
    }
    gb_status st = gb::check_grid(op, g);
    if (st != GB_OK) { return st; }
    if (loc != GB_LOC_CELL && loc != GB_LOC_XFACE && loc != GB_LOC_YFACE && loc != GB_LOC_ZFACE) {
        gb::set_error("gust: implicit_coefficients: loc must be the cells or a face");
        return GB_BAD_ARG;
    }
    if (F0 == nullptr || F1 == nullptr || F2 == nullptr || gamma == nullptr || z_nd == nullptr || detJ == nullptr
        || A == nullptr) {
        gb::set_error("gust: implicit_coefficients: F, gamma, z_nd, detJ and A must be device arrays of the grid");
        return GB_BAD_ARG;
    }
    double* F[3] = {const_cast<double*>(F0), const_cast<double*>(F1), const_cast<double*>(F2)};
    return gb::implicit_coefficients_at(ctx, *g, loc, F, gamma, z_nd, detJ, log_mean != 0, A);
}

gb_status gb_simplec_iterate(gb_simplec* s, const gb_state* q, const double* dtau, gb_iter_info* info)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || dtau == nullptr || info == nullptr) {
        gb::set_error("gust: SimplecStage::iterate: null argument");
        return GB_BAD_ARG;
    }
    return gb::simplec_iterate(s, *q, dtau, info);
}

gb_status gb_local_dtau(gb_simplec* s, const gb_state* q, double cfl, double* dtau)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || dtau == nullptr) {
        gb::set_error("gust: local_dtau: null argument");
        return GB_BAD_ARG;
    }
    if (std::isnan(cfl) || !std::isfinite(cfl) || !(cfl > 0)) {
        gb::set_error("gust: local_dtau: cfl must be finite and > 0 (got %g)", cfl);
        return GB_BAD_ARG;
    }
    return gb::simplec_local_dtau(s, *q, cfl, dtau);
}

gb_status gb_init_options_default(gb_init_opts* o)
{
    gb::clear_error();
    if (o == nullptr) {
        gb::set_error("gust: gb_init_options_default: null argument");
        return GB_BAD_ARG;
    }
    *o = gb_init_opts{};
    o->z_agl_min = 0.0;
    o->alpha_h = 1.0;
    o->alpha_v = 1.0;
    o->k_decay_height = 0.0;
    o->projection = 1;
    o->obrien = 0;
    return gb_poisson_options_default(&o->poisson);
}

gb_status gb_simplec_initialize(gb_simplec* s, const gb_state* q, const gb_init_opts* o, gb_init_result* r)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || o == nullptr || r == nullptr) {
        gb::set_error("gust: initialize_state: null argument");
        return GB_BAD_ARG;
    }
    // check_init_options (Source/Initializer.cpp:110-140)
    auto bad = [](double x, bool ok) { return std::isnan(x) || !std::isfinite(x) || !ok; };
    if (bad(o->z_agl_min, o->z_agl_min >= 0)) {
        gb::set_error("gust: invalid inputs:\n  init.z_agl_min = %g: must be finite and >= 0 (m)", o->z_agl_min);
        return GB_BAD_ARG;
    }
    if (bad(o->alpha_h, o->alpha_h > 0)) {
        gb::set_error("gust: invalid inputs:\n  init.alpha_h = %g: must be finite and > 0", o->alpha_h);
        return GB_BAD_ARG;
    }
    if (bad(o->alpha_v, o->alpha_v > 0)) {
        gb::set_error("gust: invalid inputs:\n  init.alpha_v = %g: must be finite and > 0", o->alpha_v);
        return GB_BAD_ARG;
    }
    if (bad(o->k_decay_height, o->k_decay_height >= 0)) {
        gb::set_error("gust: invalid inputs:\n  init.k_decay_height = %g: must be finite and >= 0 (m)", o->k_decay_height);
        return GB_BAD_ARG;
    }
    if (o->projection != 0 && o->projection != 1) {
        gb::set_error("gust: init.projection must be 0 or 1");
        return GB_BAD_ARG;
    }
    if (o->obrien != 0 && o->obrien != 1) {
        gb::set_error("gust: init.obrien must be 0 or 1");
        return GB_BAD_ARG;
    }
    gb_status st = gb::check_poisson_options(o->poisson);
    if (st != GB_OK) { return st; }
    return gb::simplec_initialize(s, *q, *o, r);
}

}  // extern "C"
