// C ABI of the mesh metrics and the Poisson layer (argument checks, error
// messages in the reference's form; the work is in gb_poisson.cu).
#include "gb_poisson_api.cuh"

#include <cmath>
#include <limits>
#include <new>

namespace {

gb_status need(bool ok, const char* fmt, const char* what)
{
    if (ok) { return GB_OK; }
    gb::set_error(fmt, what);
    return GB_BAD_ARG;
}

}  // namespace

gb_status gb::check_poisson_options(const gb_poisson_opts& o)
{
    const double eps = std::numeric_limits<double>::epsilon();
    if (!std::isfinite(o.reltol) || !(o.reltol >= 10 * eps) || !(o.reltol < 1)) {
        gb::set_error("gust: invalid inputs: solver.poisson_reltol must be >= %g (10 machine epsilon) and < 1", 10 * eps);
        return GB_BAD_ARG;
    }
    if (!std::isfinite(o.abstol) || !(o.abstol >= 0)) {
        gb::set_error("gust: invalid inputs: solver.poisson_abstol must be finite and >= 0");
        return GB_BAD_ARG;
    }
    if (o.max_iter < 1) {
        gb::set_error("gust: invalid inputs: solver.poisson_max_iter must be >= 1");
        return GB_BAD_ARG;
    }
    if (o.restart < 1 || o.restart > 200) {
        gb::set_error("gust: invalid inputs: solver.poisson_restart must be >= 1 (and <= 200 here)");
        return GB_BAD_ARG;
    }
    if (o.precision != 0 && o.precision != 1) {
        gb::set_error("gust: invalid inputs: the Poisson precision must be 0 (FP64) or 1 (FP32 multigrid)");
        return GB_BAD_ARG;
    }
    if (o.nu1 < 0 || o.nu2 < 0 || o.nu_coarse < 1 || o.nu1 + o.nu2 < 1 || o.max_levels < 1
        || o.max_levels > gb::kMaxLevels || o.min_coarse < 1) {
        gb::set_error("gust: invalid inputs: multigrid settings out of range (nu1, nu2 >= 0 with nu1 + nu2 >= 1, "
                      "nu_coarse >= 1, 1 <= max_levels <= %d, min_coarse >= 1)", gb::kMaxLevels);
        return GB_BAD_ARG;
    }
    return GB_OK;
}

namespace {

gb_status check_opts(const gb_poisson_opts& o) { return gb::check_poisson_options(o); }

}  // namespace

extern "C" {

gb_status gb_mesh_metrics(gb_ctx* ctx, const gb_grid* g, const double* z_nd, double* detJ, double* ax, double* ay,
                          double* az, double* z_cc)
{
    gb::clear_error();
    gb_status st = need(ctx != nullptr, "gust: %s: ctx is null", "mesh_metrics");
    if (st == GB_OK) { st = gb::check_grid("mesh_metrics", g); }
    if (st == GB_OK) {
        st = need(z_nd && detJ && ax && ay && az && z_cc, "gust: %s: every array must be a device array of the grid",
                  "mesh_metrics");
    }
    if (st != GB_OK) { return st; }
    return gb::mesh_metrics(ctx, *g, z_nd, detJ, ax, ay, az, z_cc);
}

gb_status gb_face_divergence(gb_ctx* ctx, const gb_grid* g, const double* ax, const double* ay, const double* az,
                             const double* detJ, const double* fx, const double* fy, const double* fz, double* div)
{
    gb::clear_error();
    gb_status st = need(ctx != nullptr, "gust: %s: ctx is null", "face_divergence");
    if (st == GB_OK) { st = gb::check_grid("face_divergence", g); }
    if (st == GB_OK) {
        st = need(ax && ay && az && detJ && fx && fy && fz && div,
                  "gust: %s: F must be face arrays on the mesh's grid", "face_divergence");
    }
    if (st != GB_OK) { return st; }
    return gb::face_divergence(ctx, *g, ax, ay, az, detJ, fx, fy, fz, div);
}

gb_status gb_poisson_options_default(gb_poisson_opts* opt)
{
    gb::clear_error();
    if (opt == nullptr) {
        gb::set_error("gust: gb_poisson_options_default: opt is null");
        return GB_BAD_ARG;
    }
    opt->reltol = 1e-10;
    opt->abstol = 0;
    opt->max_iter = 200;
    opt->restart = 50;
    opt->precision = 0;
    opt->nu1 = 1;
    opt->nu2 = 1;
    opt->nu_coarse = 8;
    opt->max_levels = 12;
    opt->min_coarse = 2;
    return GB_OK;
}

gb_status gb_poisson_create(gb_ctx* ctx, const gb_grid* g, const int32_t* bc, const double* z_nd, const double* detJ,
                            const gb_poisson_opts* opt, gb_poisson** out)
{
    gb::clear_error();
    gb_status st = need(ctx != nullptr && out != nullptr, "gust: %s: ctx and out must not be null", "PoissonSolver");
    if (st == GB_OK) { st = gb::check_grid("PoissonSolver", g); }
    if (st == GB_OK) { st = need(bc != nullptr && z_nd && detJ, "gust: %s: bc, z_nd and detJ are needed", "PoissonSolver"); }
    if (st != GB_OK) { return st; }
    *out = nullptr;
    const char* names[6] = {"xlo", "ylo", "zlo", "xhi", "yhi", "zhi"};
    const int per[3] = {g->periodic_x, g->periodic_y, 0};
    for (int f = 0; f < 6; ++f) {
        const int d = f % 3;
        if (bc[f] < 0 || bc[f] > 2) {
            gb::set_error("gust: invalid inputs:\n  Poisson BC %s: must be periodic, neumann or dirichlet", names[f]);
            return GB_BAD_ARG;
        }
        if ((per[d] != 0) != (bc[f] == GB_POISSON_PERIODIC)) {
            const char* dn[3] = {"x", "y", "z"};
            gb::set_error("gust: invalid inputs:\n  Poisson BC %s: periodic exactly when the domain is periodic in %s",
                          names[f], dn[d]);
            return GB_BAD_ARG;
        }
    }
    gb_poisson_opts o;
    if (opt) {
        o = *opt;
    } else {
        gb_poisson_options_default(&o);
    }
    if ((st = check_opts(o)) != GB_OK) { return st; }
    auto* P = new (std::nothrow) gb_poisson;
    if (P == nullptr) { return GB_OOM; }
    P->ctx = ctx;
    P->g = *g;
    for (int f = 0; f < 6; ++f) { P->bc[f] = bc[f]; }
    P->opt = o;
    P->z_fine = z_nd;
    P->J_fine = detJ;
    st = gb::poisson_build(P);
    if (st != GB_OK) {
        delete P;
        return st;
    }
    *out = P;
    return GB_OK;
}

gb_status gb_poisson_destroy(gb_poisson* p)
{
    gb::clear_error();
    if (p == nullptr) { return GB_OK; }
    cudaStreamSynchronize(p->ctx->stream);
    delete p;
    return gb::check_cuda("PoissonSolver::~PoissonSolver");
}

gb_status gb_poisson_set_coeffs(gb_poisson* p, const double* ax, const double* ay, const double* az, const double* bx,
                                const double* by, const double* bz)
{
    gb::clear_error();
    gb_status st = need(p != nullptr && ax && ay && az, "gust: %s: the solver and the mesh areas are needed",
                        "PoissonSolver::set_coeffs");
    if (st != GB_OK) { return st; }
    return gb::poisson_set_coeffs(p, ax, ay, az, bx, by, bz);
}

gb_status gb_poisson_set_z_cross(gb_poisson* p, const double* az, const double* bz, const double* z_cross)
{
    gb::clear_error();
    gb_status st = need(p != nullptr && (z_cross == nullptr || az != nullptr),
                        "gust: %s: the solver and the z areas are needed", "PoissonSolver::set_z_cross");
    if (st != GB_OK) { return st; }
    return gb::poisson_set_z_cross(p, az, bz, z_cross);
}

gb_status gb_poisson_apply(gb_poisson* p, const double* phi, double* Aphi)
{
    gb::clear_error();
    gb_status st = need(p != nullptr && phi && Aphi, "gust: %s: null argument", "PoissonSolver::apply");
    if (st == GB_OK) { st = need(p->coeffs_set, "gust: %s: call gb_poisson_set_coeffs first", "PoissonSolver::apply"); }
    if (st != GB_OK) { return st; }
    return gb::poisson_apply(p, phi, Aphi);
}

gb_status gb_poisson_vcycle(gb_poisson* p, const double* r, double* e)
{
    gb::clear_error();
    gb_status st = need(p != nullptr && r && e, "gust: %s: null argument", "PoissonSolver::vcycle");
    if (st == GB_OK) { st = need(p->coeffs_set, "gust: %s: call gb_poisson_set_coeffs first", "PoissonSolver::vcycle"); }
    if (st != GB_OK) { return st; }
    return gb::poisson_vcycle(p, r, e);
}

gb_status gb_poisson_solve(gb_poisson* p, double* rhs, double* phi, gb_poisson_result* res)
{
    gb::clear_error();
    gb_status st = need(p != nullptr && rhs && phi && res, "gust: %s: null argument", "PoissonSolver::solve");
    if (st == GB_OK) { st = need(p->coeffs_set, "gust: %s: call gb_poisson_set_coeffs first", "PoissonSolver::solve"); }
    if (st != GB_OK) { return st; }
    return gb::poisson_solve(p, rhs, phi, res);
}

gb_status gb_poisson_fluxes(gb_poisson* p, const double* phi, const double* bx, const double* by, const double* bz,
                            double* fx, double* fy, double* fz)
{
    gb::clear_error();
    gb_status st = need(p != nullptr && phi && fx && fy && fz, "gust: %s: null argument", "PoissonSolver::fluxes");
    if (st != GB_OK) { return st; }
    return gb::poisson_fluxes(p, phi, bx, by, bz, fx, fy, fz);
}

}  // extern "C"
