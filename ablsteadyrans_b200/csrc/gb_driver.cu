// The steady driver on the host (gust::Driver::step, Source/Driver.cpp:
// 403-468, with seed_reference, release_reference_hold and start_cfl,
// :275-313; gust::ser_cfl, Source/PseudoTime.cpp:53-61), and a runner that
// drives many independent stages from native threads.
//
// Per step: the local dtau at the current CFL, one SIMPLEC iteration, the
// scaled residual norms and the monitors into the steady criterion
// (gb_criterion). r_n = max over equations of |res| / max(res_ref,
// residual_tol) after the reference hold (1 during it); the next CFL is
// cfl0 during the hold, then the SER law.
#include "gb_simplec.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <new>
#include <string>
#include <thread>
#include <vector>

namespace gb {
gb_criterion* criterion_new(const gb_driver_opts& o, int n_res, const char* const* res_names, int n_mon,
                            const char* const* mon_names, const double* mon_scales);
void criterion_add(gb_criterion* c, const double* res, const double* mon);
int criterion_verdict(const gb_criterion* c, bool* residuals_met, bool* monitors_met, std::vector<std::string>* why);
bool criterion_seed(gb_criterion* c, const double* ref);
}  // namespace gb

struct gb_driver {
    gb_simplec* stage{nullptr};
    gb_state q{};
    gb_driver_opts opt{};
    double* dtau{nullptr};
    double cfl{1};
    double r_last{0};
    int iterations{0};
    int hold{-1};              // -1: residual_ref_iterations (Driver::hold_iterations)
    int n_mon{2};
    bool nonfinite{false};
    gb_criterion* crit{nullptr};
    ~gb_driver()
    {
        if (dtau) { cudaFree(dtau); }
        gb_criterion_destroy(crit);
    }
    int hold_iterations() const { return hold < 0 ? opt.residual_ref_iterations : hold; }
};

namespace {

//! Source/PseudoTime.cpp:53-61: min(cfl_max, growth cfl, cfl0 r^-p).
double ser_cfl(double cfl, double r, const gb_driver_opts& o)
{
    const double capped = std::min(o.cfl_max, o.ser_max_growth * cfl);
    if (o.ser_exponent == 0) { return std::min(capped, o.cfl0); }
    const double r_min = std::pow(o.cfl0 / o.cfl_max, 1.0 / o.ser_exponent);
    if (!(r > r_min)) { return capped; }
    return std::min(capped, o.cfl0 * std::pow(r, -o.ser_exponent));
}

gb_status driver_step(gb_driver* d, int32_t* verdict, gb_iter_info* info_out, double* cfl_out)
{
    const gb_driver_opts& o = d->opt;
    if (cfl_out) { *cfl_out = d->cfl; }
    gb_status st = gb_local_dtau(d->stage, &d->q, d->cfl, d->dtau);
    if (st != GB_OK) { return st; }
    gb_iter_info info{};
    st = gb_simplec_iterate(d->stage, &d->q, d->dtau, &info);
    ++d->iterations;
    if (st == GB_NONFINITE) {
        d->nonfinite = true;
        *verdict = GB_DRIVER_DIVERGED;
        return GB_OK;
    }
    if (st != GB_OK) { return st; }
    if (info_out) { *info_out = info; }
    const double* res = info.residual_norms;
    const double mon[3] = {info.max_speed, info.mean_tke, info.mean_ustar};
    gb::criterion_add(d->crit, res, mon);
    gb_steady_history h{};
    gb_criterion_history(d->crit, &h);
    if (h.nonfinite) {
        d->nonfinite = true;
        *verdict = GB_DRIVER_DIVERGED;
        return GB_OK;
    }
    double r = 1.0;
    if (h.count > d->hold_iterations()) {
        r = 0;
        for (int n = 0; n < 6; ++n) { r = std::max(r, std::fabs(res[n]) / std::max(h.res_ref[n], o.residual_tol)); }
    }
    d->r_last = r;
    bool rm = false, mm = false;
    const int v = gb::criterion_verdict(d->crit, &rm, &mm, nullptr);
    if (v == GB_STEADY) {
        *verdict = GB_DRIVER_STEADY;
        return GB_OK;
    }
    // the confidence stop (Driver.cpp:453-477): the residual criterion met
    // cell by cell on steady.confidence of the cells (and, with
    // confidence_height, on every cell above it), every monitor met
    if (o.confidence > 0 && v == GB_NOT_STEADY && h.count > d->hold_iterations() && mm) {
        const double drop = std::pow(10.0, -o.residual_drop_orders);
        double t[6];
        for (int n = 0; n < 6; ++n) { t[n] = std::min(o.residual_tol, std::max(h.res_ref[n], o.residual_tol) * drop); }
        double share = 0, height = 0;
        if ((st = gb_simplec_confidence(d->stage, t, &share, &height)) != GB_OK) { return st; }
        if (share >= o.confidence && (o.confidence_height == 0 || height <= o.confidence_height)) {
            *verdict = GB_DRIVER_STEADY;
            return GB_OK;
        }
    }
    d->cfl = (h.count <= d->hold_iterations()) ? o.cfl0 : ser_cfl(d->cfl, r, o);
    *verdict = GB_DRIVER_RUNNING;
    return GB_OK;
}

bool before_first(const gb_driver* d, const char* what)
{
    if (d->iterations != 0) {
        gb::set_error("gust: Driver::%s: only before the first iteration", what);
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

gb_status gb_driver_options_default(gb_driver_opts* o, int32_t line_sweep)
{
    gb::clear_error();
    if (o == nullptr) {
        gb::set_error("gust: gb_driver_options_default: null argument");
        return GB_BAD_ARG;
    }
    o->cfl0 = 1.0;
    o->cfl_max = (line_sweep == 1) ? 8.0 : 10.0;   // default_cfl_max (Source/Driver.cpp:133-136)
    o->ser_exponent = 1.0;
    o->ser_max_growth = 2.0;
    o->residual_tol = 5.0e-5;
    o->residual_drop_orders = 4.0;
    o->residual_ref_iterations = 5;
    o->monitor_rel_tol = 1.0e-3;
    o->monitor_window = 50;
    o->confidence = 0.0;
    o->confidence_height = 0.0;
    return GB_OK;
}

gb_status gb_driver_create(gb_simplec* s, const gb_state* q, const gb_driver_opts* o, gb_driver** out)
{
    gb::clear_error();
    if (s == nullptr || q == nullptr || o == nullptr || out == nullptr) {
        gb::set_error("gust: Driver: null argument");
        return GB_BAD_ARG;
    }
    // range checks (Source/Driver.cpp:56-90, Source/SteadyCriterion.cpp:26-48)
    auto bad = [](double x, bool ok) { return std::isnan(x) || !std::isfinite(x) || !ok; };
    if (bad(o->cfl0, o->cfl0 > 0)) { gb::set_error("gust: invalid inputs:\n  steady.cfl0 = %g: must be finite and > 0", o->cfl0); return GB_BAD_ARG; }
    if (bad(o->cfl_max, o->cfl_max >= o->cfl0)) {
        gb::set_error("gust: invalid inputs:\n  steady.cfl_max = %g: must be finite and >= steady.cfl0", o->cfl_max);
        return GB_BAD_ARG;
    }
    if (bad(o->ser_exponent, o->ser_exponent >= 0)) {
        gb::set_error("gust: invalid inputs:\n  steady.ser_exponent = %g: must be finite and >= 0", o->ser_exponent);
        return GB_BAD_ARG;
    }
    if (bad(o->ser_max_growth, o->ser_max_growth >= 1)) {
        gb::set_error("gust: invalid inputs:\n  steady.ser_max_growth = %g: must be finite and >= 1", o->ser_max_growth);
        return GB_BAD_ARG;
    }
    if (bad(o->confidence, o->confidence == 0 || (o->confidence > 0 && o->confidence <= 1))) {
        gb::set_error("gust: invalid inputs:\n  steady.confidence = %g: must be 0 (off) or finite, > 0 and <= 1", o->confidence);
        return GB_BAD_ARG;
    }
    if (bad(o->confidence_height, o->confidence_height >= 0)) {
        gb::set_error("gust: invalid inputs:\n  steady.confidence_height = %g: must be 0 (anywhere) or finite and > 0 (m)",
                      o->confidence_height);
        return GB_BAD_ARG;
    }
    if (o->confidence == 0 && o->confidence_height > 0) {
        gb::set_error("gust: invalid inputs:\n  steady.confidence_height has no effect without steady.confidence > 0");
        return GB_BAD_ARG;
    }
    // the criterion's residuals and monitors (stage_residual_names,
    // stage_monitor_specs: Source/Simplec.cpp:363-371)
    static const char* const kRes[6] = {"u", "v", "w", "p", "theta", "tke"};
    static const char* const kMon[3] = {"max_speed", "mean_tke", "mean_ustar"};
    const gb_physics& ph = gb::simplec_physics(s);
    const double scales[3] = {ph.scale_velocity, ph.scale_tke, 0.1};
    const int n_mon = gb::simplec_has_wall(s) ? 3 : 2;
    gb_criterion* crit = gb::criterion_new(*o, 6, kRes, n_mon, kMon, scales);
    if (crit == nullptr) { return GB_BAD_ARG; }
    gb_driver* d = new (std::nothrow) gb_driver;
    if (d == nullptr) {
        gb_criterion_destroy(crit);
        gb::set_error("gust: Driver: out of host memory");
        return GB_OOM;
    }
    d->crit = crit;
    d->n_mon = n_mon;
    d->stage = s;
    d->q = *q;
    d->opt = *o;
    d->cfl = o->cfl0;
    const int64_t vol = gb::volume(gb::simplec_grid(s));
    if (cudaMalloc(&d->dtau, sizeof(double) * vol) != cudaSuccess) {
        cudaGetLastError();
        delete d;
        gb::set_error("gust: Driver: cannot allocate the local dtau");
        return GB_OOM;
    }
    *out = d;
    return GB_OK;
}

gb_status gb_driver_criterion(gb_driver* d, gb_criterion** c)
{
    gb::clear_error();
    if (d == nullptr || c == nullptr) {
        gb::set_error("gust: Driver::criterion: null argument");
        return GB_BAD_ARG;
    }
    *c = d->crit;
    return GB_OK;
}

gb_status gb_driver_seed_reference(gb_driver* d, const double* ref)
{
    gb::clear_error();
    if (d == nullptr || ref == nullptr) {
        gb::set_error("gust: Driver::seed_reference: null argument");
        return GB_BAD_ARG;
    }
    if (!before_first(d, "seed_reference")) { return GB_BAD_ARG; }
    return gb::criterion_seed(d->crit, ref) ? GB_OK : GB_BAD_ARG;
}

gb_status gb_driver_release_hold(gb_driver* d)
{
    gb::clear_error();
    if (d == nullptr) {
        gb::set_error("gust: Driver::release_reference_hold: null argument");
        return GB_BAD_ARG;
    }
    if (!before_first(d, "release_reference_hold")) { return GB_BAD_ARG; }
    gb_steady_history h{};
    gb_criterion_history(d->crit, &h);
    bool seeded = false;
    for (int n = 0; n < h.n_residuals; ++n) { seeded = seeded || h.res_ref[n] > 0; }
    if (!seeded) {
        gb::set_error("gust: Driver::release_reference_hold: the reference is not seeded (seed_reference first)");
        return GB_BAD_ARG;
    }
    d->hold = 0;
    return GB_OK;
}

gb_status gb_driver_start_cfl(gb_driver* d, double cfl)
{
    gb::clear_error();
    if (d == nullptr) {
        gb::set_error("gust: Driver::start_cfl: null argument");
        return GB_BAD_ARG;
    }
    if (!before_first(d, "start_cfl")) { return GB_BAD_ARG; }
    if (d->hold_iterations() > 0) {
        gb::set_error("gust: Driver::start_cfl: the reference hold is on");
        return GB_BAD_ARG;
    }
    if (std::isnan(cfl) || !std::isfinite(cfl) || !(cfl > 0) || cfl > d->opt.cfl_max) {
        gb::set_error("gust: Driver::start_cfl: %.3e is not finite, > 0 and <= steady.cfl_max = %.3e", cfl, d->opt.cfl_max);
        return GB_BAD_ARG;
    }
    d->cfl = std::max(cfl, d->opt.cfl0);
    return GB_OK;
}

gb_status gb_driver_status(const gb_driver* d, int32_t* hold_iterations, double* next_cfl, double* relative_residual)
{
    gb::clear_error();
    if (d == nullptr) {
        gb::set_error("gust: Driver: null argument");
        return GB_BAD_ARG;
    }
    if (hold_iterations) { *hold_iterations = d->hold_iterations(); }
    if (next_cfl) { *next_cfl = d->cfl; }
    if (relative_residual) { *relative_residual = d->r_last; }
    return GB_OK;
}

gb_status gb_driver_destroy(gb_driver* d)
{
    gb::clear_error();
    delete d;
    return gb::check_cuda("gb_driver_destroy");
}

gb_status gb_driver_step(gb_driver* d, int32_t* verdict, gb_iter_info* info, double* cfl)
{
    gb::clear_error();
    if (d == nullptr || verdict == nullptr) {
        gb::set_error("gust: Driver::step: null argument");
        return GB_BAD_ARG;
    }
    if (d->nonfinite) {
        *verdict = GB_DRIVER_DIVERGED;
        return GB_OK;
    }
    return driver_step(d, verdict, info, cfl);
}

gb_status gb_driver_run(gb_driver* const* drivers, int32_t n, int32_t max_iterations, int32_t threads,
                        int32_t* verdicts, int32_t* iterations)
{
    gb::clear_error();
    if (drivers == nullptr || verdicts == nullptr || iterations == nullptr || n < 0 || max_iterations < 0) {
        gb::set_error("gust: gb_driver_run: bad arguments");
        return GB_BAD_ARG;
    }
    for (int i = 0; i < n; ++i) {
        if (drivers[i] == nullptr) {
            gb::set_error("gust: gb_driver_run: driver %d is null", i);
            return GB_BAD_ARG;
        }
        verdicts[i] = GB_DRIVER_RUNNING;
        iterations[i] = 0;
    }
    const int nt = (threads <= 0 || threads > n) ? n : threads;
    std::atomic<int> next{0};
    auto work = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) { return; }
            gb_driver* d = drivers[i];
            cudaSetDevice(gb::simplec_ctx(d->stage)->device);
            int32_t v = GB_DRIVER_RUNNING;
            int it = 0;
            while (v == GB_DRIVER_RUNNING && it < max_iterations) {
                if (gb_driver_step(d, &v, nullptr, nullptr) != GB_OK) {
                    v = GB_DRIVER_FAILED;
                }
                ++it;
            }
            verdicts[i] = v;
            iterations[i] = it;
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(nt);
    for (int t = 0; t < nt; ++t) { pool.emplace_back(work); }
    for (auto& th : pool) { th.join(); }
    return GB_OK;
}

}  // extern "C"
