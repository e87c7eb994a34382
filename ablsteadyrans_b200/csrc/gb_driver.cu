// The steady driver on the host (gust::Driver::step, Source/Driver.cpp:
// 403-468; gust::SteadyCriterion, Source/SteadyCriterion.cpp:96-224 without
// the monitor window; gust::ser_cfl, Source/PseudoTime.cpp:53-61), and a
// runner that drives many independent stages from native threads.
//
// Per step: the local dtau at the current CFL, one SIMPLEC iteration, the
// scaled residual norms into the criterion. r_n = max over equations of
// res / max(res_ref, residual_tol) after the reference hold (res_ref: each
// residual's largest value over the first residual_ref_iterations); steady
// when every residual is below residual_tol and has dropped
// residual_drop_orders orders below its reference; otherwise the next CFL
// from the SER law.
#include "gb_simplec.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <new>
#include <thread>
#include <vector>

struct gb_driver {
    gb_simplec* stage{nullptr};
    gb_state q{};
    gb_driver_opts opt{};
    double* dtau{nullptr};
    double cfl{1};
    int iterations{0};
    bool nonfinite{false};
    double res_ref[6]{};
    ~gb_driver()
    {
        if (dtau) { cudaFree(dtau); }
    }
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
    for (int n = 0; n < 6; ++n) {
        if (!std::isfinite(res[n])) {
            d->nonfinite = true;
            *verdict = GB_DRIVER_DIVERGED;
            return GB_OK;
        }
    }
    if (d->iterations == 1) {
        for (int n = 0; n < 6; ++n) { d->res_ref[n] = res[n]; }
    } else if (d->iterations <= o.residual_ref_iterations) {
        for (int n = 0; n < 6; ++n) { d->res_ref[n] = std::max(d->res_ref[n], res[n]); }
    }
    double r = 1.0;
    bool steady = false;
    if (d->iterations > o.residual_ref_iterations) {
        r = 0;
        steady = true;
        const double drop = std::pow(10.0, -o.residual_drop_orders);
        for (int n = 0; n < 6; ++n) {
            const double ref = std::max(d->res_ref[n], o.residual_tol);
            r = std::max(r, std::fabs(res[n]) / ref);
            if (!(res[n] < o.residual_tol) || !(res[n] <= ref * drop)) { steady = false; }
        }
    }
    if (steady) {
        *verdict = GB_DRIVER_STEADY;
        return GB_OK;
    }
    d->cfl = ser_cfl(d->cfl, r, o);
    *verdict = GB_DRIVER_RUNNING;
    return GB_OK;
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
    if (bad(o->residual_tol, o->residual_tol > 0)) {
        gb::set_error("gust: steady.residual_tol must be finite and > 0");
        return GB_BAD_ARG;
    }
    if (bad(o->residual_drop_orders, o->residual_drop_orders >= 0 && o->residual_drop_orders <= 300)) {
        gb::set_error("gust: steady.residual_drop_orders must be >= 0 and <= 300");
        return GB_BAD_ARG;
    }
    if (o->residual_ref_iterations < 1) {
        gb::set_error("gust: steady.residual_ref_iterations must be >= 1");
        return GB_BAD_ARG;
    }
    gb_driver* d = new (std::nothrow) gb_driver;
    if (d == nullptr) {
        gb::set_error("gust: Driver: out of host memory");
        return GB_OOM;
    }
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
