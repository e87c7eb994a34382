// The steady criterion and the loose stop of grid sequencing on the host
// (gust::SteadyCriterion, Source/SteadyCriterion.H:13-150, SteadyCriterion.cpp;
// gust::loose_stop and check_sequencing_options, Source/Sequencing.H:97-136,
// Sequencing.cpp:120-222). The steady driver keeps one per stage; the C ABI
// also gives it to callers that drive their own loop.
//
// A history is the count of iterations, each residual's reference (the
// largest of its first residual_ref_iterations values, or a seed raised by
// them), each residual's last value and each monitor's last
// monitor_window + 1 values. Steady: every residual below residual_tol and
// residual_drop_orders orders below its reference (floored at residual_tol),
// and every monitor with a full window that changed over it by at most
// monitor_rel_tol of max(|last|, scale) and whose Aitken extrapolation from
// the window's halves is within the same amount of its limit. A NaN or an
// infinity anywhere is Diverged for good.
#include "gb_common.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <sstream>

struct gb_criterion {
    double residual_tol{5e-5}, drop_orders{4}, monitor_rel_tol{1e-3};
    int ref_iterations{5}, window{50};
    std::vector<std::string> res_names, mon_names;
    std::vector<double> mon_scale;
    int count{0};
    bool nonfinite{false};
    std::string nonfinite_what;
    std::vector<double> res_ref, res_last;
    std::vector<std::vector<double>> mon_hist;
};

namespace {

//! fmt (SteadyCriterion.cpp:14-20): three significant digits.
std::string fmt3(double x)
{
    std::ostringstream os;
    os.precision(3);
    os << x;
    return os.str();
}

//! fmt (Sequencing.cpp:26-31): %.3e.
std::string fmte(double x)
{
    char b[32];
    std::snprintf(b, sizeof(b), "%.3e", x);
    return b;
}

//! validate (SteadyCriterion.cpp:26-48).
std::vector<std::string> validate(const gb_driver_opts& o)
{
    std::vector<std::string> err;
    if (!std::isfinite(o.residual_tol) || !(o.residual_tol > 0)) { err.emplace_back("steady.residual_tol must be finite and > 0"); }
    const int max10 = std::numeric_limits<double>::max_exponent10;
    if (!std::isfinite(o.residual_drop_orders) || !(o.residual_drop_orders >= 0) || !(o.residual_drop_orders <= max10)) {
        err.emplace_back("steady.residual_drop_orders must be >= 0 and <= " + std::to_string(max10));
    }
    if (o.residual_ref_iterations < 1) { err.emplace_back("steady.residual_ref_iterations must be >= 1"); }
    if (!std::isfinite(o.monitor_rel_tol) || !(o.monitor_rel_tol > 0)) {
        err.emplace_back("steady.monitor_rel_tol must be finite and > 0");
    }
    if (o.monitor_window < 2) { err.emplace_back("steady.monitor_window must be >= 2"); }
    return err;
}

std::string joined(const char* head, const std::vector<std::string>& err)
{
    std::string all = head;
    for (const auto& e : err) { all += "\n  " + e; }
    return all;
}

}  // namespace

namespace gb {

gb_criterion* criterion_new(const gb_driver_opts& o, int n_res, const char* const* res_names, int n_mon,
                            const char* const* mon_names, const double* mon_scales)
{
    auto err = validate(o);
    if (n_res < 1 || n_res > GB_CRITERION_MAX_RESIDUALS) {
        err.emplace_back("SteadyCriterion needs from 1 to " + std::to_string(GB_CRITERION_MAX_RESIDUALS) + " residuals");
    }
    if (n_mon < 0 || n_mon > GB_CRITERION_MAX_MONITORS) {
        err.emplace_back("SteadyCriterion takes at most " + std::to_string(GB_CRITERION_MAX_MONITORS) + " monitors");
    }
    for (int m = 0; m < n_mon && n_mon <= GB_CRITERION_MAX_MONITORS; ++m) {
        const double s = mon_scales ? mon_scales[m] : 0.0;
        if (!std::isfinite(s) || !(s > 0)) {
            err.emplace_back(std::string("monitor '") + (mon_names && mon_names[m] ? mon_names[m] : "?")
                             + "': scale must be finite and > 0");
        }
    }
    if (!err.empty()) {
        set_error("%s", joined("gust: invalid steady criterion:", err).c_str());
        return nullptr;
    }
    gb_criterion* c = new (std::nothrow) gb_criterion;
    if (c == nullptr) {
        set_error("gust: SteadyCriterion: out of host memory");
        return nullptr;
    }
    c->residual_tol = o.residual_tol;
    c->drop_orders = o.residual_drop_orders;
    c->ref_iterations = o.residual_ref_iterations;
    c->monitor_rel_tol = o.monitor_rel_tol;
    c->window = o.monitor_window;
    for (int q = 0; q < n_res; ++q) { c->res_names.emplace_back(res_names && res_names[q] ? res_names[q] : "?"); }
    for (int m = 0; m < n_mon; ++m) {
        c->mon_names.emplace_back(mon_names && mon_names[m] ? mon_names[m] : "?");
        c->mon_scale.push_back(mon_scales[m]);
    }
    c->res_ref.assign(n_res, 0.0);
    c->res_last.assign(n_res, 0.0);
    c->mon_hist.assign(n_mon, {});
    return c;
}

//! SteadyCriterion::add (SteadyCriterion.cpp:96-137).
void criterion_add(gb_criterion* c, const double* res, const double* mon)
{
    for (size_t q = 0; q < c->res_names.size(); ++q) {
        const double r = res[q];
        if (!std::isfinite(r)) {
            if (!c->nonfinite) { c->nonfinite_what = "residual '" + c->res_names[q] + "'"; }
            c->nonfinite = true;
            continue;
        }
        if (c->count < c->ref_iterations) { c->res_ref[q] = std::max(c->res_ref[q], std::fabs(r)); }
        c->res_last[q] = std::fabs(r);
    }
    const size_t keep = static_cast<size_t>(c->window) + 1;
    for (size_t m = 0; m < c->mon_names.size(); ++m) {
        const double v = mon[m];
        if (!std::isfinite(v)) {
            if (!c->nonfinite) { c->nonfinite_what = "monitor '" + c->mon_names[m] + "'"; }
            c->nonfinite = true;
            continue;
        }
        auto& h = c->mon_hist[m];
        h.push_back(v);
        if (h.size() > keep) { h.erase(h.begin()); }
    }
    ++c->count;
}

//! SteadyCriterion::verdict (SteadyCriterion.cpp:139-224): the status and
//! the reasons it is not steady, one per line.
int criterion_verdict(const gb_criterion* c, bool* residuals_met, bool* monitors_met, std::vector<std::string>* why)
{
    std::vector<std::string> reasons;
    *residuals_met = false;
    *monitors_met = false;
    if (c->count == 0) {
        reasons.emplace_back("no iterations recorded");
        if (why) { *why = reasons; }
        return GB_NOT_STEADY;
    }
    if (c->nonfinite) {
        reasons.emplace_back(c->nonfinite_what + " became NaN or infinite");
        if (why) { *why = reasons; }
        return GB_DIVERGED;
    }
    const double drop = std::pow(10.0, -c->drop_orders);
    for (size_t q = 0; q < c->res_names.size(); ++q) {
        const double r = c->res_last[q];
        const double ref = std::max(c->res_ref[q], c->residual_tol);
        if (!(r < c->residual_tol)) {
            reasons.emplace_back("residual '" + c->res_names[q] + "' = " + fmt3(r) + " is not below steady.residual_tol = "
                                 + fmt3(c->residual_tol));
        }
        if (!(r <= ref * drop)) {
            const double orders = (r > 0) ? std::log10(ref / r) : 0.0;
            reasons.emplace_back("residual '" + c->res_names[q] + "' dropped " + fmt3(orders)
                                 + " orders, less than steady.residual_drop_orders = " + fmt3(c->drop_orders));
        }
    }
    *residuals_met = reasons.empty();
    const size_t residual_reasons = reasons.size();
    const size_t need = static_cast<size_t>(c->window) + 1;
    for (size_t m = 0; m < c->mon_names.size(); ++m) {
        const auto& h = c->mon_hist[m];
        if (h.size() < need) {
            reasons.emplace_back("monitor '" + c->mon_names[m] + "': " + std::to_string(h.size()) + " of the "
                                 + std::to_string(need) + " values steady.monitor_window needs");
            continue;
        }
        const double last = h.back();
        double change = 0;
        for (const double x : h) { change = std::max(change, std::fabs(x - last)); }
        const double ref = std::max(std::fabs(last), c->mon_scale[m]);
        const double tol = c->monitor_rel_tol * ref;
        if (!(change <= tol)) {
            reasons.emplace_back("monitor '" + c->mon_names[m] + "' changed by " + fmt3(change / ref)
                                 + " of max(|value|, scale) over the last " + std::to_string(c->window)
                                 + " iterations; steady.monitor_rel_tol = " + fmt3(c->monitor_rel_tol));
            continue;
        }
        // Aitken's estimate of the distance to the limit from the changes
        // over the window's two halves (d2 = rho d1): d2 rho / (1 - rho)
        const size_t W = h.size() - 1;
        const size_t half = W / 2;
        const double d1 = h[W - half] - h[W - 2 * half];
        const double d2 = h[W] - h[W - half];
        const double noise = 1.0e-3 * tol;
        if (std::max(std::fabs(d1), std::fabs(d2)) <= noise) { continue; }
        const double rho = (d1 != 0) ? d2 / d1 : std::numeric_limits<double>::infinity();
        if (!(rho > -1 && rho < 1)) {
            reasons.emplace_back("monitor '" + c->mon_names[m]
                                 + "' is not converging over the window (half-window change ratio " + fmt3(rho) + ")");
            continue;
        }
        const double remaining = std::fabs(d2 * rho / (1 - rho));
        if (!(remaining <= tol)) {
            reasons.emplace_back("monitor '" + c->mon_names[m] + "' is an extrapolated " + fmt3(remaining / ref)
                                 + " of max(|value|, scale) from its limit; steady.monitor_rel_tol = "
                                 + fmt3(c->monitor_rel_tol));
        }
    }
    *monitors_met = reasons.size() == residual_reasons;
    if (why) { *why = reasons; }
    return reasons.empty() ? GB_STEADY : GB_NOT_STEADY;
}

//! SteadyCriterion::seed_reference (SteadyCriterion.cpp:85-94).
bool criterion_seed(gb_criterion* c, const double* ref)
{
    bool ok = c->count == 0;
    for (size_t q = 0; q < c->res_ref.size(); ++q) { ok = ok && std::isfinite(ref[q]) && ref[q] >= 0; }
    if (!ok) {
        set_error("gust: SteadyCriterion::seed_reference: needs one finite reference >= 0 per residual, before the "
                  "first iteration");
        return false;
    }
    for (size_t q = 0; q < c->res_ref.size(); ++q) { c->res_ref[q] = ref[q]; }
    return true;
}

//! loose_stop (Sequencing.cpp:172-222): GB_LOOSE_NONE, _RESIDUALS or _MONITORS.
int loose_stop(const gb_criterion* c, const gb_sequencing_opts& o, int hold_iterations)
{
    if (c->count == 0 || c->nonfinite) { return GB_LOOSE_NONE; }
    // (a): after the hold, or on a released seeded level after
    // min(residual_ref_iterations, 3) iterations
    const int first = hold_iterations > 0 ? hold_iterations : std::min(c->ref_iterations, 3);
    if (c->count >= first && !c->res_last.empty()) {
        const double drop = std::pow(10.0, -o.drop_orders);
        bool all = true;
        for (size_t q = 0; q < c->res_last.size(); ++q) {
            const double ref = std::max(c->res_ref[q], c->residual_tol);
            const double r = c->res_last[q];
            all = all && (r <= ref * drop || r < c->residual_tol);
        }
        if (all) { return GB_LOOSE_RESIDUALS; }
    }
    // (b): every monitor within monitor_tol over a full window, not before
    // residual_ref_iterations whatever the hold
    const size_t need = static_cast<size_t>(c->window) + 1;
    if (o.monitor_tol > 0 && c->count >= c->ref_iterations && !c->mon_names.empty()) {
        bool all = true;
        for (size_t m = 0; m < c->mon_names.size() && all; ++m) {
            const auto& w = c->mon_hist[m];
            if (w.size() < need) {
                all = false;
                break;
            }
            const double last = w.back();
            double change = 0;
            for (const double x : w) { change = std::max(change, std::fabs(x - last)); }
            all = change <= o.monitor_tol * std::max(std::fabs(last), c->mon_scale[m]);
        }
        if (all) { return GB_LOOSE_MONITORS; }
    }
    return GB_LOOSE_NONE;
}

std::string loose_reason(int branch, const gb_criterion* c, const gb_sequencing_opts& o)
{
    if (branch == GB_LOOSE_RESIDUALS) { return "every residual " + fmte(o.drop_orders) + " orders below its reference"; }
    if (branch == GB_LOOSE_MONITORS) {
        return "every monitor within " + fmte(o.monitor_tol) + " over " + std::to_string(c->window) + " iterations";
    }
    return "";
}

}  // namespace gb

namespace {

void copy_text(const std::vector<std::string>& lines, char* out, int32_t cap)
{
    if (out == nullptr || cap <= 0) { return; }
    std::string all;
    for (size_t n = 0; n < lines.size(); ++n) { all += (n ? "\n" : "") + lines[n]; }
    const size_t len = std::min(all.size(), static_cast<size_t>(cap - 1));
    std::memcpy(out, all.data(), len);
    out[len] = '\0';
}

}  // namespace

extern "C" {

gb_status gb_criterion_create(const gb_driver_opts* o, int32_t n_residuals, const char* const* residual_names,
                              int32_t n_monitors, const char* const* monitor_names, const double* monitor_scales,
                              gb_criterion** out)
{
    gb::clear_error();
    if (o == nullptr || out == nullptr || (n_monitors > 0 && monitor_scales == nullptr)) {
        gb::set_error("gust: SteadyCriterion: null argument");
        return GB_BAD_ARG;
    }
    gb_criterion* c = gb::criterion_new(*o, n_residuals, residual_names, n_monitors, monitor_names, monitor_scales);
    if (c == nullptr) { return GB_BAD_ARG; }
    *out = c;
    return GB_OK;
}

gb_status gb_criterion_destroy(gb_criterion* c)
{
    gb::clear_error();
    delete c;
    return GB_OK;
}

gb_status gb_criterion_add(gb_criterion* c, const double* residuals, const double* monitors)
{
    gb::clear_error();
    if (c == nullptr || residuals == nullptr || (!c->mon_names.empty() && monitors == nullptr)) {
        gb::set_error("gust: SteadyCriterion::add: null argument (one residual per residual name, one value per monitor)");
        return GB_BAD_ARG;
    }
    gb::criterion_add(c, residuals, monitors);
    return GB_OK;
}

gb_status gb_criterion_seed_reference(gb_criterion* c, const double* ref)
{
    gb::clear_error();
    if (c == nullptr || ref == nullptr) {
        gb::set_error("gust: SteadyCriterion::seed_reference: null argument");
        return GB_BAD_ARG;
    }
    return gb::criterion_seed(c, ref) ? GB_OK : GB_BAD_ARG;
}

gb_status gb_criterion_verdict(const gb_criterion* c, int32_t* status, int32_t* residuals_met, int32_t* monitors_met,
                               char* reasons, int32_t reasons_cap)
{
    gb::clear_error();
    if (c == nullptr || status == nullptr) {
        gb::set_error("gust: SteadyCriterion::verdict: null argument");
        return GB_BAD_ARG;
    }
    bool rm = false, mm = false;
    std::vector<std::string> why;
    *status = gb::criterion_verdict(c, &rm, &mm, &why);
    if (residuals_met) { *residuals_met = rm; }
    if (monitors_met) { *monitors_met = mm; }
    copy_text(why, reasons, reasons_cap);
    return GB_OK;
}

gb_status gb_criterion_history(const gb_criterion* c, gb_steady_history* h)
{
    gb::clear_error();
    if (c == nullptr || h == nullptr) {
        gb::set_error("gust: SteadyCriterion::history: null argument");
        return GB_BAD_ARG;
    }
    *h = gb_steady_history{};
    h->count = c->count;
    h->nonfinite = c->nonfinite ? 1 : 0;
    h->n_residuals = static_cast<int32_t>(c->res_ref.size());
    h->n_monitors = static_cast<int32_t>(c->mon_names.size());
    for (size_t q = 0; q < c->res_ref.size(); ++q) {
        h->res_ref[q] = c->res_ref[q];
        h->res_last[q] = c->res_last[q];
    }
    for (size_t m = 0; m < c->mon_hist.size(); ++m) {
        h->monitor_values[m] = static_cast<int32_t>(c->mon_hist[m].size());
        if (!c->mon_hist[m].empty()) { h->monitor_last[m] = c->mon_hist[m].back(); }
    }
    return GB_OK;
}

gb_status gb_criterion_monitor_window(const gb_criterion* c, int32_t m, double* values, int32_t cap, int32_t* n)
{
    gb::clear_error();
    if (c == nullptr || n == nullptr || m < 0 || m >= static_cast<int32_t>(c->mon_hist.size())) {
        gb::set_error("gust: SteadyCriterion: no monitor %d", m);
        return GB_BAD_ARG;
    }
    const auto& w = c->mon_hist[m];
    *n = static_cast<int32_t>(w.size());
    for (int32_t k = 0; k < *n && k < cap && values; ++k) { values[k] = w[k]; }
    return GB_OK;
}

gb_status gb_sequencing_check(const gb_sequencing_opts* o, const gb_driver_opts* strict, int32_t nx, int32_t ny,
                              int32_t hierarchy_levels)
{
    gb::clear_error();
    if (o == nullptr || strict == nullptr) {
        gb::set_error("gust: check_sequencing_options: null argument");
        return GB_BAD_ARG;
    }
    // check_sequencing_options (Sequencing.cpp:120-169); the keys given
    // without steady.sequencing = 1 are the caller's to report (it reads them)
    std::vector<std::string> err;
    if (o->enabled) {
        if (!std::isfinite(o->drop_orders) || !(o->drop_orders > 0)
            || !(std::isfinite(strict->residual_drop_orders) && o->drop_orders <= strict->residual_drop_orders)) {
            err.emplace_back("steady.sequencing_drop_orders = " + fmte(o->drop_orders)
                             + ": must be > 0 and <= steady.residual_drop_orders = " + fmte(strict->residual_drop_orders)
                             + " (the loose stop of the coarse levels is not stricter than the strict one)");
        }
        if (!std::isfinite(o->monitor_tol) || !(o->monitor_tol >= 0) || !(o->monitor_tol < 1)) {
            err.emplace_back("steady.sequencing_monitor_tol = " + fmte(o->monitor_tol) + ": must be 0 (off) or > 0 and < 1");
        }
        if (o->hold != 0 && o->hold != 1) {
            err.emplace_back("steady.sequencing_hold = " + std::to_string(o->hold) + ": must be 0 or 1");
        }
        if (hierarchy_levels < 2) {
            err.emplace_back("steady.sequencing = 1 needs mesh.hierarchy_levels >= 2 (it is " + std::to_string(hierarchy_levels)
                             + ")");
        } else if (hierarchy_levels <= 10) {
            const int r = 1 << (hierarchy_levels - 1);
            const int cx = nx / r, cy = ny / r;
            if (cx < 2 || cy < 2) {
                err.emplace_back("steady.sequencing = 1 needs at least 2 cells in x and in y on the coarsest level: "
                                 "mesh.n_cell x and y / 2^(mesh.hierarchy_levels - 1) = " + std::to_string(cx) + " "
                                 + std::to_string(cy) + "; use fewer levels");
            }
        }
        if (o->cfl_previous && o->hold == 1) {
            err.emplace_back("steady.sequencing_cfl_start = previous needs steady.sequencing_hold = 0 "
                             "(the hold runs the first steady.residual_ref_iterations iterations at steady.cfl0)");
        }
    }
    if (!err.empty()) {
        gb::set_error("%s", joined("gust: invalid inputs:", err).c_str());
        return GB_BAD_ARG;
    }
    return GB_OK;
}

gb_status gb_loose_stop(const gb_criterion* c, const gb_sequencing_opts* o, int32_t hold_iterations, int32_t* branch,
                        char* reason, int32_t reason_cap)
{
    gb::clear_error();
    if (c == nullptr || o == nullptr || branch == nullptr) {
        gb::set_error("gust: loose_stop: null argument");
        return GB_BAD_ARG;
    }
    *branch = gb::loose_stop(c, *o, hold_iterations);
    copy_text({gb::loose_reason(*branch, c, *o)}, reason, reason_cap);
    return GB_OK;
}

}  // extern "C"
