// The k-L closure (Axell and Liungman 2001; Source/Closure_K.H,
// Source/Closure.cpp:270-460) and the surface layer's wall model
// (Source/SurfaceLayer.cpp, Source/StabilityFunctions.H,
// Source/BoundaryConditions.cpp:549-648) as CUDA kernels, one thread per
// cell or per ground column, in the reference's operation order.
#include "gb_turbulence.cuh"

#include <cfloat>

namespace gb {

using namespace st;

namespace {

// ---------------------------------------------------------- the closure ---

struct ClosureConst {
    double kappa, Cmu0, Cmu0_pow3, inv_Cb_sq, Rt_crit, Rt_min, l_g_max, tke_floor, n2_eps;
};

//! closure_constants (Closure.cpp:258-272).
ClosureConst closure_constants(const gb_physics& ph)
{
    ClosureConst c;
    c.kappa = ph.turb_kappa;
    c.Cmu0 = ph.turb_Cmu0;
    c.Cmu0_pow3 = ph.turb_Cmu0 * ph.turb_Cmu0 * ph.turb_Cmu0;
    c.inv_Cb_sq = 1.0 / (ph.turb_Cb * ph.turb_Cb);
    c.Rt_crit = ph.turb_Rt_crit;
    c.Rt_min = ph.turb_Rt_min;
    c.l_g_max = ph.turb_max_geom_lscale;
    c.tke_floor = std::max(ph.turb_tke_floor, DBL_EPSILON);
    c.n2_eps = DBL_EPSILON;
    return c;
}

struct Switches {
    int branch;
    bool smooth_Rt_g, smooth_Rt, floored;
};

struct Point {
    double k, L, Rt, cmu, cmu_prime, nut, eps;
};

struct Ptrs4 {
    double* p[4];
};
struct ClosureOut {
    double* p[kClosureFields];
};

__device__ __forceinline__ double pos_part(double x) { return 0.5 * (x + fabs(x)); }
__device__ __forceinline__ double neg_part(double x) { return 0.5 * (x - fabs(x)); }

__device__ __forceinline__ double smooth_Rt(double Rt, bool smooth, double Rt_crit, double Rt_min)
{
    const double x = neg_part(Rt - Rt_crit);
    const double a = Rt_min - Rt_crit;
    const double smoothed = Rt_crit + a * x / (x + a);
    return smooth ? smoothed : Rt;
}

//! switches_for (Closure_K.H:96-114): the branch decisions of the primal values.
__device__ __forceinline__ Switches switches_for(double k, double N2, double l_g, const ClosureConst& c)
{
    Switches s;
    s.floored = !(k > c.tke_floor);
    const double kf = s.floored ? c.tke_floor : k;
    s.branch = (fabs(N2) <= c.n2_eps) ? 0 : (N2 > c.n2_eps) ? 1 : 2;
    const double c6 = c.Cmu0_pow3 * c.Cmu0_pow3;
    const double N2s = pos_part(N2), N2u = neg_part(N2);
    const double Rt_g = l_g * l_g * N2u / (kf * c.Cmu0_pow3 * c.Cmu0_pow3);
    s.smooth_Rt_g = (s.branch == 2) && (Rt_g < c.Rt_crit);
    const double L_unstable = l_g * sqrt(1.0 - c6 * c.inv_Cb_sq * smooth_Rt(Rt_g, s.smooth_Rt_g, c.Rt_crit, c.Rt_min));
    const double L_stable = sqrt(1.0 / (1.0 / (l_g * l_g) + c.inv_Cb_sq * N2s / kf));
    const double L = (s.branch == 0) ? l_g : (s.branch == 1) ? L_stable : L_unstable;
    s.smooth_Rt = (L * L * N2 / (kf * c.Cmu0_pow3 * c.Cmu0_pow3) < c.Rt_crit);
    return s;
}

//! closure_point (Closure_K.H:134-165) in double.
__device__ __forceinline__ Point closure_point(double k, double N2, double l_g, const ClosureConst& c, const Switches& s)
{
    Point p;
    p.k = s.floored ? c.tke_floor : k;
    const double c6 = c.Cmu0_pow3 * c.Cmu0_pow3;
    const double N2s = pos_part(N2), N2u = neg_part(N2);
    const double L_stable = sqrt(1.0 / (1.0 / (l_g * l_g) + c.inv_Cb_sq * N2s / p.k));
    const double Rt_g = l_g * l_g * N2u / (p.k * c.Cmu0_pow3 * c.Cmu0_pow3);
    const double L_unstable = l_g * sqrt(1.0 - c6 * c.inv_Cb_sq * smooth_Rt(Rt_g, s.smooth_Rt_g, c.Rt_crit, c.Rt_min));
    p.L = (s.branch == 0) ? l_g : (s.branch == 1) ? L_stable : L_unstable;
    p.eps = c.Cmu0_pow3 * pow(p.k, 1.5) / p.L;
    p.Rt = smooth_Rt(p.L * p.L * N2 / (p.k * c.Cmu0_pow3 * c.Cmu0_pow3), s.smooth_Rt, c.Rt_crit, c.Rt_min);
    p.cmu = (c.Cmu0 + 0.108 * p.Rt) / (1.0 + 0.308 * p.Rt + 0.00837 * p.Rt * p.Rt);
    p.cmu_prime = c.Cmu0 / (1.0 + 0.277 * p.Rt);
    p.nut = p.cmu * sqrt(p.k) * p.L;
    return p;
}

//! The vertical ghost layers take the adjacent cell's values over the
//! columns -1..nx, -1..ny (copy_vertical_ghosts, Closure.cpp:130-146).
void copy_vertical_ghosts(gb_ctx* ctx, const gb_grid& g, double* const* a, int n)
{
    Ptrs4 P{};
    for (int m = 0; m < n; ++m) { P.p[m] = a[m]; }
    const gb_grid gg = g;
    for_box(ctx, Box{{-1, -1, 0}, {g.nx, g.ny, 0}}, [=] __device__(int i, int j, int) {
        for (int m = 0; m < n; ++m) {
            double* x = P.p[m];
            x[at(gg, i, j, -1)] = x[at(gg, i, j, 0)];
            x[at(gg, i, j, gg.nz)] = x[at(gg, i, j, gg.nz - 1)];
        }
    }, GB_KERNEL_RESIDUAL);
}

// ---------------------------------------------------- the surface layer ---

//! The vertical height of cell (i, j, k)'s centre above its column's ground.
__device__ __forceinline__ double column_height(const double* __restrict__ z, const gb_grid& g, int i, int j, int k)
{
    const double ground = 0.25 * ((z[at(g, i, j, 0)] + z[at(g, i + 1, j, 0)]) + (z[at(g, i, j + 1, 0)] + z[at(g, i + 1, j + 1, 0)]));
    return interp<NODE, CC>(z, g, i, j, k) - ground;
}

__device__ __forceinline__ void tangential_wind(const double* u, const double* v, const double* w, const gb_grid& g, int i,
                                                int j, int k, const double n[3], double ut[3])
{
    const double U[3] = {0.5 * (u[at(g, i, j, k)] + u[at(g, i + 1, j, k)]), 0.5 * (v[at(g, i, j, k)] + v[at(g, i, j + 1, k)]),
                         0.5 * (w[at(g, i, j, k)] + w[at(g, i, j, k + 1)])};
    const double un = U[0] * n[0] + U[1] * n[1] + U[2] * n[2];
    for (int d = 0; d < 3; ++d) { ut[d] = U[d] - un * n[d]; }
}

__device__ __forceinline__ void tangential_wind_ground(const double* u, const double* v, const gb_grid& g, int i, int j,
                                                       int k, double zx, double zy, const double n[3], double ut[3])
{
    const double uc = 0.5 * (u[at(g, i, j, k)] + u[at(g, i + 1, j, k)]);
    const double vc = 0.5 * (v[at(g, i, j, k)] + v[at(g, i, j + 1, k)]);
    const double U[3] = {uc, vc, zx * uc + zy * vc};
    const double un = U[0] * n[0] + U[1] * n[1] + U[2] * n[2];
    for (int d = 0; d < 3; ++d) { ut[d] = U[d] - un * n[d]; }
}

//! The stable side's coefficients (StabilityFunctions.H StableCoefficients):
//! Businger-Dyer (5, 0, 5, 0) or QNSE's from the options.
struct Stable {
    bool qnse;
    double am, bm, ah, bh;
};

__host__ Stable stable_of(const gb_bc& bc)
{
    if (bc.surface_qnse) { return {true, bc.surface_qnse_am, bc.surface_qnse_bm, bc.surface_qnse_ah, bc.surface_qnse_bh}; }
    return {false, 5.0, 0.0, 5.0, 0.0};
}

//! psi_m (StabilityFunctions.H most_psi_m): the Businger-Dyer unstable side
//! (ERF's calc_psi_m), the stable side -5 zeta or QNSE's -((a - b)/b) ln(1 + b zeta).
__device__ __forceinline__ double psi_m(double zeta, const Stable& sc)
{
    const double az = fabs(zeta);
    const double zs = 0.5 * (az + zeta), zu = 0.5 * (zeta - az);
    if (zeta > 0) { return sc.qnse ? -((sc.am - sc.bm) / sc.bm) * log(1.0 + sc.bm * zs) : -5.0 * zs; }
    const double x = sqrt(sqrt(1.0 - 16.0 * zu));
    const double pi = 3.14159265358979323846264338327950288;
    return 2.0 * log(0.5 * (1.0 + x)) + log(0.5 * (1.0 + x * x)) - 2.0 * atan(x) + pi / 2.0;
}

//! most_phi (StabilityFunctions.H) with the stable side's coefficients.
__device__ __forceinline__ void most_phi(double zeta, const Stable& sc, double& phi_m, double& phi_h)
{
    const double one = 1, gamma = 16, am = sc.am, bm = sc.bm, ah = sc.ah, bh = sc.bh;
    const double az = fabs(zeta);
    const double zs = 0.5 * (az + zeta);
    const double zu = 0.5 * (zeta - az);
    const double r = sqrt(one - gamma * zu);
    phi_m = (one + am * zs) / (one + bm * zs) + (one / sqrt(r) - one);
    phi_h = (one + ah * zs) / (one + bh * zs) + (one / r - one);
}

//! u - kappa U / max(ln((d + z0)/z0) - psi_m(d/L(u)), m) (MostRelation, SurfaceLayer.cpp:78-95).
struct MostRelation {
    double kappa, U, d, lz, den_min, gq, ustar_min;
    Stable sc;
    __device__ double inv_L(double u) const
    {
        const double uf = fmax(u, ustar_min);
        return -kappa * gq / (uf * uf * uf);
    }
    __device__ double operator()(double u) const
    {
        const double zeta = fmax(fmin(d * inv_L(u), 100.0), -100.0);
        return u - kappa * U / fmax(lz - psi_m(zeta, sc), den_min);
    }
};

__device__ __forceinline__ int reference_interval(const double* z, const gb_grid& g, int i, int j, int n, double zr)
{
    if (zr < column_height(z, g, i, j, 0)) { return -1; }
    if (zr > column_height(z, g, i, j, n - 1)) { return n - 1; }
    int k = 0;
    while (k < n - 2 && !(zr < column_height(z, g, i, j, k + 1))) { ++k; }
    return k;
}

struct Planes11 {
    double* p[kSsPlanes];
};
struct CPlanes11 {
    const double* p[kSsPlanes];
};
struct Planes3 {
    double* p[3];
};

CPlanes11 cplanes(const double* const* ss)
{
    CPlanes11 P{};
    for (int n = 0; n < kSsPlanes; ++n) { P.p[n] = ss[n]; }
    return P;
}

}  // namespace

void turb_height_above_ground(gb_ctx* ctx, const gb_grid& g, const double* z, double* dist)
{
    const gb_grid gg = g;
    for_box(ctx, Box{{-1, -1, 0}, {g.nx, g.ny, g.nz - 1}}, [=] __device__(int i, int j, int k) {
        double zc = 0, zg = 0;
        for (int a = 0; a < 2; ++a) {
            for (int b = 0; b < 2; ++b) {
                zg += z[at(gg, i + a, j + b, 0)];
                zc += z[at(gg, i + a, j + b, k)] + z[at(gg, i + a, j + b, k + 1)];
            }
        }
        dist[at(gg, i, j, k)] = 0.125 * zc - 0.25 * zg;
    }, GB_KERNEL_RESIDUAL);
    double* one[1] = {dist};
    copy_vertical_ghosts(ctx, g, one, 1);
}

void turb_closure(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const gb_physics& ph, const gb_state& q,
                  const double* z, const double* dist, const double* z0map, double* const* cf, const double* nut_prev)
{
    const gb_grid gg = g;
    const ClosureConst c = closure_constants(ph);
    const double g_over_theta0 = ph.gravity / ph.theta0;
    const double nu_mol = ph.turb_nu_molecular, alpha_mol = ph.turb_alpha_molecular;
    const double inv_sigma = 1 / ph.turb_sigma_k;
    // turb.ri_gate (gate_stratification, Closure.cpp:337-354) and
    // turb.realizability (nut_cap_field, ClosureWake.cpp:8-29)
    const double ri0 = ph.turb_ri_gate, r2 = ri0 * ri0, cr = ph.turb_realizability;
    const bool gate = ri0 > 0, capped = cr > 0;
    // the nu_t relaxation (Closure.cpp:407-411): the history when there is
    // one, else k with the weight 1 - w = 0
    const double wgt = nut_prev ? ph.turb_nut_relax : 1.0;
    // the ground's roughness in kappa (d + z0): a map, the uniform value, or 0
    // without a surface layer (ground_roughness, SurfaceLayer.H:176-181)
    const bool wall = bc.face[2] == GB_FACE_SURFACE_LAYER;
    const double z0u = wall ? bc.surface_z0 : 0.0;
    const double* zmap = wall ? z0map : nullptr;
    const double* u = q.u;
    const double* v = q.v;
    const double* w = q.w;
    const double* th = q.theta;
    const double* tk = q.tke;
    const double* prev = nut_prev ? nut_prev : q.tke;
    ClosureOut O{};
    for (int n = 0; n < kClosureFields; ++n) { O.p[n] = cf[n]; }
    for_box(ctx, Box{{-1, -1, 0}, {g.nx, g.ny, g.nz - 1}}, [=] __device__(int i, int j, int k) {
        const int64_t o = at(gg, i, j, k);
        // N^2 and S^2 (stratification_and_strain, Closure.cpp:302-345)
        const Metric<double> m = metric_at<CC>(z, gg, i, j, k);
        double gt[3], gu[3], gv[3], gw[3];
        grad_at<CC, CC>(th, gg, i, j, k, m, gt);
        const double N2 = g_over_theta0 * gt[2];
        grad_at<XF, CC>(u, gg, i, j, k, m, gu);
        grad_at<YF, CC>(v, gg, i, j, k, m, gv);
        grad_at<ZF, CC>(w, gg, i, j, k, m, gw);
        const double G[3][3] = {{gu[0], gu[1], gu[2]}, {gv[0], gv[1], gv[2]}, {gw[0], gw[1], gw[2]}};
        double s = 0;
        for (int a = 0; a < 3; ++a) {
            for (int b = 0; b < 3; ++b) {
                const double e = G[a][b] + G[b][a];
                s += e * e;
            }
        }
        const double S2 = 0.5 * s;
        const double z0 = zmap ? zmap[plane_at(gg, i, j)] : z0u;
        const double lraw = c.kappa * (dist[o] + z0);
        const double l_g = c.l_g_max * lraw / (c.l_g_max + lraw);
        // the length and Rt see the gated N^2; P_b keeps N^2
        double N2c = N2;
        if (gate) {
            const double a = N2 * N2, b = S2 * S2;
            N2c *= a / (a + r2 * b + DBL_MIN);
        }
        const Switches sw = switches_for(tk[o], N2c, l_g, c);
        const Point p = closure_point(tk[o], N2c, l_g, c, sw);
        const double ratio = p.cmu_prime / p.cmu;
        double cap = DBL_MAX;
        if (capped) {
            const double sr = sqrt(S2);
            cap = (sr > DBL_MIN) ? cr * fmax(tk[o], c.tke_floor) / sr : DBL_MAX;
        }
        const double nt = wgt * fmin(p.nut, cap) + (1 - wgt) * prev[o];
        O.p[kClosureNut][o] = nt;
        O.p[kClosureNu][o] = nu_mol + nt;
        O.p[kClosureGammaTheta][o] = alpha_mol + ratio * nt;
        O.p[kClosureGammaTke][o] = nu_mol + nt * inv_sigma;
        if (i >= 0 && i < gg.nx && j >= 0 && j < gg.ny) {
            const double Ps = nt * S2, Pb = -ratio * nt * N2;
            O.p[kClosureLength][o] = p.L;
            O.p[kClosureRt][o] = p.Rt;
            O.p[kClosurePs][o] = Ps;
            O.p[kClosurePb][o] = Pb;
            O.p[kClosureEps][o] = p.eps;
            O.p[kClosureDSdk][o] = (p.eps + pos_part(-Pb)) / p.k;
        }
    }, GB_KERNEL_RESIDUAL);
    copy_vertical_ghosts(ctx, g, cf, 4);
}

void turb_surface_state(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const gb_physics& ph, const gb_state& q,
                        const double* z, const double* z0map, double* const* ss, unsigned long long* bad)
{
    const gb_grid gg = g;
    const int nz = g.nz;
    const double kappa = bc.kappa;
    const bool heat = bc.surface_stability == GB_SURFACE_HEAT_FLUX;
    const bool first = !(bc.surface_zref > 0);
    const double zref_in = bc.surface_zref;
    const bool floor_one = bc.surface_denominator_floor == GB_DENOMINATOR_ONE;
    const double gq = (ph.gravity / ph.theta0) * bc.surface_heat_flux;
    const double inv_cmu2 = 1.0 / (bc.Cmu0 * bc.Cmu0);
    const double eps = DBL_EPSILON, tol = 64 * eps, hrel = std::sqrt(eps);
    const double z0u = bc.surface_z0;
    const double dxinv = 1.0 / g.dx, dyinv = 1.0 / g.dy;
    const Stable sc = stable_of(bc);
    const double* u = q.u;
    const double* v = q.v;
    const double* w = q.w;
    Planes11 P{};
    for (int n = 0; n < kSsPlanes; ++n) { P.p[n] = ss[n]; }
    for_box(ctx, Box{{-1, -1, 0}, {g.nx, g.ny, 0}}, [=] __device__(int i, int j, int) {
        const double z0 = z0map ? z0map[plane_at(gg, i, j)] : z0u;
        const double zx = deriv<NODE, ZF, 0>(z, gg, i, j, 0) * dxinv;
        const double zy = deriv<NODE, ZF, 1>(z, gg, i, j, 0) * dyinv;
        const double area = sqrt(1 + zx * zx + zy * zy);
        const double n[3] = {-zx / area, -zy / area, 1 / area};
        const double h0 = column_height(z, gg, i, j, 0);
        const double zr = first ? h0 : zref_in;
        int k = reference_interval(z, gg, i, j, nz, zr);
        k = max(0, min(nz - 2, k));
        double ua[3], ub[3];
        if (k == 0) {
            tangential_wind_ground(u, v, gg, i, j, 0, zx, zy, n, ua);
        } else {
            tangential_wind(u, v, w, gg, i, j, k, n, ua);
        }
        tangential_wind(u, v, w, gg, i, j, k + 1, n, ub);
        const double ia = 1.0 / area;
        const double la = log(column_height(z, gg, i, j, k) * ia + z0);
        const double f = (log(zr * ia + z0) - la) / (log(column_height(z, gg, i, j, k + 1) * ia + z0) - la);
        double ut[3];
        for (int cc = 0; cc < 3; ++cc) { ut[cc] = ua[cc] + f * (ub[cc] - ua[cc]); }
        const double mag = sqrt(ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2]);
        const double U = fmax(mag, 0.1);
        const double d = zr * ia;
        const double lz = log((d + z0) / z0);
        double den_min = fmin(lz, 1.0);
        if (floor_one) { den_min = 1.0; }
        double ustar = kappa * U / fmax(lz, den_min);
        double invL = 0;
        if (heat) {
            const MostRelation F{kappa, U, d, lz, den_min, gq, 0.001, sc};
            bool converged = false;
            for (int it = 0; it < 50 && !converged; ++it) {
                const double fu = F(ustar);
                const double du = hrel * ustar;
                const double fp = (F(ustar + du) - fu) / du;
                double next = (fp > 0) ? ustar - fu / fp : ustar - 0.5 * fu;
                next = fmax(0.5 * ustar, fmin(2.0 * ustar, next));
                converged = fabs(next - ustar) <= tol * next;
                ustar = next;
            }
            if (!converged) { ustar = __longlong_as_double(0x7ff8000000000000LL); }
            invL = F.inv_L(ustar);
        }
        const double d0 = h0 * ia;
        const int64_t p = plane_at(gg, i, j);
        P.p[kSsUstar][p] = ustar;
        P.p[kSsSpeed][p] = U;
        P.p[kSsZref][p] = zr;
        P.p[kSsD0][p] = d0;
        P.p[kSsInvL][p] = invL;
        P.p[kSsArea][p] = area;
        const double cdrag = ustar * ustar / U * area;
        P.p[kSsDrag][p] = cdrag;
        P.p[kSsTauX][p] = cdrag * ut[0];
        P.p[kSsTauY][p] = cdrag * ut[1];
        P.p[kSsTauZ][p] = cdrag * ut[2];
        double kwall = ustar * ustar * inv_cmu2;
        if (heat) { kwall = inv_cmu2 * pow(ustar * ustar * ustar + kappa * fmax(gq, 0.0) * d0, 2.0 / 3.0); }
        P.p[kSsKwall][p] = kwall;
        if (bad && (!(ustar == ustar) || !(kwall == kwall) || !(ustar > 0 && ustar < DBL_MAX))) { atomicAdd(bad, 1ULL); }
    }, GB_KERNEL_BC);
}

void turb_ground_gradients(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const double* const* ss,
                           const double* z0map, double* const* gg_out)
{
    const gb_grid gg = g;
    const double unset = DBL_MAX;
    const Stable sc = stable_of(bc);
    const double kappa = bc.kappa;
    const double qs = (bc.surface_stability == GB_SURFACE_HEAT_FLUX) ? bc.surface_heat_flux : 0.0;
    const double z0u = bc.surface_z0;
    const CPlanes11 S = cplanes(ss);
    Planes3 O{};
    for (int n = 0; n < 3; ++n) { O.p[n] = gg_out[n]; }
    // the surface state's columns -1..nx, -1..ny; every other column unset
    for_box(ctx, Box{{-2, -2, 0}, {g.nx + 1, g.ny + 1, 0}}, [=] __device__(int i, int j, int) {
        const int64_t p = plane_at(gg, i, j);
        if (i < -1 || i > gg.nx || j < -1 || j > gg.ny) {
            for (int n = 0; n < 3; ++n) { O.p[n][p] = unset; }
            return;
        }
        const double zeta = fmax(fmin(S.p[kSsD0][p] * S.p[kSsInvL][p], 100.0), -100.0);
        double phi_m, phi_h;
        most_phi(zeta, sc, phi_m, phi_h);
        const double z0 = z0map ? z0map[p] : z0u;
        const double s = kappa * (S.p[kSsD0][p] + z0);
        const double tx = S.p[kSsTauX][p], ty = S.p[kSsTauY][p], tz = S.p[kSsTauZ][p];
        const double tmag = sqrt(tx * tx + ty * ty + tz * tz);
        const double tsafe = tmag + DBL_MIN;
        const double dir_x = tx / tsafe, dir_y = ty / tsafe;
        const double us = S.p[kSsUstar][p];
        O.p[0][p] = us / s * dir_x * phi_m;
        O.p[1][p] = us / s * dir_y * phi_m;
        O.p[2][p] = -qs / (us * s) * phi_h;
    }, GB_KERNEL_BC);
    // FillBoundary: a column outside the domain that images a domain column
    // across the periodic directions takes its value
    for_box(ctx, Box{{-2, -2, 0}, {g.nx + 1, g.ny + 1, 0}}, [=] __device__(int i, int j, int) {
        if (i >= 0 && i < gg.nx && j >= 0 && j < gg.ny) { return; }
        int si = i, sj = j;
        if (gg.periodic_x) { si = ((i % gg.nx) + gg.nx) % gg.nx; }
        if (gg.periodic_y) { sj = ((j % gg.ny) + gg.ny) % gg.ny; }
        if (si >= 0 && si < gg.nx && sj >= 0 && sj < gg.ny) {
            for (int n = 0; n < 3; ++n) { O.p[n][plane_at(gg, i, j)] = O.p[n][plane_at(gg, si, sj)]; }
        }
    }, GB_KERNEL_BC);
    // what is left takes the nearest domain column along the non-periodic
    // directions (the columns read are never unset themselves)
    for_box(ctx, Box{{-2, -2, 0}, {g.nx + 1, g.ny + 1, 0}}, [=] __device__(int i, int j, int) {
        const int64_t p = plane_at(gg, i, j);
        if (O.p[0][p] != unset) { return; }
        const int ic = gg.periodic_x ? i : min(max(i, 0), gg.nx - 1);
        const int jc = gg.periodic_y ? j : min(max(j, 0), gg.ny - 1);
        for (int n = 0; n < 3; ++n) { O.p[n][p] = O.p[n][plane_at(gg, ic, jc)]; }
    }, GB_KERNEL_BC);
}

void turb_ground_flux(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const double* const* ss, int field, double* Gz)
{
    const gb_grid gg = g;
    const double qs = (bc.surface_stability == GB_SURFACE_HEAT_FLUX) ? bc.surface_heat_flux : 0.0;
    const CPlanes11 S = cplanes(ss);
    Box b{{0, 0, 0}, {g.nx - 1 + (field == 0 ? 1 : 0), g.ny - 1 + (field == 1 ? 1 : 0), 0}};
    for_box(ctx, b, [=] __device__(int i, int j, int) {
        const int64_t o = at(gg, i, j, 0);
        if (field == 0) {
            Gz[o] = 0.5 * (S.p[kSsTauX][plane_at(gg, i - 1, j)] + S.p[kSsTauX][plane_at(gg, i, j)]);
        } else if (field == 1) {
            Gz[o] = 0.5 * (S.p[kSsTauY][plane_at(gg, i, j - 1)] + S.p[kSsTauY][plane_at(gg, i, j)]);
        } else if (field == 2) {
            Gz[o] = -qs * S.p[kSsArea][plane_at(gg, i, j)];
        } else {
            Gz[o] = 0;
        }
    }, GB_KERNEL_RESIDUAL);
}

void turb_k_sources(gb_ctx* ctx, const gb_grid& g, const double* const* cf, double* Rk)
{
    const gb_grid gg = g;
    const double* Ps = cf[kClosurePs];
    const double* Pb = cf[kClosurePb];
    const double* ep = cf[kClosureEps];
    for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
        const int64_t o = at(gg, i, j, k);
        Rk[o] = ((Rk[o] - Ps[o]) - Pb[o]) + ep[o];
    }, GB_KERNEL_RESIDUAL);
}

void turb_apply_wall_k(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const double* const* ss, const double* tke,
                       double* Rk)
{
    const gb_grid gg = g;
    const bool dirichlet = bc.surface_wall_k == GB_WALL_K_DIRICHLET;
    const CPlanes11 S = cplanes(ss);
    for_box(ctx, Box{{0, 0, 0}, {g.nx - 1, g.ny - 1, 0}}, [=] __device__(int i, int j, int) {
        const int64_t p = plane_at(gg, i, j), o = at(gg, i, j, 0);
        const double r = fmax(S.p[kSsUstar][p], 0.01) / S.p[kSsD0][p] * (tke[o] - S.p[kSsKwall][p]);
        Rk[o] = dirichlet ? r : Rk[o] + r;
    }, GB_KERNEL_RESIDUAL);
}

void turb_patankar(gb_ctx* ctx, const gb_grid& g, const double* dSdk, double* A)
{
    const gb_grid gg = g;
    const int64_t cs = volume(g);
    for_box(ctx, valid_box(g, CC), [=] __device__(int i, int j, int k) {
        const int64_t o = at(gg, i, j, k);
        A[GB_COEF_P * cs + o] += dSdk[o];
    }, GB_KERNEL_COEFS);
}

void turb_wall_rows(gb_ctx* ctx, const gb_grid& g, const double* const* ss, int loc, const double* J, double* A)
{
    const gb_grid gg = g;
    const int64_t cs = volume(g);
    const double dzinv = 1.0 / g.dzeta;
    const CPlanes11 S = cplanes(ss);
    Box b = valid_box(g, loc);
    b.hi[2] = 0;
    for_box(ctx, b, [=] __device__(int i, int j, int) {
        const int64_t o = at(gg, i, j, 0);
        A[GB_COEF_P * cs + o] -= A[GB_COEF_ZM * cs + o];
        A[GB_COEF_ZM * cs + o] = 0;
        if (loc == XF) {
            A[GB_COEF_P * cs + o] += 0.5 * (S.p[kSsDrag][plane_at(gg, i - 1, j)] + S.p[kSsDrag][plane_at(gg, i, j)]) * dzinv
                                     / interp<CC, XF>(J, gg, i, j, 0);
        } else if (loc == YF) {
            A[GB_COEF_P * cs + o] += 0.5 * (S.p[kSsDrag][plane_at(gg, i, j - 1)] + S.p[kSsDrag][plane_at(gg, i, j)]) * dzinv
                                     / interp<CC, YF>(J, gg, i, j, 0);
        }
    }, GB_KERNEL_COEFS);
}

void turb_wall_k_rows(gb_ctx* ctx, const gb_grid& g, const gb_bc& bc, const double* const* ss, double* A)
{
    const gb_grid gg = g;
    const int64_t cs = volume(g);
    const bool dirichlet = bc.surface_wall_k == GB_WALL_K_DIRICHLET;
    const CPlanes11 S = cplanes(ss);
    for_box(ctx, Box{{0, 0, 0}, {g.nx - 1, g.ny - 1, 0}}, [=] __device__(int i, int j, int) {
        const int64_t p = plane_at(gg, i, j), o = at(gg, i, j, 0);
        const double a = fmax(S.p[kSsUstar][p], 0.01) / S.p[kSsD0][p];
        if (dirichlet) {
            for (int n = 0; n < GB_N_COEFS; ++n) { A[n * cs + o] = 0; }
            A[GB_COEF_P * cs + o] = a;
        } else {
            A[GB_COEF_P * cs + o] += a;
        }
    }, GB_KERNEL_COEFS);
}

}  // namespace gb
