// The GUST-side adaptor over libgustb200.so's C ABI (include/gust_b200.h):
// the gust:: signatures of the hot path's free functions, and a stage object
// whose methods are the SIMPLEC iteration's steps, so that GUST's call sites
// (SimplecStage::iterate, NewtonPreconditioner, Transfer's prolong_state)
// keep their shape. A GUST build compiles this file with its own AMReX and
// GUST headers and links -lgustb200 -lcudart.
//
// Layout: one box per level spanning the domain with two ghost layers, i
// fastest (AMReX's Array4 order), so a MultiFab's fab data is passed as is.
// A build with several boxes per level packs each MultiFab into that layout
// first (a device copy per stage) and unpacks the results.
//
// Errors: every call returns a gb_status; a status other than GB_OK becomes
// amrex::Abort with the library's message (which names the input key), the
// reference's convention.
#include "gust_b200.h"

#include "ImplicitOperator.H"
#include "Predictor.H"
#include "Residual.H"
#include "Simplec.H"

namespace gust {
namespace b200 {

//! One context per host thread, on the stream AMReX launches on.
gb_ctx* context()
{
    thread_local gb_ctx* ctx = nullptr;
    if (ctx == nullptr && gb_ctx_create(amrex::Gpu::gpuStream(), &ctx) != GB_OK) { amrex::Abort(gb_last_error()); }
    return ctx;
}

void check(gb_status st)
{
    if (st != GB_OK) { amrex::Abort(gb_last_error()); }
}

gb_grid grid_of(const amrex::Geometry& geom, const Mesh& mesh)
{
    const amrex::Box& dom = geom.Domain();
    gb_grid g;
    check(gb_grid_init(&g, dom.length(0), dom.length(1), dom.length(2), 2, geom.CellSize(0), geom.CellSize(1),
                       mesh.dzeta(), geom.isPeriodic(0) ? 1 : 0, geom.isPeriodic(1) ? 1 : 0));
    return g;
}

double* data(amrex::MultiFab& mf) { return mf[0].dataPtr(); }
const double* data(const amrex::MultiFab& mf) { return mf[0].dataPtr(); }

gb_state state_of(State& q, const double* z_nd)
{
    return gb_state{data(q.u), data(q.v), data(q.w), data(q.p), data(q.theta), data(q.tke), z_nd};
}

//! gust::Equation (u, v, w, theta, tke) to the ABI's equation index (p is 3).
int32_t equation_index(Equation eq)
{
    switch (eq) {
    case Equation::u: return 0;
    case Equation::v: return 1;
    case Equation::w: return 2;
    case Equation::theta: return 4;
    default: return 5;
    }
}

}  // namespace b200

//! gust::zline_jacobi (Source/Predictor.H:267-268).
amrex::Real zline_jacobi(Loc loc, const amrex::MultiFab& A, const amrex::MultiFab& ap, const amrex::MultiFab& rhs,
                         int sweeps, const Mesh& mesh, const amrex::Geometry& geom, amrex::MultiFab& delta)
{
    const gb_grid g = b200::grid_of(geom, mesh);
    double change = 0;
    b200::check(gb_zline_jacobi(b200::context(), &g, static_cast<int32_t>(loc), b200::data(A), b200::data(ap),
                                b200::data(rhs), sweeps, b200::data(delta), &change));
    return change;
}

//! gust::implicit_coefficients (Source/ImplicitOperator.H:65-67).
void implicit_coefficients(Loc loc, const amrex::Array<const amrex::MultiFab*, 3>& F, const amrex::MultiFab& gamma,
                           const amrex::MultiFab& z_nd, const Mesh& mesh, const amrex::Geometry& geom,
                           amrex::MultiFab& A, FaceMean mean)
{
    const gb_grid g = b200::grid_of(geom, mesh);
    b200::check(gb_implicit_coefficients(b200::context(), &g, static_cast<int32_t>(loc), b200::data(*F[0]),
                                         b200::data(*F[1]), b200::data(*F[2]), b200::data(gamma), b200::data(z_nd),
                                         b200::data(mesh.detJ), mean == FaceMean::logarithmic ? 1 : 0,
                                         b200::data(A)));
}

//! The SIMPLEC stage on the B200 (SimplecStage, Source/Simplec.H:185-263):
//! the stage's options and inputs go to gb_simplec_create once; each method
//! is one of the iteration's steps on the caller's state, in the order
//! SimplecStage::iterate takes them.
class B200SimplecStage
{
public:
    B200SimplecStage(const gb_grid& g, const gb_bc& bc, const gb_physics& ph, const gb_simplec_opts& opt,
                     const amrex::MultiFab& z_nd, const gb_mesh_fields& mesh, const gb_diffusivities& df)
        : m_z(b200::data(z_nd))
    {
        b200::check(gb_simplec_create(b200::context(), &g, &bc, &ph, &opt, m_z, &mesh, &df, &m_s));
    }
    ~B200SimplecStage() { gb_simplec_destroy(m_s); }
    B200SimplecStage(const B200SimplecStage&) = delete;
    B200SimplecStage& operator=(const B200SimplecStage&) = delete;

    //! BoundaryConditions::fill_ghosts (Source/BoundaryConditions.H:174-175) with the wall state.
    void fill_ghosts(State& q)
    {
        gb_state s = b200::state_of(q, m_z);
        b200::check(gb_simplec_fill_ghosts(m_s, &s));
    }

    //! gust::residual (Source/Residual.H:133-134), the closure's fields kept by the stage.
    void residual(State& q, ResidualFields& R)
    {
        gb_state s = b200::state_of(q, m_z);
        double* r[6] = {b200::data(R.u), b200::data(R.v), b200::data(R.w), b200::data(R.p), b200::data(R.theta),
                        b200::data(R.tke)};
        b200::check(gb_simplec_residual(m_s, &s, r));
    }

    //! gust::momentum_predictor (Source/Predictor.H:242-252) from the cell dtau.
    MomentumPredictorResult momentum_predictor(State& q, ResidualFields& R, const amrex::MultiFab& dtau,
                                               PredictorFields& pf)
    {
        gb_state s = b200::state_of(q, m_z);
        double* r[6] = {b200::data(R.u), b200::data(R.v), b200::data(R.w), b200::data(R.p), b200::data(R.theta),
                        b200::data(R.tke)};
        double* ap[3] = {b200::data(pf.ap_u), b200::data(pf.ap_v), b200::data(pf.ap_w)};
        double* d[3] = {b200::data(pf.d_u), b200::data(pf.d_v), b200::data(pf.d_w)};
        gb_predictor_result res{};
        b200::check(gb_momentum_predictor(m_s, &s, r, b200::data(dtau), ap, d, &res));
        MomentumPredictorResult out;
        out.max_du = res.max_du;
        out.max_dv = res.max_dv;
        out.max_dw = res.max_dw;
        out.last_sweep_du = res.last_sweep_du;
        out.last_sweep_dv = res.last_sweep_dv;
        out.last_sweep_dw = res.last_sweep_dw;
        return out;
    }

    //! gust::pressure_correction (Source/Simplec.H:139-141) with pf's denominators.
    PressureCorrectionResult pressure_correction(State& q, const PredictorFields& pf)
    {
        gb_state s = b200::state_of(q, m_z);
        const double* d[3] = {b200::data(pf.d_u), b200::data(pf.d_v), b200::data(pf.d_w)};
        gb_pressure_result res{};
        b200::check(gb_pressure_correction(m_s, &s, d, &res));
        PressureCorrectionResult out;
        out.poisson.iterations = res.poisson_iterations;
        out.poisson.removed_mean = res.poisson_removed_mean;
        out.divergence_before = res.divergence_before;
        out.divergence_after = res.divergence_after;
        out.max_dp = res.max_dp;
        out.max_du = res.max_du;
        out.max_dv = res.max_dv;
        out.max_dw = res.max_dw;
        return out;
    }

    //! gust::scalar_sweep (Source/Simplec.H:156-163) of theta or tke.
    ScalarSweepResult scalar_sweep(Equation eq, State& q, const amrex::MultiFab& R_eq, const amrex::MultiFab& dtau,
                                   bool clip = true)
    {
        if (eq != Equation::theta && eq != Equation::tke) { amrex::Abort("gust: scalar_sweep: eq must be theta or tke"); }
        gb_state s = b200::state_of(q, m_z);
        gb_scalar_result res{};
        b200::check(gb_scalar_sweep(m_s, &s, b200::equation_index(eq), b200::data(R_eq), b200::data(dtau),
                                    clip ? 1 : 0, &res));
        ScalarSweepResult out;
        out.max_dq = res.max_dq;
        out.last_sweep = res.last_sweep;
        out.clipped = res.clipped;
        return out;
    }

    //! SimplecStage::iterate (Source/Simplec.cpp:452-506): one outer iteration.
    gb_iter_info iterate(State& q, const amrex::MultiFab& dtau)
    {
        gb_state s = b200::state_of(q, m_z);
        gb_iter_info info{};
        b200::check(gb_simplec_iterate(m_s, &s, b200::data(dtau), &info));
        return info;
    }

    //! gust::local_dtau (Source/PseudoTime.H:32-33) at the stage's closure viscosity.
    void local_dtau(State& q, amrex::Real cfl, amrex::MultiFab& dtau)
    {
        gb_state s = b200::state_of(q, m_z);
        b200::check(gb_local_dtau(m_s, &s, cfl, b200::data(dtau)));
    }

private:
    gb_simplec* m_s{nullptr};
    const double* m_z{nullptr};
};

//! The stage's construction for the test of this file: one stage object, so
//! that every member function above is instantiated and checked.
void b200_stage_example(const gb_grid& g, const gb_bc& bc, const gb_physics& ph, const gb_simplec_opts& opt,
                        const amrex::MultiFab& z_nd, const gb_mesh_fields& mesh, const gb_diffusivities& df, State& q,
                        ResidualFields& R, PredictorFields& pf, amrex::MultiFab& dtau)
{
    B200SimplecStage st(g, bc, ph, opt, z_nd, mesh, df);
    st.fill_ghosts(q);
    st.local_dtau(q, 1.0, dtau);
    st.residual(q, R);
    st.momentum_predictor(q, R, dtau, pf);
    st.pressure_correction(q, pf);
    st.scalar_sweep(Equation::theta, q, R.theta, dtau, false);
    st.scalar_sweep(Equation::tke, q, R.tke, dtau);
    st.iterate(q, dtau);
}

}  // namespace gust
