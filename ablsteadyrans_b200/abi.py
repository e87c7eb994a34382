"""ctypes mirrors of the C ABI's plain structs (include/gust_b200.h) and
constructors with the reference's defaults. No library is needed to use them."""
import ctypes

import numpy as np

from .grid import GbGrid  # noqa: F401

FACE_PERIODIC, FACE_INFLOW, FACE_OUTFLOW, FACE_SLIP_WALL, FACE_NO_SLIP_WALL, FACE_SURFACE_LAYER = range(6)
SURFACE_NEUTRAL, SURFACE_HEAT_FLUX = range(2)
WALL_K_DIRICHLET, WALL_K_SOURCE = range(2)
DENOMINATOR_LOG_LAW, DENOMINATOR_ONE = range(2)
LIMITER_VAN_LEER, LIMITER_VAN_ALBADA, LIMITER_UPWIND = range(3)
MAX_PROFILE = 32


class LineSystem(ctypes.Structure):
    """gb_line_system / gb_line_system_f32 (the same layout: pointers by address)."""
    _fields_ = [("grid", GbGrid), ("loc", ctypes.c_int32), ("A", ctypes.c_void_p), ("ap", ctypes.c_void_p),
                ("rhs", ctypes.c_void_p), ("delta", ctypes.c_void_p)]


class PoissonOptions(ctypes.Structure):
    """gb_poisson_opts: the solver.poisson_* inputs plus the multigrid settings."""
    _fields_ = [("reltol", ctypes.c_double), ("abstol", ctypes.c_double), ("max_iter", ctypes.c_int32),
                ("restart", ctypes.c_int32), ("precision", ctypes.c_int32), ("nu1", ctypes.c_int32),
                ("nu2", ctypes.c_int32), ("nu_coarse", ctypes.c_int32), ("max_levels", ctypes.c_int32),
                ("min_coarse", ctypes.c_int32)]

    @classmethod
    def defaults(cls, **kw):
        """The reference's solver.poisson_* defaults (Source/Poisson.H:41-75) and
        this project's multigrid settings."""
        o = cls(reltol=1e-10, abstol=0.0, max_iter=200, restart=50, precision=0, nu1=1, nu2=1, nu_coarse=8,
                max_levels=12, min_coarse=2)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class BC(ctypes.Structure):
    """gb_bc: bc.* (Source/BoundaryConditions.H:99-143) with the log-law inflow."""
    _fields_ = [("face", ctypes.c_int32 * 6), ("wall_velocity", (ctypes.c_double * 3) * 6),
                ("zhi_theta_grad", ctypes.c_double), ("inflow_ustar", ctypes.c_double),
                ("inflow_z0", ctypes.c_double), ("inflow_direction", ctypes.c_double), ("kappa", ctypes.c_double),
                ("Cmu0", ctypes.c_double), ("inflow_inv_lmax", ctypes.c_double), ("theta_ref_n", ctypes.c_int32),
                ("theta_ref_z", ctypes.c_double * MAX_PROFILE), ("theta_ref_theta", ctypes.c_double * MAX_PROFILE),
                ("surface_z0", ctypes.c_double), ("surface_zref", ctypes.c_double),
                ("surface_stability", ctypes.c_int32), ("surface_heat_flux", ctypes.c_double),
                ("surface_wall_k", ctypes.c_int32), ("surface_denominator_floor", ctypes.c_int32),
                ("rayleigh_zdamp", ctypes.c_double), ("rayleigh_dampcoef", ctypes.c_double),
                ("rayleigh_fields", ctypes.c_int32), ("rayleigh_above_ground", ctypes.c_int32),
                ("sponge_width", ctypes.c_double), ("sponge_strength", ctypes.c_double),
                ("surface_qnse", ctypes.c_int32), ("surface_qnse_am", ctypes.c_double),
                ("surface_qnse_bm", ctypes.c_double), ("surface_qnse_ah", ctypes.c_double),
                ("surface_qnse_bh", ctypes.c_double)]

    @classmethod
    def make(cls, faces, theta_ref=((0.0,), (300.0,)), ustar=0.4, z0=0.1, direction=0.0, kappa=0.41, Cmu0=0.5562,
             l_max=30.0, zhi_theta_grad=0.0, wall_velocity=None, surface=None, damping=None):
        """surface: bc.surface_* of a surface_layer ground as a dict (z0, zref,
        stability, heat_flux, wall_k, denominator_floor); the reference's
        defaults (Source/SurfaceLayer.H: z0 0.1 m, first cell centre, neutral,
        Dirichlet wall k, log-law floor) otherwise. damping: bc.rayleigh_* and
        bc.sponge_* as a dict (zdamp, dampcoef, fields, above_ground, width,
        strength); off otherwise."""
        b = cls()
        b.rayleigh_fields = 31
        for k, v in (damping or {}).items():
            setattr(b, ("sponge_" if k in ("width", "strength") else "rayleigh_") + k, v)
        b.surface_z0, b.surface_zref, b.surface_stability = 0.1, 0.0, SURFACE_NEUTRAL
        b.surface_heat_flux, b.surface_wall_k, b.surface_denominator_floor = 0.0, WALL_K_DIRICHLET, DENOMINATOR_LOG_LAW
        b.surface_qnse, b.surface_qnse_am, b.surface_qnse_bm, b.surface_qnse_ah, b.surface_qnse_bh = 0, 2.5, 0.2, 2.5, 0.2
        for k, v in (surface or {}).items():
            setattr(b, "surface_" + k, v)
        for n, f in enumerate(faces):
            b.face[n] = int(f)
        if wall_velocity:
            for n, vel in wall_velocity.items():
                for c in range(3):
                    b.wall_velocity[n][c] = float(vel[c])
        b.zhi_theta_grad = zhi_theta_grad
        b.inflow_ustar, b.inflow_z0, b.inflow_direction = ustar, z0, direction
        b.kappa, b.Cmu0 = kappa, Cmu0
        b.inflow_inv_lmax = 0.0 if not l_max else 1.0 / l_max
        zs, ts = theta_ref
        b.theta_ref_n = len(zs)
        for n, (zz, tt) in enumerate(zip(zs, ts)):
            b.theta_ref_z[n] = zz
            b.theta_ref_theta[n] = tt
        return b


class Physics(ctypes.Structure):
    """gb_physics: forcing.*, convection.* and the residual scales."""
    _fields_ = [("gravity", ctypes.c_double), ("theta0", ctypes.c_double), ("coriolis", ctypes.c_int32),
                ("coriolis_3d", ctypes.c_int32), ("geostrophic", ctypes.c_int32), ("latitude", ctypes.c_double),
                ("rotation_period", ctypes.c_double), ("ug", ctypes.c_double), ("vg", ctypes.c_double),
                ("pressure_gradient", ctypes.c_double * 3), ("limiter", ctypes.c_int32),
                ("smooth_eps_velocity", ctypes.c_double), ("smooth_eps_theta", ctypes.c_double),
                ("log_mean", ctypes.c_int32), ("scale_velocity", ctypes.c_double), ("scale_theta", ctypes.c_double),
                ("scale_tke", ctypes.c_double), ("scale_height", ctypes.c_double), ("closure", ctypes.c_int32),
                ("turb_Cmu0", ctypes.c_double), ("turb_Cb", ctypes.c_double), ("turb_Rt_crit", ctypes.c_double),
                ("turb_Rt_min", ctypes.c_double), ("turb_max_geom_lscale", ctypes.c_double),
                ("turb_tke_floor", ctypes.c_double), ("turb_sigma_k", ctypes.c_double),
                ("turb_nu_molecular", ctypes.c_double), ("turb_alpha_molecular", ctypes.c_double),
                ("turb_kappa", ctypes.c_double), ("turb_ri_gate", ctypes.c_double),
                ("turb_realizability", ctypes.c_double), ("turb_nut_relax", ctypes.c_double)]

    @classmethod
    def make(cls, scale_height, **kw):
        """The reference's defaults (Source/Forcing.H: gravity 9.81, theta0 300, Coriolis
        off, rotation period 86400 s; convection van Leer, eps 1e-5; JvpScales 10, 10, 0.1;
        Source/Closure.H: turb.Cmu0 0.5562, Cb 0.35, Rt_crit -1, Rt_min -3,
        max_geom_lscale 30 m, tke_floor 0, sigma_k 1, molecular 0, kappa 0.41;
        closure off: the diffusivities are given)."""
        p = cls(gravity=9.81, theta0=300.0, coriolis=0, coriolis_3d=1, geostrophic=0, latitude=0.0,
                rotation_period=86400.0, ug=0.0, vg=0.0, limiter=LIMITER_VAN_LEER, smooth_eps_velocity=1e-5,
                smooth_eps_theta=1e-5, log_mean=0, scale_velocity=10.0, scale_theta=10.0, scale_tke=0.1,
                scale_height=scale_height, closure=0, turb_Cmu0=0.5562, turb_Cb=0.35, turb_Rt_crit=-1.0,
                turb_Rt_min=-3.0, turb_max_geom_lscale=30.0, turb_tke_floor=0.0, turb_sigma_k=1.0,
                turb_nu_molecular=0.0, turb_alpha_molecular=0.0, turb_kappa=0.41, turb_ri_gate=0.0,
                turb_realizability=0.0, turb_nut_relax=1.0)
        for k, v in kw.items():
            if k == "pressure_gradient":
                for d in range(3):
                    p.pressure_gradient[d] = v[d]
            else:
                setattr(p, k, v)
        return p


class SimplecOptions(ctypes.Structure):
    """gb_simplec_opts: simplec.*, steady.zline_sweeps, steady.sweep (0 zjacobi,
    1 lusgs), steady.line_alternate, turb.tke_floor and the correction's
    Poisson solver."""
    _fields_ = [("pressure_reltol", ctypes.c_double), ("alpha_p", ctypes.c_double),
                ("rotation_relax", ctypes.c_double), ("w_vnn_cap", ctypes.c_double),
                ("w_vnn_cap_slope_margin", ctypes.c_double), ("tke_floor", ctypes.c_double),
                ("zline_sweeps", ctypes.c_int32), ("precision", ctypes.c_int32), ("poisson", PoissonOptions),
                ("line_sweep", ctypes.c_int32), ("line_alternate", ctypes.c_int32)]

    @classmethod
    def make(cls, **kw):
        """The reference's defaults (Source/Simplec.H:80-90, Source/Driver.H:92)."""
        o = cls(pressure_reltol=1e-3, alpha_p=1.0, rotation_relax=0.3, w_vnn_cap=0.0, w_vnn_cap_slope_margin=4.0,
                tke_floor=0.0, zline_sweeps=2, precision=0, poisson=PoissonOptions.defaults(), line_sweep=0,
                line_alternate=0)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class InitOptions(ctypes.Structure):
    """gb_init_opts: init.* of the mass-consistent initializer and the
    projection's solver.poisson_*."""
    _fields_ = [("z_agl_min", ctypes.c_double), ("alpha_h", ctypes.c_double), ("alpha_v", ctypes.c_double),
                ("k_decay_height", ctypes.c_double), ("projection", ctypes.c_int32), ("obrien", ctypes.c_int32),
                ("poisson", PoissonOptions)]

    @classmethod
    def make(cls, **kw):
        """The reference's defaults (Source/Initializer.H:63-111, Source/Poisson.H:41-75)."""
        o = cls(z_agl_min=0.0, alpha_h=1.0, alpha_v=1.0, k_decay_height=0.0, projection=1, obrien=0,
                poisson=PoissonOptions.defaults())
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class InitResult(ctypes.Structure):
    _fields_ = [("divergence_before", ctypes.c_double), ("divergence_after", ctypes.c_double),
                ("poisson_iterations", ctypes.c_int32), ("poisson_final_residual", ctypes.c_double),
                ("obrien_top_residual", ctypes.c_double)]


class ProlongResult(ctypes.Structure):
    _fields_ = [("divergence_before", ctypes.c_double), ("divergence_after", ctypes.c_double),
                ("poisson_iterations", ctypes.c_int32), ("tke_clipped", ctypes.c_int64)]


class State(ctypes.Structure):
    _fields_ = [("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("w", ctypes.c_void_p), ("p", ctypes.c_void_p),
                ("theta", ctypes.c_void_p), ("tke", ctypes.c_void_p), ("z_nd", ctypes.c_void_p)]


class MeshFields(ctypes.Structure):
    _fields_ = [("detJ", ctypes.c_void_p), ("ax", ctypes.c_void_p), ("ay", ctypes.c_void_p), ("az", ctypes.c_void_p),
                ("z0", ctypes.c_void_p)]


class Diffusivities(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_void_p), ("gamma_theta", ctypes.c_void_p), ("gamma_tke", ctypes.c_void_p)]


class IterInfo(ctypes.Structure):
    _fields_ = [("residual_norms", ctypes.c_double * 6), ("max_speed", ctypes.c_double),
                ("mean_tke", ctypes.c_double), ("max_du", ctypes.c_double), ("max_dv", ctypes.c_double),
                ("max_dw", ctypes.c_double), ("last_sweep_du", ctypes.c_double), ("last_sweep_dv", ctypes.c_double),
                ("last_sweep_dw", ctypes.c_double), ("divergence_before", ctypes.c_double),
                ("divergence_after", ctypes.c_double), ("max_dp", ctypes.c_double),
                ("poisson_removed_mean", ctypes.c_double), ("poisson_iterations", ctypes.c_int32),
                ("max_dtheta", ctypes.c_double), ("max_dtke", ctypes.c_double), ("tke_clipped", ctypes.c_int64),
                ("mean_ustar", ctypes.c_double)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "residual_norms"}
        d["residual_norms"] = list(self.residual_norms)
        return d


class PredictorResult(ctypes.Structure):
    """gb_predictor_result (gust::MomentumPredictorResult)."""
    _fields_ = [("max_du", ctypes.c_double), ("max_dv", ctypes.c_double), ("max_dw", ctypes.c_double),
                ("last_sweep_du", ctypes.c_double), ("last_sweep_dv", ctypes.c_double),
                ("last_sweep_dw", ctypes.c_double)]


class PressureResult(ctypes.Structure):
    """gb_pressure_result (gust::PressureCorrectionResult)."""
    _fields_ = [("poisson_iterations", ctypes.c_int32), ("poisson_removed_mean", ctypes.c_double),
                ("divergence_before", ctypes.c_double), ("divergence_after", ctypes.c_double),
                ("max_dp", ctypes.c_double), ("max_du", ctypes.c_double), ("max_dv", ctypes.c_double),
                ("max_dw", ctypes.c_double)]


class ScalarResult(ctypes.Structure):
    """gb_scalar_result (gust::ScalarSweepResult)."""
    _fields_ = [("max_dq", ctypes.c_double), ("last_sweep", ctypes.c_double), ("clipped", ctypes.c_int64)]


CRITERION_MAX_RESIDUALS, CRITERION_MAX_MONITORS = 8, 4
NOT_STEADY, STEADY, DIVERGED = 0, 1, 2
LOOSE_NONE, LOOSE_RESIDUALS, LOOSE_MONITORS = 0, 1, 2


class SteadyHistory(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32), ("nonfinite", ctypes.c_int32), ("n_residuals", ctypes.c_int32),
                ("n_monitors", ctypes.c_int32), ("res_ref", ctypes.c_double * CRITERION_MAX_RESIDUALS),
                ("res_last", ctypes.c_double * CRITERION_MAX_RESIDUALS),
                ("monitor_values", ctypes.c_int32 * CRITERION_MAX_MONITORS),
                ("monitor_last", ctypes.c_double * CRITERION_MAX_MONITORS)]


class SequencingOptions(ctypes.Structure):
    """gb_sequencing_opts: steady.sequencing_* (defaults: off, drop 2 orders,
    monitor branch off, no hold on the seeded levels, start at cfl0)."""
    _fields_ = [("enabled", ctypes.c_int32), ("drop_orders", ctypes.c_double), ("monitor_tol", ctypes.c_double),
                ("hold", ctypes.c_int32), ("cfl_previous", ctypes.c_int32)]

    @classmethod
    def make(cls, **kw):
        o = cls(enabled=0, drop_orders=2.0, monitor_tol=0.0, hold=0, cfl_previous=0)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


def np_ptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


class DriverOptions(ctypes.Structure):
    """gb_driver_opts: steady.* of the pseudo-time driver and the criterion."""
    _fields_ = [("cfl0", ctypes.c_double), ("cfl_max", ctypes.c_double), ("ser_exponent", ctypes.c_double),
                ("ser_max_growth", ctypes.c_double), ("residual_tol", ctypes.c_double),
                ("residual_drop_orders", ctypes.c_double), ("residual_ref_iterations", ctypes.c_int32),
                ("monitor_rel_tol", ctypes.c_double), ("monitor_window", ctypes.c_int32),
                ("confidence", ctypes.c_double), ("confidence_height", ctypes.c_double)]

    @classmethod
    def make(cls, line_sweep=0, **kw):
        """The reference's defaults (cfl_max 8 with steady.sweep = lusgs, else 10)."""
        o = cls(cfl0=1.0, cfl_max=8.0 if line_sweep == 1 else 10.0, ser_exponent=1.0, ser_max_growth=2.0,
                residual_tol=5e-5, residual_drop_orders=4.0, residual_ref_iterations=5, monitor_rel_tol=1e-3,
                monitor_window=50, confidence=0.0, confidence_height=0.0)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


DRIVER_VERDICTS = {0: "running", 1: "steady", 2: "diverged", 3: "failed"}
