"""gust::SimplecStage on the GPU (Source/Simplec.H:185-263): one instance's
SIMPLEC outer iteration through the C ABI. The fields are torch tensors in
the grid layout (ablsteadyrans_b200.grid.Grid)."""
import ctypes

from . import abi
from .grid import GbGrid


def _declare(L):
    P = ctypes.c_void_p
    G = ctypes.POINTER(GbGrid)
    L.gb_simplec_create.argtypes = [P, G, ctypes.POINTER(abi.BC), ctypes.POINTER(abi.Physics),
                                    ctypes.POINTER(abi.SimplecOptions), P, ctypes.POINTER(abi.MeshFields),
                                    ctypes.POINTER(abi.Diffusivities), ctypes.POINTER(P)]
    L.gb_simplec_destroy.argtypes = [P]
    L.gb_simplec_fill_ghosts.argtypes = [P, ctypes.POINTER(abi.State)]
    L.gb_simplec_residual.argtypes = [P, ctypes.POINTER(abi.State), ctypes.POINTER(ctypes.c_void_p)]
    L.gb_simplec_iterate.argtypes = [P, ctypes.POINTER(abi.State), P, ctypes.POINTER(abi.IterInfo)]
    L.gb_local_dtau.argtypes = [P, ctypes.POINTER(abi.State), ctypes.c_double, P]
    L.gb_init_options_default.argtypes = [ctypes.POINTER(abi.InitOptions)]
    L.gb_driver_create.argtypes = [P, ctypes.POINTER(abi.State), ctypes.POINTER(abi.DriverOptions), ctypes.POINTER(P)]
    L.gb_driver_destroy.argtypes = [P]
    L.gb_driver_step.argtypes = [P, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(abi.IterInfo),
                                 ctypes.POINTER(ctypes.c_double)]
    L.gb_driver_run.argtypes = [ctypes.POINTER(P), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    L.gb_simplec_initialize.argtypes = [P, ctypes.POINTER(abi.State), ctypes.POINTER(abi.InitOptions),
                                        ctypes.POINTER(abi.InitResult)]
    L.gb_simplec_turbulence.argtypes = [P, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]
    L.gb_simplec_set_wall_distance.argtypes = [P, P]
    L.gb_simplec_implicit_rows.argtypes = [P, ctypes.POINTER(abi.State), ctypes.c_int32, P]
    L.gb_simplec_norms.argtypes = [P, ctypes.POINTER(abi.State), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]
    L.gb_simplec_confidence.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double)]
    L.gb_driver_criterion.argtypes = [P, ctypes.POINTER(P)]
    L.gb_driver_seed_reference.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
    L.gb_driver_release_hold.argtypes = [P]
    L.gb_driver_start_cfl.argtypes = [P, ctypes.c_double]
    L.gb_driver_status.argtypes = [P, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]
    L.gb_simplec_prolong.argtypes = [P, ctypes.POINTER(abi.State), G, ctypes.POINTER(abi.State), ctypes.c_double,
                                     ctypes.POINTER(abi.ProlongResult)]
    L.gb_momentum_predictor.argtypes = [P, ctypes.POINTER(abi.State), ctypes.POINTER(P), P, ctypes.POINTER(P),
                                        ctypes.POINTER(P), ctypes.POINTER(abi.PredictorResult)]
    L.gb_pressure_correction.argtypes = [P, ctypes.POINTER(abi.State), ctypes.POINTER(P),
                                         ctypes.POINTER(abi.PressureResult)]
    L.gb_scalar_sweep.argtypes = [P, ctypes.POINTER(abi.State), ctypes.c_int32, P, P, ctypes.c_int32,
                                  ctypes.POINTER(abi.ScalarResult)]
    L.gb_simplec_precondition.argtypes = [P, ctypes.POINTER(abi.State), P, ctypes.c_double, ctypes.c_int32,
                                          ctypes.POINTER(P), ctypes.POINTER(P)]


# The closure's fields and the surface state's planes, in the ABI's order.
CLOSURE_FIELDS = ("nu", "gamma_theta", "gamma_tke", "nut", "length", "Rt", "Ps", "Pb", "eps", "dSdk")
SURFACE_FIELDS = ("ustar", "speed", "zref", "d0", "inv_L", "tau_x", "tau_y", "tau_z", "drag", "kwall", "area")


FIELDS = ("u", "v", "w", "p", "theta", "tke")


class DeviceCase:
    """Device copies of one instance: state (u, v, w, p, theta, k), node
    heights, metrics, diffusivities."""

    def __init__(self, grid, z, J, ax, ay, az, nu, gamma_theta, gamma_tke, q=None, z0map=None):
        import torch

        def dev(a):
            return torch.from_numpy(a).cuda() if not isinstance(a, torch.Tensor) else a.cuda()

        self.grid = grid
        self.z, self.J, self.ax, self.ay, self.az = map(dev, (z, J, ax, ay, az))
        self.nu, self.gt, self.gk = map(dev, (nu, gamma_theta, gamma_tke))
        self.z0map = None if z0map is None else dev(z0map)
        self.q = {f: (dev(q[f]) if q is not None else torch.zeros(grid.shape, dtype=torch.float64, device="cuda"))
                  for f in FIELDS}

    @classmethod
    def from_oracle(cls, case):
        return cls(case.grid, case.z, case.J, case.ax, case.ay, case.az, case.nu, case.gt, case.gk, case.q,
                   getattr(case, "z0map", None))

    def state(self):
        return abi.State(*[self.q[f].data_ptr() for f in FIELDS], self.z.data_ptr())

    def mesh(self):
        return abi.MeshFields(self.J.data_ptr(), self.ax.data_ptr(), self.ay.data_ptr(), self.az.data_ptr(),
                              None if self.z0map is None else self.z0map.data_ptr())

    def diffusivities(self):
        return abi.Diffusivities(self.nu.data_ptr(), self.gt.data_ptr(), self.gk.data_ptr())

    def host(self, f):
        return self.q[f].cpu().numpy()


class SimplecStage:
    """One instance's SIMPLEC stage (gb_simplec)."""

    def __init__(self, ctx, case, bc, physics, options):
        from . import _lib_full, check
        self._L = _lib_full()
        if not getattr(self._L, "_gb_simplec", False):
            _declare(self._L)
            self._L._gb_simplec = True
        self.ctx = ctx
        self.case = case
        self.bc, self.physics, self.options = bc, physics, options
        self._m = case.mesh()
        self._d = case.diffusivities()
        self._h = ctypes.c_void_p()
        check(self._L.gb_simplec_create(ctx.handle, ctypes.byref(case.grid.c), ctypes.byref(bc), ctypes.byref(physics),
                                        ctypes.byref(options), ctypes.c_void_p(case.z.data_ptr()),
                                        ctypes.byref(self._m), ctypes.byref(self._d), ctypes.byref(self._h)))
        ctx.own(self)

    def fill_ghosts(self):
        from . import check
        st = self.case.state()
        check(self._L.gb_simplec_fill_ghosts(self._h, ctypes.byref(st)))

    def residual(self, out=None):
        """The six residuals at the state (into `out`, six grid tensors, when given)."""
        import torch
        from . import check
        R = out if out is not None else [torch.zeros(self.case.grid.shape, dtype=torch.float64, device="cuda")
                                         for _ in range(6)]
        arr = (ctypes.c_void_p * 6)(*[r.data_ptr() for r in R])
        st = self.case.state()
        check(self._L.gb_simplec_residual(self._h, ctypes.byref(st), arr))
        return R

    def implicit_rows(self, eq):
        """implicit_rows of equation eq (0 u .. 5 k) at the state: A (7 x grid)."""
        import torch
        from . import check
        A = torch.zeros((7,) + tuple(self.case.grid.shape), dtype=torch.float64, device="cuda")
        st = self.case.state()
        check(self._L.gb_simplec_implicit_rows(self._h, ctypes.byref(st), int(eq), ctypes.c_void_p(A.data_ptr())))
        return A

    def set_wall_distance(self, dist):
        """The closure's wall distance from now on (a device volume of the
        grid, e.g. gb.tucker_wall_distance's): turb.wall_distance = tucker."""
        from . import check
        check(self._L.gb_simplec_set_wall_distance(self._h, ctypes.c_void_p(dist.data_ptr())))

    def turbulence(self, closure=True, surface=True):
        """(closure fields, surface state) as dicts of host arrays: the
        closure's at the last residual, the wall state of the last fill."""
        import torch
        from . import check
        g = self.case.grid
        cf = [torch.zeros(g.shape, dtype=torch.float64, device="cuda") for _ in CLOSURE_FIELDS] if closure else None
        np_ = int(g.c.sy) * (g.ny + 1 + 2 * g.ng)
        ss = [torch.zeros(np_, dtype=torch.float64, device="cuda") for _ in SURFACE_FIELDS] if surface else None
        ca = (ctypes.c_void_p * len(cf))(*[t.data_ptr() for t in cf]) if cf else None
        sa = (ctypes.c_void_p * len(ss))(*[t.data_ptr() for t in ss]) if ss else None
        check(self._L.gb_simplec_turbulence(self._h, ca, sa))
        torch.cuda.synchronize()
        out_c = dict(zip(CLOSURE_FIELDS, [t.cpu().numpy() for t in cf])) if cf else None
        out_s = dict(zip(SURFACE_FIELDS, [t.cpu().numpy() for t in ss])) if ss else None
        return out_c, out_s

    def local_dtau(self, cfl, out=None):
        import torch
        from . import check
        dt = out if out is not None else torch.zeros(self.case.grid.shape, dtype=torch.float64, device="cuda")
        st = self.case.state()
        check(self._L.gb_local_dtau(self._h, ctypes.byref(st), float(cfl), ctypes.c_void_p(dt.data_ptr())))
        return dt

    def norms(self):
        """stage_norms at the stage's state: (six residual norms, three monitors)."""
        from . import check
        res, mon = (ctypes.c_double * 6)(), (ctypes.c_double * 3)()
        st = self.case.state()
        check(self._L.gb_simplec_norms(self._h, ctypes.byref(st), res, mon))
        return list(res), list(mon)

    def confidence(self, thresholds):
        """SimplecStage::confidence on the last iteration's residual: (share
        of the cells within the six thresholds, largest height above the
        ground of a cell that is not)."""
        from . import check
        share, height = ctypes.c_double(), ctypes.c_double()
        t = (ctypes.c_double * 6)(*[float(x) for x in thresholds])
        check(self._L.gb_simplec_confidence(self._h, t, ctypes.byref(share), ctypes.byref(height)))
        return share.value, height.value

    def local_dtau_of(self, state, cfl, out):
        """local_dtau at another state of this stage's grid (an abi.State)."""
        from . import check
        check(self._L.gb_local_dtau(self._h, ctypes.byref(state), float(cfl), ctypes.c_void_p(out.data_ptr())))
        return out

    def _fill_state(self, state):
        """The ghost fill of another state of this stage's grid (an abi.State)."""
        from . import check
        check(self._L.gb_simplec_fill_ghosts(self._h, ctypes.byref(state)))

    def iterate(self, dtau):
        from . import check
        info = abi.IterInfo()
        st = self.case.state()
        check(self._L.gb_simplec_iterate(self._h, ctypes.byref(st), ctypes.c_void_p(dtau.data_ptr()), ctypes.byref(info)))
        return info

    def momentum_predictor(self, R, dtau, with_fields=False):
        """gust::momentum_predictor (Predictor.H:242-252) on the stage's state
        with R the residual at it (gb_simplec_residual's, after
        fill_ghosts): returns the PredictorResult, and with with_fields also
        (ap, d) as three device tensors each."""
        import torch
        from . import check
        res = abi.PredictorResult()
        st = self.case.state()
        Ra = (ctypes.c_void_p * 6)(*[r.data_ptr() for r in R])
        ap = d = None
        apa = da = None
        if with_fields:
            ap = [torch.zeros(self.case.grid.shape, dtype=torch.float64, device="cuda") for _ in range(3)]
            d = [torch.zeros(self.case.grid.shape, dtype=torch.float64, device="cuda") for _ in range(3)]
            apa = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in ap])
            da = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in d])
        check(self._L.gb_momentum_predictor(self._h, ctypes.byref(st), Ra, ctypes.c_void_p(dtau.data_ptr()), apa, da,
                                            ctypes.byref(res)))
        return (res, ap, d) if with_fields else res

    def pressure_correction(self, d=None):
        """gust::pressure_correction (Simplec.H:139-141) on the stage's state
        with the denominators d (three device tensors; None: the last
        predictor's). Returns the PressureResult."""
        from . import check
        res = abi.PressureResult()
        st = self.case.state()
        da = None if d is None else (ctypes.c_void_p * 3)(*[t.data_ptr() for t in d])
        check(self._L.gb_pressure_correction(self._h, ctypes.byref(st), da, ctypes.byref(res)))
        return res

    def scalar_sweep(self, eq, R_eq, dtau, clip=True):
        """gust::scalar_sweep (Simplec.H:156-163) of eq (4 theta, 5 k) on the
        stage's state. Returns the ScalarResult."""
        from . import check
        res = abi.ScalarResult()
        st = self.case.state()
        check(self._L.gb_scalar_sweep(self._h, ctypes.byref(st), int(eq), ctypes.c_void_p(R_eq.data_ptr()),
                                      ctypes.c_void_p(dtau.data_ptr()), int(bool(clip)), ctypes.byref(res)))
        return res

    def precondition(self, r, dtau=None, inf_cfl=10.0, denominators=1):
        """gust::SimplecPreconditioner setup at the stage's state and one
        apply to r (six device tensors): dq for (D + J) dq = r by one SIMPLEC
        iteration (denominators 1: d = a_P; 2: the stage's d)."""
        import torch
        from . import check
        dq = [torch.zeros(self.case.grid.shape, dtype=torch.float64, device="cuda") for _ in range(6)]
        st = self.case.state()
        ra = (ctypes.c_void_p * 6)(*[t.data_ptr() for t in r])
        da = (ctypes.c_void_p * 6)(*[t.data_ptr() for t in dq])
        check(self._L.gb_simplec_precondition(self._h, ctypes.byref(st),
                                              None if dtau is None else ctypes.c_void_p(dtau.data_ptr()),
                                              float(inf_cfl), int(denominators), ra, da))
        return dq

    def initialize(self, options=None):
        """gust::initialize_state with init.first_guess = profile: the
        mass-consistent initial state (gb_simplec_initialize) in place."""
        from . import check
        o = options if options is not None else abi.InitOptions.make()
        res = abi.InitResult()
        st = self.case.state()
        check(self._L.gb_simplec_initialize(self._h, ctypes.byref(st), ctypes.byref(o), ctypes.byref(res)))
        return res

    def prolong(self, coarse, reltol):
        """prolong_state (Transfer.cpp:322-385) into this stage's state from
        a coarser level's DeviceCase (its valid points): the bilinear fields, k at the floor, the ghost fill and the
        projection to reltol. Returns the ProlongResult."""
        from . import check
        res = abi.ProlongResult()
        st, sc = self.case.state(), coarse.state()
        check(self._L.gb_simplec_prolong(self._h, ctypes.byref(st), ctypes.byref(coarse.grid.c), ctypes.byref(sc),
                                         float(reltol), ctypes.byref(res)))
        return res

    def own(self, obj):
        """Record a native object made on this stage (a Newton core): close()
        destroys the live ones first."""
        import weakref
        deps = getattr(self, "_dependents", [])
        self._dependents = [r for r in deps if r() is not None] + [weakref.ref(obj)]

    def close(self):
        from . import check
        for r in reversed(getattr(self, "_dependents", [])):
            obj = r()
            if obj is not None:
                obj.close()
        self._dependents = []
        if self._h:
            check(self._L.gb_simplec_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NativeDriver:
    """gust::Driver in C++ (gb_driver): the local dtau, one iteration, the
    steady criterion and the SER law per step, with no Python in the loop."""

    def __init__(self, stage, options=None):
        from . import check
        self.stage = stage
        self._L = stage._L
        self.options = options or abi.DriverOptions.make(getattr(stage.options, "line_sweep", 0))
        self._state = stage.case.state()
        self._h = ctypes.c_void_p()
        check(self._L.gb_driver_create(stage._h, ctypes.byref(self._state), ctypes.byref(self.options),
                                       ctypes.byref(self._h)))
        stage.ctx.own(self)
        self.iterations = 0

    @property
    def handle(self):
        return self._h

    def step(self):
        """One step; returns ('running' | 'steady' | 'diverged', IterInfo, cfl used)."""
        from . import check
        v = ctypes.c_int32()
        info = abi.IterInfo()
        cfl = ctypes.c_double()
        check(self._L.gb_driver_step(self._h, ctypes.byref(v), ctypes.byref(info), ctypes.byref(cfl)))
        self.iterations += 1
        return abi.DRIVER_VERDICTS[v.value], info, cfl.value

    @property
    def criterion(self):
        """The driver's steady criterion (history, verdict, loose stop)."""
        from . import check
        from .driver import SteadyCriterion
        h = ctypes.c_void_p()
        check(self._L.gb_driver_criterion(self._h, ctypes.byref(h)))
        return SteadyCriterion(handle=h, owner=self)

    def seed_reference(self, ref):
        """Driver::seed_reference: the coarsest level's references (before the first step)."""
        from . import check
        check(self._L.gb_driver_seed_reference(self._h, (ctypes.c_double * 6)(*[float(x) for x in ref])))

    def release_hold(self):
        """Driver::release_reference_hold (steady.sequencing_hold = 0)."""
        from . import check
        check(self._L.gb_driver_release_hold(self._h))

    def start_cfl(self, cfl):
        """Driver::start_cfl (steady.sequencing_cfl_start = previous)."""
        from . import check
        check(self._L.gb_driver_start_cfl(self._h, float(cfl)))

    def status(self):
        """(hold iterations, the next step's CFL, r_n of the last step)."""
        from . import check
        hold, cfl, r = ctypes.c_int32(), ctypes.c_double(), ctypes.c_double()
        check(self._L.gb_driver_status(self._h, ctypes.byref(hold), ctypes.byref(cfl), ctypes.byref(r)))
        return hold.value, cfl.value, r.value

    def close(self):
        from . import check
        if self._h:
            check(self._L.gb_driver_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_drivers(drivers, max_iterations, threads=0):
    """gb_driver_run: every driver steps until it is steady, diverged or has
    taken max_iterations steps, on native threads (0: one per driver).
    Returns [(verdict, iterations)]."""
    from . import check
    if not drivers:
        return []
    L = drivers[0]._L
    n = len(drivers)
    hs = (ctypes.c_void_p * n)(*[d.handle.value for d in drivers])
    v = (ctypes.c_int32 * n)()
    it = (ctypes.c_int32 * n)()
    check(L.gb_driver_run(hs, n, int(max_iterations), int(threads), v, it))
    out = []
    for d, a, b in zip(drivers, v, it):
        d.iterations += b
        out.append((abi.DRIVER_VERDICTS[a], b))
    return out
