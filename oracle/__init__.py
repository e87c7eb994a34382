"""ORACLE -- test infrastructure, not product code.

ctypes bindings of liboracle.so, the FP64 C restatement of the reference's
SIMPLEC hot path (gust_oracle.c). Only the tests, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it, as the checker; the product path never
calls it. Arrays are numpy float64, C-contiguous, in the grid layout of
include/gust_b200.h (ablsteadyrans_b200.grid.Grid.shape).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force=False):
    args = ["make", "-C", HERE]
    if force:
        args.append("-B")
    r = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout.decode(errors="replace"))
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or the machine type."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.machine()


def use_fast_build():
    """Switch this process's oracle calls to the speed build of the same
    sources (-O3 -march=native, contraction allowed; results differ from the
    parity build by rounding), compiled on this host into a directory named
    by the CPU model. Only the timed CPU baseline uses it. Returns the
    library's path."""
    import hashlib
    global _lib
    d = os.path.join(HERE, "_fast", hashlib.sha1(cpu_model().encode()).hexdigest()[:12])
    r = subprocess.run(["make", "-C", HERE, "fast", f"FAST_DIR={d}"], stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("oracle speed build failed:\n" + r.stdout.decode(errors="replace"))
    path = os.path.join(d, "liboracle_fast.so")
    L = ctypes.CDLL(path)
    _declare(L)
    _declare_simplec(L)
    L._og_simplec = True
    _lib = L
    return path


def _declare(L):
    from ablsteadyrans_b200.grid import GbGrid
    G = ctypes.POINTER(GbGrid)
    P = ctypes.c_void_p
    i32, f64 = ctypes.c_int32, ctypes.c_double
    L.og_set_threads.argtypes = [i32]
    L.og_max_threads.restype = i32
    L.og_fill_periodic.argtypes = [G, i32, P, i32]
    L.og_override_sync.argtypes = [G, i32, P]
    L.og_zline_jacobi.argtypes = [G, i32, P, P, P, i32, P]
    L.og_zline_jacobi.restype = f64
    L.og_zline_lusgs.argtypes = [G, i32, P, P, P, i32, i32, i32, P]
    L.og_zline_lusgs.restype = f64
    # mesh and Poisson layer
    I = ctypes.POINTER(ctypes.c_int)
    L.og_btf_heights.argtypes = [G, P, P, P]
    L.og_metrics.argtypes = [G, P, P, P, P, P, P]
    L.og_poisson_fill_ghosts.argtypes = [G, I, P, i32]
    L.og_poisson_zero_flux_faces.argtypes = [G, I]
    L.og_poisson_zero_flux_faces.restype = i32
    L.og_poisson_apply.argtypes = [G, I, P, P, P, P, P, P, P]
    L.og_poisson_fluxes.argtypes = [G, I, P, P, P, P, P, P, P, P]
    L.og_face_divergence.argtypes = [G, P, P, P, P, P, P, P, P]
    L.og_weighted_mean.argtypes = [G, P, P]
    L.og_weighted_mean.restype = f64
    L.og_mg_create.argtypes = [G, I, P, P, P, P, P, i32, i32, i32, i32, i32]
    L.og_mg_create.restype = P
    L.og_mg_destroy.argtypes = [P]
    L.og_mg_levels.argtypes = [P]
    L.og_mg_levels.restype = i32
    L.og_mg_vcycle.argtypes = [P, P, P]
    L.og_mg_set_cross.argtypes = [P, P, P, P]
    L.og_mg_apply.argtypes = [P, P, P]
    L.og_poisson_add_cross.argtypes = [G, I, P, P, P, P, P, P]
    L.og_poisson_cross_flux.argtypes = [G, I, P, P, P, P]
    L.og_poisson_solve.argtypes = [P, P, P, f64, f64, i32, i32, i32, ctypes.POINTER(f64)]
    L.og_poisson_solve.restype = i32
    L.og_line_tridiag.argtypes = [G, I, i32, P, P, P, P, P, i32, i32, i32, ctypes.POINTER(f64),
                                  ctypes.POINTER(f64), ctypes.POINTER(f64)]


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous float64"
    return ctypes.c_void_p(a.ctypes.data)


def set_threads(n):
    lib().og_set_threads(int(n))


def max_threads():
    return int(lib().og_max_threads())


def fill_periodic(grid, loc, f, layers=1):
    lib().og_fill_periodic(ctypes.byref(grid.c), loc, _p(f), layers)


def zline_jacobi(grid, loc, A, ap, rhs, sweeps, delta):
    """Source/Predictor.cpp:87-127 restated; returns the last sweep's change."""
    return float(lib().og_zline_jacobi(ctypes.byref(grid.c), loc, _p(A), _p(ap), _p(rhs), int(sweeps), _p(delta)))


def zline_lusgs(grid, loc, A, ap, rhs, sweeps, delta, order=0, alternate=0):
    """Source/LineSweeps.cpp:183-210, 415-428 restated (line_ghosts =
    lagged): order 0 sequential, 1 diagonal wavefronts; returns the last
    backward pass's change."""
    return float(lib().og_zline_lusgs(ctypes.byref(grid.c), loc, _p(A), _p(ap), _p(rhs), int(sweeps), int(order),
                                      int(alternate), _p(delta)))


# ------------------------------------------------------------ mesh / Poisson
PERIODIC, NEUMANN, DIRICHLET = 0, 1, 2


def _bc(bc):
    arr = (ctypes.c_int * 6)(*[int(b) for b in bc])
    return arr


def btf_heights(grid, zlevels, ground):
    """BTF node heights (ERF_TerrainMetrics.cpp BTF, Source/Mesh.cpp fill_ghost_columns).
    ground: (ny+3, nx+3) heights of node columns i, j in [-1, n+1]."""
    z = grid.np_zeros()
    zl = np.ascontiguousarray(zlevels, dtype=np.float64)
    gr = np.ascontiguousarray(ground, dtype=np.float64)
    lib().og_btf_heights(ctypes.byref(grid.c), _p(zl), _p(gr), _p(z))
    return z


def metrics(grid, z):
    """detJ, ax, ay, az, z_cc (ERF_TerrainMetrics.cpp:680-808)."""
    out = [grid.np_zeros() for _ in range(5)]
    lib().og_metrics(ctypes.byref(grid.c), _p(z), *[_p(a) for a in out])
    return out


def poisson_fill_ghosts(grid, bc, phi, ground_even=True):
    lib().og_poisson_fill_ghosts(ctypes.byref(grid.c), _bc(bc), _p(phi), int(ground_even))


def poisson_apply(grid, bc, AX, AY, AZ, J, z, phi):
    y = grid.np_zeros()
    lib().og_poisson_apply(ctypes.byref(grid.c), _bc(bc), _p(AX), _p(AY), _p(AZ), _p(J), _p(z), _p(phi), _p(y))
    return y


def poisson_fluxes(grid, bc, z, phi, bx=None, by=None, bz=None):
    f = [grid.np_zeros() for _ in range(3)]
    lib().og_poisson_fluxes(ctypes.byref(grid.c), _bc(bc), _p(z), _p(phi), _p(bx), _p(by), _p(bz), *[_p(a) for a in f])
    return f


def poisson_apply_split(grid, bc, ax, ay, az, J, z, phi, bx, by, bz, z_cross):
    """PoissonSolver::apply with FaceCoeffs {bx, by, bz, z_cross}
    (Source/Poisson.cpp:524-529): the operator on the premultiplied areas plus,
    when z_cross is given, the split correction (add_cross)."""
    AX, AY, AZ = ax * bx, ay * by, az * bz
    y = poisson_apply(grid, bc, AX, AY, AZ, J, z, phi)
    if z_cross is not None:
        d = np.ascontiguousarray(bz - z_cross)
        lib().og_poisson_add_cross(ctypes.byref(grid.c), _bc(bc), _p(az), _p(d), _p(J), _p(z), _p(phi), _p(y))
    return y


def poisson_fluxes_split(grid, bc, z, phi, bx, by, bz, z_cross):
    """The solve's fluxes with FaceCoeffs {bx, by, bz, z_cross}
    (Source/Poisson.cpp:603-615)."""
    f = poisson_fluxes(grid, bc, z, phi, bx, by, bz)
    if z_cross is not None:
        d = np.ascontiguousarray(bz - z_cross)
        lib().og_poisson_cross_flux(ctypes.byref(grid.c), _bc(bc), _p(d), _p(z), _p(phi), _p(f[2]))
    return f


def face_divergence(grid, ax, ay, az, J, fx, fy, fz):
    d = grid.np_zeros()
    lib().og_face_divergence(ctypes.byref(grid.c), _p(ax), _p(ay), _p(az), _p(J), _p(fx), _p(fy), _p(fz), _p(d))
    return d


def weighted_mean(grid, f, J):
    return float(lib().og_weighted_mean(ctypes.byref(grid.c), _p(f), _p(J)))


class Multigrid:
    """This project's multigrid (poisson.c): levels, one V-cycle, the solve."""

    def __init__(self, grid, bc, z, J, AX, AY, AZ, max_levels=12, min_coarse=2, nu1=1, nu2=1, nu_coarse=8):
        self.grid = grid
        self._keep = [np.ascontiguousarray(a) for a in (z, J, AX, AY, AZ)]
        self._h = lib().og_mg_create(ctypes.byref(grid.c), _bc(bc), *[_p(a) for a in self._keep],
                                     max_levels, min_coarse, nu1, nu2, nu_coarse)

    @property
    def levels(self):
        return int(lib().og_mg_levels(self._h))

    def set_cross(self, az, bz, z_cross):
        """FaceCoeffs::z_cross for the solve's operator (not the V-cycle)."""
        lib().og_mg_set_cross(self._h, _p(np.ascontiguousarray(az)), _p(bz), _p(z_cross))

    def apply(self, phi):
        """The solve's operator (the split correction included when set)."""
        y = self.grid.np_zeros()
        lib().og_mg_apply(self._h, _p(phi), _p(y))
        return y

    def vcycle(self, r):
        e = self.grid.np_zeros()
        lib().og_mg_vcycle(self._h, _p(np.ascontiguousarray(r)), _p(e))
        return e

    def solve(self, rhs, reltol=1e-10, abstol=0.0, max_iter=200, restart=30, precond=True):
        """Returns (phi, iterations, initial residual, final residual, removed mean);
        rhs is modified (its J-weighted mean removed when singular)."""
        phi = self.grid.np_zeros()
        res = (ctypes.c_double * 3)()
        it = lib().og_poisson_solve(self._h, _p(rhs), _p(phi), reltol, abstol, max_iter, restart, int(precond), res)
        return phi, int(it), res[0], res[1], res[2]

    def close(self):
        if self._h:
            lib().og_mg_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ------------------------------------------------------------------ SIMPLEC
def _declare_simplec(L):
    from ablsteadyrans_b200.abi import BC, Diffusivities, IterInfo, MeshFields, Physics, SimplecOptions, State
    from ablsteadyrans_b200.grid import GbGrid
    G = ctypes.POINTER(GbGrid)
    P = ctypes.c_void_p
    i32, f64 = ctypes.c_int32, ctypes.c_double
    PP = ctypes.POINTER(ctypes.c_void_p)
    L.og_fill_ghosts.argtypes = [G, ctypes.POINTER(BC), P, P, P, P, P, P, P]
    L.og_residual.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), ctypes.POINTER(State),
                              ctypes.POINTER(MeshFields), ctypes.POINTER(Diffusivities), PP]
    L.og_implicit_rows.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), i32, P, P, P, P, P,
                                   ctypes.POINTER(Diffusivities), P]
    L.og_simplec_iterate.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), ctypes.POINTER(SimplecOptions),
                                     ctypes.POINTER(State), ctypes.POINTER(MeshFields), ctypes.POINTER(Diffusivities),
                                     P, PP, ctypes.POINTER(IterInfo)]
    L.og_simplec_iterate.restype = i32
    from ablsteadyrans_b200.abi import InitOptions
    L.og_initialize.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(InitOptions), ctypes.POINTER(State),
                                ctypes.POINTER(MeshFields), P]
    L.og_initialize.restype = i32
    L.og_implicit_rows2.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), i32, P, P, P, P, P,
                                    ctypes.POINTER(Diffusivities), PP, PP, P]
    L.og_prolong_fields.argtypes = [G, ctypes.POINTER(State), G, ctypes.POINTER(State), i32]
    L.og_set_nut_history.argtypes = [P]
    L.og_set_wall_distance.argtypes = [P]
    L.og_tucker_distance.argtypes = [G, P, P, P]
    L.og_restrict_state.argtypes = [G, ctypes.POINTER(State), ctypes.POINTER(MeshFields), G, ctypes.POINTER(State),
                                    ctypes.POINTER(MeshFields), i32, P]
    L.og_prolong_state.argtypes = [G, ctypes.POINTER(State), G, ctypes.POINTER(State), i32, ctypes.POINTER(BC),
                                   ctypes.POINTER(Physics), ctypes.POINTER(SimplecOptions), ctypes.POINTER(MeshFields),
                                   f64, ctypes.POINTER(f64)]
    L.og_prolong_state.restype = i32
    L.og_fill_ghosts2.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), P, P, P, P, P, P, P, P, PP]
    L.og_residual2.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), ctypes.POINTER(State),
                               ctypes.POINTER(MeshFields), ctypes.POINTER(Diffusivities), PP, PP, PP]
    L.og_simplec_iterate2.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), ctypes.POINTER(SimplecOptions),
                                      ctypes.POINTER(State), ctypes.POINTER(MeshFields), ctypes.POINTER(Diffusivities),
                                      P, PP, ctypes.POINTER(IterInfo), PP, PP]
    L.og_simplec_iterate2.restype = i32
    L.og_stage_steps.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), ctypes.POINTER(SimplecOptions),
                                 ctypes.POINTER(State), ctypes.POINTER(MeshFields), ctypes.POINTER(Diffusivities),
                                 P, PP, PP, PP, PP, P, P, P]
    L.og_stage_steps.restype = i32
    L.og_closure_evaluate.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), P, P, P, P, P, P, P, PP]
    L.og_surface_state.argtypes = [G, ctypes.POINTER(BC), ctypes.POINTER(Physics), P, P, P, P, P, PP]
    L.og_surface_state.restype = i32
    L.og_height_above_ground.argtypes = [G, P, P]
    L.og_obrien_omega.argtypes = [G, P, P, P, P, P, P, P, P]
    L.og_obrien_omega.restype = f64
    L.og_local_dtau.argtypes = [G, P, P, P, P, P, P, f64, P]
    L.og_transport_fluxes.argtypes = [G, P, P, P, P, P, P, P, P, P]
    L.og_velocity_divergence.argtypes = [G, P, P, P, P, P, P, P, P, P]
    L.og_pressure_gradient.argtypes = [G, P, P, P, P, P, P, P, P]
    L.og_convection.argtypes = [G, i32, P, P, P, P, P, i32, f64, i32, P]
    L.og_scalar_diffusive_fluxes.argtypes = [G, P, P, P, i32, P, P, P]
    L.og_momentum_diffusive_fluxes.argtypes = [G, i32, P, P, P, P, P, i32, P, P, P]
    L.og_flux_divergence.argtypes = [G, i32, P, P, P, P, P]
    L.og_implicit_coefficients.argtypes = [G, i32, P, P, P, P, P, P, i32, P]
    L.og_omega_from_w.argtypes = [G, P, P, P, P, P, i32]
    L.og_w_from_omega.argtypes = [G, P, P, P, P, P]
    L.og_face_dtau.argtypes = [G, P, P, P, P]


class Case:
    """The host arrays of one SIMPLEC instance in the grid layout: state, mesh,
    diffusivities, and the ctypes views the oracle and the GPU take."""

    FIELDS = ("u", "v", "w", "p", "theta", "tke")

    def __init__(self, grid, z, J, ax, ay, az, nu, gamma_theta, gamma_tke, z0map=None):
        self.grid = grid
        self.z, self.J, self.ax, self.ay, self.az = z, J, ax, ay, az
        self.nu, self.gt, self.gk = nu, gamma_theta, gamma_tke
        self.z0map = z0map                 # per-column roughness plane (CLOSURE_FIELDS / SURFACE_FIELDS below)
        self.q = {f: grid.np_zeros() for f in self.FIELDS}
        self.cf = None                     # the closure's fields of the last iteration (with turbulence)
        self.closure_nu = None             # nu the next local dtau reads (0 before the first iteration)
        self.nut_hist = None               # the closure's nu_t history (Closure::accept), None before the first

    def state(self):
        from ablsteadyrans_b200.abi import State
        return State(*[self.q[f].ctypes.data for f in self.FIELDS], self.z.ctypes.data)

    def mesh(self):
        from ablsteadyrans_b200.abi import MeshFields
        return MeshFields(self.J.ctypes.data, self.ax.ctypes.data, self.ay.ctypes.data, self.az.ctypes.data,
                          None if self.z0map is None else self.z0map.ctypes.data)

    def diffusivities(self):
        from ablsteadyrans_b200.abi import Diffusivities
        return Diffusivities(self.nu.ctypes.data, self.gt.ctypes.data, self.gk.ctypes.data)

    def copy(self):
        c = Case(self.grid, self.z, self.J, self.ax, self.ay, self.az, self.nu, self.gt, self.gk, self.z0map)
        c.q = {f: a.copy() for f, a in self.q.items()}
        c.nut_hist = None if self.nut_hist is None else self.nut_hist.copy()
        return c

    def plane(self):
        """A zeroed per-column plane of the grid (the layout of z0map and the surface state)."""
        g = self.grid
        return np.zeros(int(g.c.sy) * (g.ny + 1 + 2 * g.ng))


def _L():
    L = lib()
    if not getattr(L, "_og_simplec", False):
        _declare_simplec(L)
        L._og_simplec = True
    return L


# The closure's fields (volumes) and the surface state's columns (planes), in the oracle's order.
CLOSURE_FIELDS = ("nu", "gamma_theta", "gamma_tke", "nut", "length", "Rt", "Ps", "Pb", "eps", "dSdk")
SURFACE_FIELDS = ("ustar", "speed", "zref", "d0", "inv_L", "tau_x", "tau_y", "tau_z", "drag", "kwall", "area")


def _arrays(arrs):
    return (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def fill_ghosts(case, bc, phys=None):
    """BoundaryConditions::fill_ghosts; with a surface_layer ground returns the
    surface state (dict of planes) the ground fill used."""
    q = case.q
    ss = [case.plane() for _ in SURFACE_FIELDS]
    _L().og_fill_ghosts2(ctypes.byref(case.grid.c), ctypes.byref(bc), None if phys is None else ctypes.byref(phys),
                         _p(case.z0map), *[_p(q[f]) for f in Case.FIELDS], _p(case.z), _arrays(ss))
    return dict(zip(SURFACE_FIELDS, ss))


def residual(case, bc, phys, fields=False):
    """Residual.cpp:159-256 at the case's state (ghosts filled by the caller);
    with fields=True also (closure fields, surface state) as dicts."""
    _history(case)
    R = [case.grid.np_zeros() for _ in range(6)]
    cf = [case.grid.np_zeros() for _ in CLOSURE_FIELDS]
    ss = [case.plane() for _ in SURFACE_FIELDS]
    st, m, d = case.state(), case.mesh(), case.diffusivities()
    _L().og_residual2(ctypes.byref(case.grid.c), ctypes.byref(bc), ctypes.byref(phys), ctypes.byref(st), ctypes.byref(m),
                      ctypes.byref(d), _arrays(R), _arrays(cf), _arrays(ss))
    if fields:
        return R, dict(zip(CLOSURE_FIELDS, cf)), dict(zip(SURFACE_FIELDS, ss))
    return R


def closure_fields(case, bc, phys):
    """Closure::evaluate at the case's state (ghosts filled): dict of volumes."""
    _history(case)
    q = case.q
    cf = [case.grid.np_zeros() for _ in CLOSURE_FIELDS]
    _L().og_closure_evaluate(ctypes.byref(case.grid.c), ctypes.byref(bc), ctypes.byref(phys), _p(q["u"]), _p(q["v"]),
                             _p(q["w"]), _p(q["theta"]), _p(q["tke"]), _p(case.z), _p(case.z0map), _arrays(cf))
    return dict(zip(CLOSURE_FIELDS, cf))


def surface_state(case, bc, phys):
    """compute_surface_state's columns (ghosts filled): (dict of planes, bad columns)."""
    q = case.q
    ss = [case.plane() for _ in SURFACE_FIELDS]
    bad = _L().og_surface_state(ctypes.byref(case.grid.c), ctypes.byref(bc), ctypes.byref(phys), _p(q["u"]), _p(q["v"]),
                                _p(q["w"]), _p(case.z), _p(case.z0map), _arrays(ss))
    return dict(zip(SURFACE_FIELDS, ss)), int(bad)


def implicit_rows(case, bc, phys, eq, cf=None, ss=None):
    """implicit_rows (Residual.cpp:272-304) of equation eq (0 u .. 5 k) with the
    case's transport fluxes: the given diffusivities, or the closure's fields
    cf and the surface state ss (dicts, as residual(fields=True) gives them):
    A (N_COEFS x grid)."""
    g = case.grid
    q = case.q
    F = transport_fluxes(g, q["u"], q["v"], q["w"], case.z, case.ax, case.ay)
    A = g.np_zeros(7)
    d = case.diffusivities()
    ca = None if cf is None else _arrays([cf[n] for n in CLOSURE_FIELDS])
    sa = None if ss is None else _arrays([ss[n] for n in SURFACE_FIELDS])
    _L().og_implicit_rows2(ctypes.byref(g.c), ctypes.byref(bc), ctypes.byref(phys), int(eq), *[_p(f) for f in F],
                           _p(case.z), _p(case.J), ctypes.byref(d), ca, sa, _p(A))
    return A


def prolong_fields(coarse, fine, r):
    """prolong_fields (Transfer.cpp:290-320): the fine case's state from the
    coarse case's valid points, r the ratio of the cell sizes."""
    sc, sf = coarse.state(), fine.state()
    _L().og_prolong_fields(ctypes.byref(coarse.grid.c), ctypes.byref(sc), ctypes.byref(fine.grid.c), ctypes.byref(sf), int(r))


def restrict_state(fine, coarse, r):
    """restrict_state (Transfer.cpp:199-286) of the fine case's state into
    the coarse case's; returns the coarse Omega. The fine u and v need one
    ghost layer."""
    om = coarse.grid.np_zeros()
    sf, sc = fine.state(), coarse.state()
    mf, mc = fine.mesh(), coarse.mesh()
    _L().og_restrict_state(ctypes.byref(fine.grid.c), ctypes.byref(sf), ctypes.byref(mf), ctypes.byref(coarse.grid.c),
                           ctypes.byref(sc), ctypes.byref(mc), int(r), _p(om))
    return om


def prolong_state(coarse, fine, r, bc, phys, opts, reltol=1e-10):
    """prolong_state (Transfer.cpp:322-385) into the fine case: returns
    (status, [divergence before, after, Poisson iterations, k cells raised])."""
    info = (ctypes.c_double * 4)()
    fine.nut_hist = None   # the prolonged state is a new level's: no nu_t history
    sc, sf, m = coarse.state(), fine.state(), fine.mesh()
    rc = _L().og_prolong_state(ctypes.byref(coarse.grid.c), ctypes.byref(sc), ctypes.byref(fine.grid.c),
                               ctypes.byref(sf), int(r), ctypes.byref(bc), ctypes.byref(phys), ctypes.byref(opts),
                               ctypes.byref(m), float(reltol), info)
    return int(rc), list(info)


def height_above_ground(case):
    d = case.grid.np_zeros()
    _L().og_height_above_ground(ctypes.byref(case.grid.c), _p(case.z), _p(d))
    return d


def local_dtau(case, cfl, use_nu=True, nu=None, phys=None):
    """local_dtau with nu: the given one, else with the closure (phys.closure)
    the last iteration's nu (0 before the first, Simplec.cpp:328), else the
    case's diffusivity."""
    dt = case.grid.np_zeros()
    q = case.q
    if nu is None and use_nu:
        if phys is not None and phys.closure:
            nu = case.closure_nu if case.closure_nu is not None else case.grid.np_zeros()
        else:
            nu = case.nu
    _L().og_local_dtau(ctypes.byref(case.grid.c), _p(q["u"]), _p(q["v"]), _p(q["w"]), _p(case.z), _p(case.J),
                       _p(nu) if use_nu else None, float(cfl), _p(dt))
    return dt


def _history(case):
    """The closure's nu_t history and wall distance of the case for the next
    evaluations (the wall distance: case.wall_dist, or the height above the
    ground when it is None)."""
    h = getattr(case, "nut_hist", None)
    _L().og_set_nut_history(_p(h) if h is not None else None)
    d = getattr(case, "wall_dist", None)
    _L().og_set_wall_distance(_p(d) if d is not None else None)


def tucker_bc(grid):
    """tucker_bc (Source/WallDistance.cpp:65-76): periodic lateral directions
    stay periodic, other lateral faces zero flux, the ground Dirichlet, the
    top zero flux."""
    x = PERIODIC if grid.periodic_x else NEUMANN
    y = PERIODIC if grid.periodic_y else NEUMANN
    return (x, y, DIRICHLET, x, y, NEUMANN)


def tucker_wall_distance(grid, z, reltol=1e-12, max_iter=400):
    """tucker_wall_distance (Source/WallDistance.cpp:78-94): solve
    laplacian(phi) = -1 with phi = 0 on the ground (tucker_bc) on the
    terrain mesh, then Tucker's distance from phi and its ghosts
    (og_tucker_distance). Returns (dist, Poisson iterations)."""
    J, ax, ay, az, _ = metrics(grid, z)
    bc = tucker_bc(grid)
    mg = Multigrid(grid, bc, z, J, ax, ay, az)
    rhs = grid.np_zeros()
    rhs[grid.valid(0)] = -1.0
    phi, it, _, _, _ = mg.solve(rhs, reltol=reltol, max_iter=max_iter)
    mg.close()
    poisson_fill_ghosts(grid, bc, phi, ground_even=False)
    d = grid.np_zeros()
    _L().og_tucker_distance(ctypes.byref(grid.c), _p(z), _p(phi), _p(d))
    return d, it


def simplec_iterate(case, bc, phys, opts, dtau):
    """One SimplecStage::iterate (Simplec.cpp:452-506); returns (status, IterInfo, R).
    With the closure the iteration's nu_t becomes the case's history
    (Closure::accept)."""
    from ablsteadyrans_b200.abi import IterInfo
    _history(case)
    R = [case.grid.np_zeros() for _ in range(6)]
    arr = (ctypes.c_void_p * 6)(*[r.ctypes.data for r in R])
    info = IterInfo()
    st, m, d = case.state(), case.mesh(), case.diffusivities()
    if phys.closure and case.cf is None:
        case.cf = [case.grid.np_zeros() for _ in CLOSURE_FIELDS]
    rc = _L().og_simplec_iterate2(ctypes.byref(case.grid.c), ctypes.byref(bc), ctypes.byref(phys), ctypes.byref(opts),
                                  ctypes.byref(st), ctypes.byref(m), ctypes.byref(d), _p(dtau), arr,
                                  ctypes.byref(info), None if case.cf is None else _arrays(case.cf), None)
    if phys.closure:
        case.closure_nu = case.cf[0]
        case.nut_hist = case.cf[3].copy()
    return int(rc), info, R


def stage_steps(case, bc, phys, opts, dtau):
    """The predictor, the pressure correction and the scalar sweeps of one
    SimplecStage::iterate (Simplec.cpp:452-506) taken one at a time
    (og_stage_steps) on the case's state, which ends as the iteration leaves
    it without theta's convection update. Returns a dict: status, R (the
    residual at the start), ap and d (the predictor's), the snapshots u, v, w
    after the predictor ("pred") and u, v, w, p after the correction ("pc"),
    and the infos: pred (max |du|, |dv|, |dw|, last sweeps), pc (divergence
    before, after, max |dp|, max |du|, |dv|, |dw|, removed mean, Poisson
    iterations), scalar (max |dtheta|, its last sweep, max |dk|, its last
    sweep, clipped)."""
    _history(case)
    g = case.grid
    R = [g.np_zeros() for _ in range(6)]
    ap = [g.np_zeros() for _ in range(3)]
    dd = [g.np_zeros() for _ in range(3)]
    snap = [g.np_zeros() for _ in range(7)]
    pinfo, cinfo, sinfo = np.zeros(6), np.zeros(8), np.zeros(5)
    st, m, d = case.state(), case.mesh(), case.diffusivities()
    rc = _L().og_stage_steps(ctypes.byref(g.c), ctypes.byref(bc), ctypes.byref(phys), ctypes.byref(opts),
                             ctypes.byref(st), ctypes.byref(m), ctypes.byref(d), _p(dtau), _arrays(R), _arrays(ap),
                             _arrays(dd), _arrays(snap), _p(pinfo), _p(cinfo), _p(sinfo))
    return {"status": int(rc), "R": R, "ap": ap, "d": dd,
            "pred": dict(zip(("u", "v", "w"), snap[:3])), "pc": dict(zip(("u", "v", "w", "p"), snap[3:])),
            "pred_info": pinfo, "pc_info": cinfo, "scalar_info": sinfo}


def initialize(case, bc, init_opts):
    """gust::initialize_state with init.first_guess = profile
    (Source/Initializer.cpp:281-430) on the case's state; returns (status,
    [divergence before, after, Poisson iterations, final residual, O'Brien's
    top residual])."""
    info = np.zeros(5)
    case.nut_hist = None   # a new initial state has no nu_t history
    st, m = case.state(), case.mesh()
    rc = _L().og_initialize(ctypes.byref(case.grid.c), ctypes.byref(bc), ctypes.byref(init_opts), ctypes.byref(st),
                            ctypes.byref(m), _p(info))
    return int(rc), info


def obrien_omega(case):
    """obrien_omega (Source/Initializer.cpp:197-274) on the case's u, v:
    returns (Omega on the z-faces, max |E|)."""
    g = case.grid
    om = g.np_zeros()
    E = _L().og_obrien_omega(ctypes.byref(g.c), _p(case.q["u"]), _p(case.q["v"]), _p(case.z), _p(case.ax),
                             _p(case.ay), _p(case.az), _p(case.J), _p(om))
    return om, float(E)


def transport_fluxes(grid, u, v, w, z, ax, ay):
    F = [grid.np_zeros() for _ in range(3)]
    _L().og_transport_fluxes(ctypes.byref(grid.c), _p(u), _p(v), _p(w), _p(z), _p(ax), _p(ay), *[_p(f) for f in F])
    return F


def convection(grid, loc, q, F, J, limiter=0, eps=1e-5, bounded=False):
    out = grid.np_zeros()
    _L().og_convection(ctypes.byref(grid.c), loc, _p(q), *[_p(f) for f in F], _p(J), limiter, eps, int(bounded), _p(out))
    return out


def implicit_coefficients(grid, C, F, gamma, z, J, logz=False):
    A = grid.np_zeros(7)
    _L().og_implicit_coefficients(ctypes.byref(grid.c), C, *[_p(f) for f in F], _p(gamma), _p(z), _p(J), int(logz), _p(A))
    return A


def velocity_divergence(grid, u, v, w, z, ax, ay, az, J):
    d = grid.np_zeros()
    _L().og_velocity_divergence(ctypes.byref(grid.c), _p(u), _p(v), _p(w), _p(z), _p(ax), _p(ay), _p(az), _p(J), _p(d))
    return d


def omega_from_w(grid, u, v, w, z):
    """MassFlux.cpp omega_from_w on the valid z-faces."""
    om = grid.np_zeros()
    _L().og_omega_from_w(ctypes.byref(grid.c), _p(u), _p(v), _p(w), _p(z), _p(om), 0)
    return om
