"""Shared test helpers: seeded random systems and fields in the grid layout,
dense reference solves, and host/device copies."""
import numpy as np

from ablsteadyrans_b200.grid import Grid, N_COEFS, LOC_CELL, LOC_XFACE, LOC_YFACE, LOC_ZFACE  # noqa: F401

LOCS = (LOC_CELL, LOC_XFACE, LOC_YFACE, LOC_ZFACE)
COEF_P, COEF_XM, COEF_XP, COEF_YM, COEF_YP, COEF_ZM, COEF_ZP = range(7)


def seam_sync(grid, loc, f):
    """OverrideSync on a host array: the high seam copy takes the low one."""
    g = grid.ng
    ni, nj, nk = grid.extents(loc)
    if (loc & 1) and grid.periodic_x:
        f[..., g:g + nk, g:g + nj, g + grid.nx] = f[..., g:g + nk, g:g + nj, g]
    if (loc & 2) and grid.periodic_y:
        f[..., g:g + nk, g + grid.ny, g:g + ni] = f[..., g:g + nk, g, g:g + ni]


def random_system(grid, loc, seed, extra=0.5, xscale=1.0):
    """A random M-matrix system at loc (after test_LineSweeps.cpp:76-110): the
    six neighbour coefficients in [0.1, 1] (x ones scaled by xscale), the
    diagonal their sum plus extra, a random right-hand side in [-1, 1]; the
    copies of a periodic seam carry one system."""
    rng = np.random.default_rng(seed)
    A = grid.np_zeros(N_COEFS)
    ap = grid.np_zeros()
    rhs = grid.np_zeros()
    v = grid.valid(loc)
    shape = A[(0,) + v].shape
    total = np.zeros(shape)
    for n in range(1, N_COEFS):
        c = rng.uniform(0.1, 1.0, size=shape)
        if n in (COEF_XM, COEF_XP):
            c *= xscale
        A[(n,) + v] = c
        total += c
    A[(COEF_P,) + v] = total
    ap[v] = total + extra
    rhs[v] = rng.uniform(-1.0, 1.0, size=shape)
    seam_sync(grid, loc, A)
    seam_sync(grid, loc, ap)
    seam_sync(grid, loc, rhs)
    return A, ap, rhs


def dense_line_system_solve(grid, loc, A, ap, rhs):
    """Direct solve of ap x - sum a_nb x_nb = rhs over the valid points of loc,
    with periodic images for the lateral neighbours and zero outside a
    non-periodic face (the system the z-line Jacobi sweeps converge to)."""
    ni, nj, nk = grid.extents(loc)
    n = ni * nj * nk
    idx = lambda i, j, k: (k * nj + j) * ni + i  # noqa: E731
    M = np.zeros((n, n))
    b = np.zeros(n)
    g = grid.ng

    def image(i, nv, nc, per):
        if 0 <= i < nv:
            return i
        if not per:
            return None
        return i + nc if i < 0 else i - nc

    for k in range(nk):
        for j in range(nj):
            for i in range(ni):
                r = idx(i, j, k)
                M[r, r] = ap[k + g, j + g, i + g]
                b[r] = rhs[k + g, j + g, i + g]
                for comp, (di, dj, dk) in ((COEF_XM, (-1, 0, 0)), (COEF_XP, (1, 0, 0)), (COEF_YM, (0, -1, 0)),
                                           (COEF_YP, (0, 1, 0)), (COEF_ZM, (0, 0, -1)), (COEF_ZP, (0, 0, 1))):
                    ii = image(i + di, ni, grid.nx, grid.periodic_x)
                    jj = image(j + dj, nj, grid.ny, grid.periodic_y)
                    kk = k + dk
                    if ii is None or jj is None or kk < 0 or kk >= nk:
                        continue
                    M[r, idx(ii, jj, kk)] -= A[comp, k + g, j + g, i + g]
    x = np.linalg.solve(M, b)
    out = grid.np_zeros()
    out[grid.valid(loc)] = x.reshape(nk, nj, ni)
    return out


def to_dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    if dtype is not None:
        t = t.to(dtype)
    return t


def to_host(t):
    return t.detach().double().cpu().numpy()


def rel_err(a, b, v=None):
    if v is not None:
        a, b = a[v], b[v]
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


# ------------------------------------------------------------------ Poisson
GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)), "golden")
PERIODIC, NEUMANN, DIRICHLET = 0, 1, 2


def askervein_case():
    """The reference's Poisson_Askervein projection (Tests/Supporting_Files/Tools/
    poisson_projection.cpp): BTF mesh on ERF's Askervein terrain (fixture), the
    fixed wind u = 8 (1 + 0.2 sin(2 pi y/Ly)), v = 2.4 cos(2 pi x/Lx) (0 on the y
    walls), w = 0; x low Neumann, x high Dirichlet, y Neumann, ground Neumann,
    top Dirichlet."""
    import oracle
    d = np.load(__import__("os").path.join(GOLDEN, "poisson_askervein.npz"))
    nx, ny, nz = 30, 30, 18
    plo, phi_hi = d["prob_lo"], d["prob_hi"]
    g = Grid(nx, ny, nz, (phi_hi[0] - plo[0]) / nx, (phi_hi[1] - plo[1]) / ny, (phi_hi[2] - plo[2]) / nz)
    z = oracle.btf_heights(g, d["zlevels"], d["ground"])
    J, ax, ay, az, zcc = oracle.metrics(g, z)
    Lx, Ly = phi_hi[0] - plo[0], phi_hi[1] - plo[1]
    U = [g.np_zeros() for _ in range(3)]
    G = g.ng
    for k in range(nz):
        for j in range(ny):
            y = plo[1] + (j + 0.5) * g.dy
            U[0][k + G, j + G, G:G + nx + 1] = 8.0 * (1 + 0.2 * np.sin(2 * np.pi * (y - plo[1]) / Ly))
        for j in range(ny + 1):
            x = plo[0] + (np.arange(nx) + 0.5) * g.dx
            wall = (j == 0) or (j == ny)
            U[1][k + G, j + G, G:G + nx] = 0.0 if wall else 2.4 * np.cos(2 * np.pi * (x - plo[0]) / Lx)
    bc = (NEUMANN, NEUMANN, NEUMANN, DIRICHLET, NEUMANN, DIRICHLET)
    return dict(grid=g, z=z, J=J, ax=ax, ay=ay, az=az, U=U, bc=bc, phi_gold=d["phi"],
                info=__import__("json").loads(str(d["info"])))


def init_askervein_case():
    """The reference's Mass_Consistent_Askervein regression (Tests/Initialization/
    Mass_Consistent_Askervein/inputs_init_askervein) on the Poisson_Askervein
    mesh: log-law first guess along x (u* 0.6 m/s, z0 0.03 m, kappa 0.41,
    Cmu0 0.5562, l_max 30 m), inflow at xlo, outflow at xhi, slip walls in y
    and at the top; the ground (surface_layer there) is a wall; theta 300 K;
    alpha_h 1, alpha_v 0.5, reltol 1e-10. Returns (case, bc, init options, gold)
    with gold's cell fields [k, j, i] and its info."""
    import json
    import os
    import oracle
    from ablsteadyrans_b200.abi import BC, InitOptions
    d = np.load(os.path.join(GOLDEN, "poisson_askervein.npz"))
    gd = np.load(os.path.join(GOLDEN, "init_askervein.npz"))
    nx, ny, nz = 30, 30, 18
    plo, phi_hi = d["prob_lo"], d["prob_hi"]
    g = Grid(nx, ny, nz, (phi_hi[0] - plo[0]) / nx, (phi_hi[1] - plo[1]) / ny, (phi_hi[2] - plo[2]) / nz)
    z = oracle.btf_heights(g, d["zlevels"], d["ground"])
    J, ax, ay, az, _ = oracle.metrics(g, z)
    nu = np.ones_like(J)
    case = oracle.Case(g, z, J, ax, ay, az, nu, nu, nu)
    bc = BC.make((1, 3, 4, 2, 3, 3), theta_ref=((0.0,), (300.0,)), ustar=0.6, z0=0.03, kappa=0.41, Cmu0=0.5562,
                 l_max=30.0)
    io = InitOptions.make(alpha_h=1.0, alpha_v=0.5)
    io.poisson.reltol = 1e-10
    gold = {f: gd[f] for f in ("u", "v", "w", "p", "theta", "tke")}
    gold["info"] = json.loads(str(gd["info"]))
    return case, bc, io, gold


def closure_column_case(ustar=0.35, z0=0.1, direction=15.0):
    """The reference's Closure_Column regression (Tests/Discretization/
    Closure_Column/inputs_closure_column, Tests/Supporting_Files/Tools/
    closure_column.cpp): ERF's Neutral_ABL_Flat mesh (8 x 8 x 64 cells over
    2560 m x 2560 m x 1000 m, flat, periodic sides), a surface_layer ground
    (z0 0.1 m), a slip top, theta 300 K, the wall law's equilibrium state
    u = (u*/kappa) ln((h + z0)/z0) along the direction at each point's height
    above the ground, k = u*^2/Cmu0^2, w = p' = 0; the k-L closure with
    turb.max_geom_lscale = 1e12 and the logarithmic face mean.
    Returns (case, bc, physics)."""
    import math
    import oracle
    from ablsteadyrans_b200.abi import BC, FACE_SLIP_WALL, FACE_SURFACE_LAYER, Physics
    nx, ny, nz = 8, 8, 64
    g = Grid(nx, ny, nz, 320.0, 320.0, 1000.0 / nz, True, True)
    z = oracle.btf_heights(g, np.arange(nz + 1) * (1000.0 / nz), np.zeros((ny + 3, nx + 3)))
    J, ax, ay, az, _ = oracle.metrics(g, z)
    case = oracle.Case(g, z, J, ax, ay, az, np.zeros_like(J), np.zeros_like(J), np.zeros_like(J))
    kappa, cmu0 = 0.41, 0.5562
    a = math.radians(direction)
    G = g.ng

    def height(t, i, j, k):
        nxp, nyp, nzp = (1 if t & 1 else 2), (1 if t & 2 else 2), (1 if t & 4 else 2)
        zp = zg = 0.0
        for aa in range(nxp):
            for b in range(nyp):
                zg += z[G, G + j + b, G + i + aa]
                for c in range(nzp):
                    zp += z[G + k + c, G + j + b, G + i + aa]
        return zp / (nxp * nyp * nzp) - zg / (nxp * nyp)

    def speed(h):
        return ustar / kappa * math.log((max(h, 0.0) + z0) / z0)

    q = case.q
    for k in range(nz):
        for j in range(ny):
            for i in range(nx + 1):
                q["u"][G + k, G + j, G + i] = speed(height(1, i, j, k)) * math.cos(a)
        for j in range(ny + 1):
            for i in range(nx):
                q["v"][G + k, G + j, G + i] = speed(height(2, i, j, k)) * math.sin(a)
    q["theta"][G:G + nz, G:G + ny, G:G + nx] = 300.0
    q["tke"][...] = ustar * ustar / (cmu0 * cmu0)
    bc = BC.make((0, 0, FACE_SURFACE_LAYER, 0, 0, FACE_SLIP_WALL), theta_ref=((0.0,), (300.0,)), ustar=ustar, z0=z0,
                 surface={"z0": z0})
    ph = Physics.make(1000.0, closure=1, turb_max_geom_lscale=1e12, log_mean=1)
    return case, bc, ph


def closure_column_outputs(g, q, R, cf, ss):
    """closure_column.cpp's plotfile fields [k, j, i]: cell means of the face
    values, the cell fields, and u* on the ground cells."""
    G, nx, ny, nz = g.ng, g.nx, g.ny, g.nz
    c = (slice(G, G + nz), slice(G, G + ny), slice(G, G + nx))
    out = {
        "u": 0.5 * (q["u"][c] + q["u"][G:G + nz, G:G + ny, G + 1:G + nx + 1]),
        "tke": q["tke"][c], "nut": cf["nut"][c], "length": cf["length"][c],
        "R_u": 0.5 * (R[0][c] + R[0][G:G + nz, G:G + ny, G + 1:G + nx + 1]),
        "R_v": 0.5 * (R[1][c] + R[1][G:G + nz, G + 1:G + ny + 1, G:G + nx]),
        "R_w": 0.5 * (R[2][c] + R[2][G + 1:G + nz + 1, G:G + ny, G:G + nx]),
        "R_theta": R[4][c], "R_tke": R[5][c], "Ps": cf["Ps"][c], "eps": cf["eps"][c],
    }
    ust = np.zeros((nz, ny, nx))
    ust[0] = np.asarray(ss["ustar"]).reshape(-1, int(g.c.sy))[G:G + ny, G:G + nx]
    out["ustar"] = ust
    return out


def gold_cell_fields(g, q):
    """The reference plotfile's cell values (Source/StateIO.cpp:59-74): u, v, w
    the means of the cell's two faces, the cell fields as they are; [k, j, i]."""
    G, nx, ny, nz = g.ng, g.nx, g.ny, g.nz
    c = (slice(G, G + nz), slice(G, G + ny), slice(G, G + nx))
    out = {
        "u": 0.5 * (q["u"][c] + q["u"][G:G + nz, G:G + ny, G + 1:G + nx + 1]),
        "v": 0.5 * (q["v"][c] + q["v"][G:G + nz, G + 1:G + ny + 1, G:G + nx]),
        "w": 0.5 * (q["w"][c] + q["w"][G + 1:G + nz + 1, G:G + ny, G:G + nx]),
    }
    for f in ("p", "theta", "tke"):
        out[f] = q[f][c]
    return out


def smooth_terrain_case(nx, ny, nz, periodic_x, periodic_y, hill=80.0, dx=40.0, seed=0):
    """A BTF mesh over a smooth Gaussian hill (periodic images or clamped
    ghost columns as the reference builds them), stretched layers to 1500 m."""
    import oracle
    g = Grid(nx, ny, nz, dx, dx, 1500.0 / nz, periodic_x, periodic_y)
    r = 1500.0 ** (1.0 / nz)
    zl = np.concatenate([[0.0], np.cumsum(2.0 * 1.06 ** np.arange(nz))])
    zl = zl * (1500.0 / zl[-1])
    ground = np.zeros((ny + 3, nx + 3))
    cx, cy = nx * dx / 2, ny * dx / 2
    for j in range(-1, ny + 2):
        for i in range(-1, nx + 2):
            ii = (i % nx) if periodic_x else min(max(i, 0), nx)
            jj = (j % ny) if periodic_y else min(max(j, 0), ny)
            x, y = ii * dx - cx, jj * dx - cy
            ground[j + 1, i + 1] = hill * np.exp(-(x * x + y * y) / (0.2 * (nx * dx) ** 2))
    z = oracle.btf_heights(g, zl, ground)
    J, ax, ay, az, zcc = oracle.metrics(g, z)
    return g, z, J, ax, ay, az, zcc


# ------------------------------------------------------------------ SIMPLEC
def flat_case(nx, ny, nz, Lx, Ly, H, periodic_x, periodic_y, visc):
    """A flat mesh with uniform layers (test_Simplec.cpp:45-58 flat_case) and
    uniform diffusivities (the Laminar fixture, :129-160)."""
    import oracle
    g = Grid(nx, ny, nz, Lx / nx, Ly / ny, H / nz, periodic_x, periodic_y)
    zl = np.arange(nz + 1) * (H / nz)
    ground = np.zeros((ny + 3, nx + 3))
    z = oracle.btf_heights(g, zl, ground)
    J, ax, ay, az, zcc = oracle.metrics(g, z)
    nu = g.np_zeros() + visc
    case = oracle.Case(g, z, J, ax, ay, az, nu, nu.copy(), nu.copy())
    return case


def terrain_simplec_case(nx, ny, nz, periodic_x, periodic_y, hill=60.0, dx=40.0, seed=0, visc=(5.0, 20.0)):
    """An oracle.Case over a BTF Gaussian hill with diffusivities that vary in
    height and a smooth seeded state (a shear profile plus small random
    perturbations; seam copies made one unknown)."""
    import oracle
    g, z, J, ax, ay, az, zcc = smooth_terrain_case(nx, ny, nz, periodic_x, periodic_y, hill=hill, dx=dx, seed=seed)
    zc = zcc.copy()
    nu = visc[0] + (visc[1] - visc[0]) * np.clip(zc / 1500.0, 0, 1)
    case = oracle.Case(g, z, J, ax, ay, az, nu, 1.3 * nu, 2.0 * nu)
    rng = np.random.default_rng(seed + 17)
    hfac = np.log1p(np.maximum(zc, 0.0) / 0.1)
    for f, loc, amp, base in (("u", 1, 0.3, 8.0), ("v", 2, 0.3, -1.5), ("w", 4, 0.05, 0.0), ("p", 0, 2.0, 0.0),
                              ("theta", 0, 0.5, 300.0), ("tke", 0, 0.05, 0.3)):
        v = g.valid(loc)
        shape = case.q[f][v].shape
        prof = hfac[g.valid(0)].mean(axis=(1, 2))
        nk = shape[0]
        col = np.interp(np.arange(nk), np.arange(len(prof)), prof)[:, None, None] / max(prof.max(), 1e-9)
        val = base * (col if f in ("u", "v") else 1.0) + amp * rng.standard_normal(shape)
        if f == "theta":
            val = base + 0.003 * np.arange(nk)[:, None, None] * 40 + amp * rng.standard_normal(shape)
        if f == "tke":
            val = np.abs(val) + 0.01
        case.q[f][v] = val
        seam_sync(g, loc, case.q[f])
    return case


def case_from_instance(inst):
    """An oracle.Case of a workloads.Instance: its node heights and metrics,
    diffusivities, initial state and roughness map."""
    import oracle
    g = inst.grid
    J, ax, ay, az, _ = oracle.metrics(g, inst.z)
    case = oracle.Case(g, inst.z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke,
                       None if inst.z0map is None else np.array(inst.z0map, dtype=np.float64))
    case.q = {f: a.copy() for f, a in inst.q.items()}
    return case
