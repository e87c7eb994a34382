"""Grid sequencing: the horizontal hierarchy (MeshHierarchy, SmoothSurface),
the prolongation (Transfer.cpp prolong_fields / prolong_state) in the oracle
and on the GPU, and the coarse-to-fine level loop (Sequencing.cpp), after
the reference's test_MeshHierarchy.cpp, test_Transfer.cpp and
test_Sequencing.cpp."""
import math

import numpy as np
import pytest

import oracle
from ablsteadyrans_b200 import abi, hierarchy, workloads
from ablsteadyrans_b200.grid import Grid
from helpers import case_from_instance, seam_sync

FIELDS = ("u", "v", "w", "p", "theta", "tke")
LOCS = {"u": 1, "v": 2, "w": 4, "p": 0, "theta": 0, "tke": 0}


def _bare_case(g):
    z = g.np_zeros()
    return oracle.Case(g, z, z, z, z, z, z, z, z)


def _pos(g, loc, i, d):
    nod = (loc >> d) & 1
    h = g.dx if d == 0 else g.dy
    return (i + (0.0 if nod else 0.5)) * h


# ------------------------------------------------------------- hierarchy ---

def test_ground_passes_are_pinned():
    expect = [[0, 0, 0, 0, 0], [0, 1, 3, 7, 15], [0, 2, 6, 14, 30], [0, 3, 9, 21, 45]]
    for p in range(4):
        for lev in range(5):
            assert hierarchy.ground_passes(lev, p) == expect[p][lev]


def _host_smooth(h, nx, ny, px, py, passes):
    """An independent rebuild of the smoothing: plain loops, the neighbour
    across a non-periodic face the edge node, the periodic images first."""
    h = h.copy()
    for _ in range(passes):
        old = h.copy()
        for j in range(ny + 1):
            for i in range(nx + 1):
                def at(ii, jj):
                    if px:
                        ii %= nx
                    else:
                        ii = min(max(ii, 0), nx)
                    if py:
                        jj %= ny
                    else:
                        jj = min(max(jj, 0), ny)
                    return old[jj + 1, ii + 1]
                s = at(i + 1, j) + at(i - 1, j)
                s = s + at(i, j + 1)
                s = s + at(i, j - 1)
                s = s - 4.0 * old[j + 1, i + 1]
                h[j + 1, i + 1] = old[j + 1, i + 1] + 0.125 * s
        # the periodic seam node n is node 0
        if px:
            h[:, nx + 1] = h[:, 1]
        if py:
            h[ny + 1, :] = h[1, :]
    return h


@pytest.mark.parametrize("passes", [0, 1, 2])
def test_coarse_grounds_are_the_smoothed_injection(passes):
    inst = workloads.config1(32, 16, 8, turbulence=False)
    levels = hierarchy.build(inst, 3, passes)
    assert levels[0].ground is inst.ground
    for lev in (1, 2):
        r = 1 << lev
        gc = levels[lev].grid
        n = hierarchy.ground_passes(lev, passes)
        inj = inst.ground[1:r * gc.ny + 2:r, 1:r * gc.nx + 2:r]
        h = np.zeros((gc.ny + 3, gc.nx + 3))
        h[1:-1, 1:-1] = inj
        ref = _host_smooth(h, gc.nx, gc.ny, gc.periodic_x, gc.periodic_y, n)
        got = levels[lev].ground[1:-1, 1:-1]
        assert np.abs(got - ref[1:-1, 1:-1]).max() < 1e-12 * 150
        if n > 0:
            fewer = _host_smooth(h, gc.nx, gc.ny, gc.periodic_x, gc.periodic_y, n - 1)
            assert np.abs(got - fewer[1:-1, 1:-1]).max() > 1e-3
        more = _host_smooth(h, gc.nx, gc.ny, gc.periodic_x, gc.periodic_y, n + 1)
        assert np.abs(got - more[1:-1, 1:-1]).max() > 1e-3


def test_constant_ground_is_unchanged_on_every_level():
    inst = workloads.config1(32, 16, 8, turbulence=False)
    inst.ground = np.full_like(inst.ground, 37.5)
    for lv in hierarchy.build(inst, 3, 3):
        assert np.array_equal(lv.ground, np.full_like(lv.ground, 37.5))


def test_z_levels_are_identical_on_every_level():
    inst = workloads.config1(32, 16, 8, turbulence=False)
    inst.ground = np.zeros_like(inst.ground)
    inst.z = workloads.btf_heights(inst.grid, inst.zlevels, inst.ground)
    G = inst.grid.ng
    col0 = inst.z[G:G + inst.grid.nz + 1, G, G]
    for lv in hierarchy.build(inst, 3, 1):
        g = lv.grid
        z = lv.inst.z
        assert np.array_equal(z[G:G + g.nz + 1, G + g.ny // 2, G + g.nx // 2], col0)
        assert g.dx == inst.grid.dx * (1 << lv.level) and g.nz == inst.grid.nz


def test_invalid_layouts_name_their_keys():
    assert hierarchy.check_hierarchy_inputs(32, 16, 3, 1) == []
    assert any("mesh.hierarchy_levels" in e for e in hierarchy.check_hierarchy_inputs(30, 16, 3, 1))
    assert any("mesh.hierarchy_levels" in e for e in hierarchy.check_hierarchy_inputs(32, 16, 0, 1))
    assert any("1 x 1 cells" in e for e in hierarchy.check_hierarchy_inputs(4, 4, 3, 1))
    assert any("terrain.hierarchy_passes" in e for e in hierarchy.check_hierarchy_inputs(32, 16, 2, 65))
    with pytest.raises(ValueError, match="mesh.hierarchy_levels"):
        hierarchy.build(workloads.config1(30, 16, 8, turbulence=False), 3)


def test_roughness_is_the_geometric_mean():
    inst = workloads.config2(n=16, nz=8, turbulence=True)
    lv = hierarchy.build(inst, 2, 1)[1]
    g0, gc = inst.grid, lv.grid
    G = g0.ng
    f = np.asarray(inst.z0map).reshape(g0.ny + 1 + 2 * G, g0.nx + 1 + 2 * G)[G:G + g0.ny, G:G + g0.nx]
    c = np.asarray(lv.z0map).reshape(gc.ny + 1 + 2 * G, gc.nx + 1 + 2 * G)[G:G + gc.ny, G:G + gc.nx]
    gm = np.exp(np.log(f).reshape(gc.ny, 2, gc.nx, 2).mean(axis=(1, 3)))
    assert np.allclose(c, gm, rtol=1e-13, atol=0)


# ---------------------------------------------------------- prolongation ---

@pytest.mark.parametrize("px", [False, True])
@pytest.mark.parametrize("r", [2, 4])
def test_prolongation_of_bilinear_fields_is_exact(px, r):
    """Fields bilinear per cell of the coarse points of their type (a tent in
    the periodic direction with its kinks on coarse points, linear in the
    other) come back exactly at the fine points; the coarse ghosts are not
    read (a large value would show)."""
    gf = Grid(16, 16, 3, 40.0, 30.0, 10.0, px, not px)
    gc = Grid(16 // r, 16 // r, 3, 40.0 * r, 30.0 * r, 10.0, px, not px)
    cc, cf = _bare_case(gc), _bare_case(gf)
    fns = {}
    for n, f in enumerate(FIELDS):
        loc = LOCS[f]
        pd = 0 if px else 1
        L = (gc.nx * gc.dx) if px else (gc.ny * gc.dy)
        D = gc.dx if px else gc.dy
        nod = (loc >> pd) & 1
        N = gc.nx if px else gc.ny
        ya = (N // 4 + (0.0 if nod else 0.5)) * D
        a, b, c_, e, gg = 1.0 + n, 0.01 * (n + 1), 0.02 - 0.003 * n, 1e-5 * (n + 2), 0.7 * n - 1

        def fn(x, y, k, a=a, b=b, c_=c_, e=e, gg=gg, ya=ya, L=L):
            s, t = (x, y) if px else (y, x)
            m = math.fmod(s - ya, L)
            if m < 0:
                m += L
            tent = abs(m - L / 2)
            return (a + b * t) * (1.0 + c_ * tent) + e * t * tent + gg * k
        fns[f] = fn
        arr = np.full(gc.shape, 1e30)
        for k in range(gc.nz + ((loc >> 2) & 1)):
            for j in range(gc.ny + ((loc >> 1) & 1)):
                for i in range(gc.nx + (loc & 1)):
                    arr[k + gc.ng, j + gc.ng, i + gc.ng] = fn(_pos(gc, loc, i, 0), _pos(gc, loc, j, 1), k)
        cc.q[f] = arr
        cf.q[f] = np.full(gf.shape, -1e30)
    oracle.prolong_fields(cc, cf, r)
    for f in FIELDS:
        loc = LOCS[f]
        err = scale = 0.0
        for k in range(gf.nz + ((loc >> 2) & 1)):
            for j in range(gf.ny + ((loc >> 1) & 1)):
                for i in range(gf.nx + (loc & 1)):
                    ex = fns[f](_pos(gf, loc, i, 0), _pos(gf, loc, j, 1), k)
                    err = max(err, abs(cf.q[f][k + gf.ng, j + gf.ng, i + gf.ng] - ex))
                    scale = max(scale, abs(ex))
        assert err < 1e-13 * scale, (f, r, px)


def _two_levels(hill, turbulence=False, nx=16, ny=16, nz=8, faces=None, surface=None):
    """A level-0 instance over a hill (or flat) and its level 1."""
    inst = workloads.config1(nx, ny, nz, turbulence=turbulence)
    if not hill:
        inst.ground = np.zeros_like(inst.ground)
        inst.z = workloads.btf_heights(inst.grid, inst.zlevels, inst.ground)
    if faces is not None:
        bc = abi.BC.make(faces, theta_ref=((0.0, 1500.0), (300.0, 300.0)), ustar=inst.ustar, z0=inst.z0,
                         direction=inst.direction, kappa=workloads.KAPPA, Cmu0=workloads.CMU0, l_max=workloads.LMAX,
                         surface=surface)
        inst.bc = bc
    lv = hierarchy.build(inst, 2, 1)
    return lv[0], lv[1]


def _smooth_state(case, seed):
    """A smooth state on a level: the inflow profile plus smooth waves."""
    g = case.grid
    rng = np.random.default_rng(seed)
    for f in FIELDS:
        loc = LOCS[f]
        v = g.valid(loc)
        shape = case.q[f][v].shape
        kk, jj, ii = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
        ph = rng.uniform(0, 2 * math.pi, 3)
        # periodic over the domain: the two copies of a periodic seam face agree
        wave = np.sin(2 * math.pi * ii / g.nx + ph[0]) * np.cos(2 * math.pi * jj / g.ny + ph[1])
        amp = {"u": 0.8, "v": 0.6, "w": 0.05, "p": 3.0, "theta": 0.3, "tke": 0.05}[f]
        case.q[f][v] = case.q[f][v] + amp * wave * (1 + 0.1 * np.cos(kk + ph[2]))
    case.q["tke"][g.valid(0)] = np.abs(case.q["tke"][g.valid(0)]) + 0.01
    for f in FIELDS:
        seam_sync(g, LOCS[f], case.q[f])


def test_prolonged_tke_is_above_the_floor():
    faces = (abi.FACE_PERIODIC, abi.FACE_SLIP_WALL, abi.FACE_SLIP_WALL, abi.FACE_PERIODIC, abi.FACE_SLIP_WALL,
             abi.FACE_SLIP_WALL)
    inst = workloads.config1(16, 16, 8, turbulence=False)
    inst.grid = Grid(16, 16, 8, inst.grid.dx, inst.grid.dy, inst.grid.dzeta, True, False)
    inst.ground = workloads.node_ground(inst.grid, lambda x, y: 40.0 * math.exp(-((x - 200) ** 2 + (y - 200) ** 2) / 150.0 ** 2))
    inst.z = workloads.btf_heights(inst.grid, inst.zlevels, inst.ground)
    inst.bc = abi.BC.make(faces, theta_ref=((0.0, 1500.0), (300.0, 300.0)))
    inst.physics = abi.Physics.make(1500.0)
    l0, l1 = hierarchy.build(inst, 2, 1)
    cc, cf = case_from_instance(l1.inst), case_from_instance(l0.inst)
    _smooth_state(cc, 3)
    g = cc.grid
    floor = 1e-4
    v = g.valid(0)
    kk, jj, ii = np.meshgrid(*[np.arange(s) for s in cc.q["tke"][v].shape], indexing="ij")
    x, y = (ii + 0.5) * g.dx, (jj + 0.5) * g.dy
    Lx, Ly = g.nx * g.dx, g.ny * g.dy
    cc.q["tke"][v] = 1e-4 * (0.6 + 1.2 * np.sin(2 * math.pi * x / Lx + 0.4 * kk) * np.cos(2 * math.pi * y / Ly))
    interp = case_from_instance(l0.inst)
    oracle.prolong_fields(cc, interp, 2)
    opts = abi.SimplecOptions.make(tke_floor=floor)
    st, info = oracle.prolong_state(cc, cf, 2, inst.bc, inst.physics, opts, reltol=1e-10)
    assert st == 0
    ki, kf = interp.q["tke"][cf.grid.valid(0)], cf.q["tke"][cf.grid.valid(0)]
    expect = np.where(ki < floor, floor, ki)
    assert kf.min() >= floor and np.array_equal(kf, expect)
    below = int((ki < floor).sum())
    assert ki.min() < 0 and below > 100
    assert int(info[3]) == below


@pytest.mark.parametrize("hill", [False, True])
def test_prolongation_and_projection_is_divergence_free(hill):
    """The divergence left is the Poisson solve's residual; the Dirichlet
    normal velocities keep their boundary values; p' is the interpolated one
    and theta is untouched (inflow / outflow in x, periodic y, the surface
    layer, a slip top)."""
    faces = (abi.FACE_INFLOW, abi.FACE_PERIODIC, abi.FACE_SURFACE_LAYER, abi.FACE_OUTFLOW, abi.FACE_PERIODIC,
             abi.FACE_SLIP_WALL)
    l0, l1 = _two_levels(hill, turbulence=True, faces=faces, surface={"z0": 0.03})
    cc, cf = case_from_instance(l1.inst), case_from_instance(l0.inst)
    _smooth_state(cc, 7)
    ref = case_from_instance(l0.inst)
    oracle.prolong_fields(cc, ref, 2)
    g = cf.grid
    v = g.valid(0)
    ref.q["tke"][v] = np.maximum(ref.q["tke"][v], 1e-6)
    oracle.fill_ghosts(ref, l0.inst.bc, l0.inst.physics)
    reltol = 1e-9
    opts = abi.SimplecOptions.make(tke_floor=1e-6)
    st, info = oracle.prolong_state(cc, cf, 2, l0.inst.bc, l0.inst.physics, opts, reltol=reltol)
    assert st == 0
    D0 = oracle.velocity_divergence(g, ref.q["u"], ref.q["v"], ref.q["w"], cf.z, cf.ax, cf.ay, cf.az, cf.J)
    D1 = oracle.velocity_divergence(g, cf.q["u"], cf.q["v"], cf.q["w"], cf.z, cf.ax, cf.ay, cf.az, cf.J)
    # the Poisson solve stops on the plain 2-norm of its residual, which is
    # the divergence left (the reference's gmres_fft back end does the same)
    n0 = np.sqrt((D0[v] ** 2).sum())
    n1 = np.sqrt((D1[v] ** 2).sum())
    assert info[0] > 1e-4 and n0 > 1e-3
    assert n1 < 1.01 * reltol * n0
    assert info[1] == np.abs(D1[v]).max()
    G = g.ng
    u, ur = cf.q["u"], ref.q["u"]
    assert np.abs(u[G:G + g.nz, G:G + g.ny, G] - ur[G:G + g.nz, G:G + g.ny, G]).max() == 0.0   # inflow face
    assert np.abs(u[G:G + g.nz, G:G + g.ny, G + 1:G + g.nx] - ur[G:G + g.nz, G:G + g.ny, G + 1:G + g.nx]).max() > 1e-3
    om = oracle.omega_from_w(g, cf.q["u"], cf.q["v"], cf.q["w"], cf.z)
    assert max(np.abs(om[G, G:G + g.ny, G:G + g.nx]).max(),
               np.abs(om[G + g.nz, G:G + g.ny, G:G + g.nx]).max()) < 1e-12 * np.abs(u[g.valid(1)]).max()
    assert np.array_equal(cf.q["p"], ref.q["p"])
    assert np.array_equal(cf.q["theta"][v], ref.q["theta"][v])


# ------------------------------------------------------------ restriction ---

def _three_levels(hill):
    faces = (abi.FACE_INFLOW, abi.FACE_PERIODIC, abi.FACE_SLIP_WALL, abi.FACE_OUTFLOW, abi.FACE_PERIODIC,
             abi.FACE_SLIP_WALL)
    inst = workloads.config1(16, 16, 6, turbulence=False)
    if not hill:
        inst.ground = np.zeros_like(inst.ground)
    else:
        inst.ground = workloads.node_ground(inst.grid, lambda x, y: 90.0 * math.exp(-((x - 200) ** 2 + (y - 210) ** 2) / 120.0 ** 2))
    inst.z = workloads.btf_heights(inst.grid, inst.zlevels, inst.ground)
    inst.bc = abi.BC.make(faces, theta_ref=((0.0, 1500.0), (300.0, 300.0)), ustar=inst.ustar, z0=inst.z0)
    inst.physics = abi.Physics.make(1500.0)
    return inst, hierarchy.build(inst, 3, 1)


@pytest.mark.parametrize("hill", [False, True])
def test_restriction_conserves_face_flux(hill):
    """Each coarse face carries the sum of its fine faces' fluxes, each coarse
    cell the detJ-weighted mean of its fine cells, and r^2 J_c D_c = sum J_f
    D_f for the divergence (Transfer.RestrictionConservesFaceFlux)."""
    inst, levels = _three_levels(hill)
    for lf, lc in ((0, 1), (1, 2), (0, 2)):
        r = 1 << (lc - lf)
        cf, cc = case_from_instance(levels[lf].inst), case_from_instance(levels[lc].inst)
        _smooth_state(cf, 20 + lf + lc)
        oracle.fill_ghosts(cf, inst.bc, inst.physics)
        om_c = oracle.restrict_state(cf, cc, r)
        gf, gc = cf.grid, cc.grid
        G = gf.ng
        F = lambda a, i, j, k: a[k + G, j + G, i + G]        # noqa: E731
        om_f = oracle.omega_from_w(gf, cf.q["u"], cf.q["v"], cf.q["w"], cf.z)
        ex = sx = ey = ez = sz = 0.0
        areas_differ = False
        for k in range(gc.nz):
            for J in range(gc.ny):
                for I in range(gc.nx + 1):
                    s = sum(F(cf.ax, r * I, r * J + b, k) * F(cf.q["u"], r * I, r * J + b, k) for b in range(r))
                    sa = sum(F(cf.ax, r * I, r * J + b, k) for b in range(r))
                    ex = max(ex, abs(F(cc.ax, I, J, k) * F(cc.q["u"], I, J, k) * r - s))
                    sx = max(sx, abs(s))
                    areas_differ |= abs(sa - r * F(cc.ax, I, J, k)) > 1e-3 * sa
            for J in range(gc.ny + 1):
                for I in range(gc.nx):
                    s = sum(F(cf.ay, r * I + a, r * J, k) * F(cf.q["v"], r * I + a, r * J, k) for a in range(r))
                    ey = max(ey, abs(F(cc.ay, I, J, k) * F(cc.q["v"], I, J, k) * r - s))
        for k in range(gc.nz + 1):
            for J in range(gc.ny):
                for I in range(gc.nx):
                    s = sum(F(cf.az, r * I + a, r * J + b, k) * F(om_f, r * I + a, r * J + b, k)
                            for b in range(r) for a in range(r))
                    ez = max(ez, abs(F(cc.az, I, J, k) * F(om_c, I, J, k) * r * r - s))
                    sz = max(sz, abs(s))
        assert ex < 1e-12 * sx and ey < 1e-12 * sx and ez < 1e-12 * sz
        assert sz > 1e-3 * sx
        assert areas_differ == hill
        v = gc.valid(0)
        Jf = cf.J[gf.valid(0)].reshape(gc.nz, gc.ny, r, gc.nx, r)
        for f in ("theta", "tke", "p"):
            qf = cf.q[f][gf.valid(0)].reshape(gc.nz, gc.ny, r, gc.nx, r)
            mean = (Jf * qf).sum(axis=(2, 4)) / Jf.sum(axis=(2, 4))
            assert np.abs(cc.q[f][v] - mean).max() < 4e-15 * np.abs(mean).max() * 10
        Df = oracle.velocity_divergence(gf, cf.q["u"], cf.q["v"], cf.q["w"], cf.z, cf.ax, cf.ay, cf.az, cf.J)
        Dc = oracle.face_divergence(gc, cc.ax, cc.ay, cc.az, cc.J, cc.q["u"], cc.q["v"], om_c)
        sJD = (cf.J * Df)[gf.valid(0)].reshape(gc.nz, gc.ny, r, gc.nx, r).sum(axis=(2, 4))
        ed = np.abs(r * r * cc.J[v] * Dc[v] - sJD).max()
        dscale = sx / gc.dx * r
        assert ed < 1e-12 * dscale and np.abs(sJD).max() > 1e-3 * dscale


def _smooth1(c, I, N, periodic):
    if not periodic and (I == 0 or I == N - 1):
        return c(I)
    im = (I - 1 + N) % N if periodic else I - 1
    ip = (I + 1) % N if periodic else I + 1
    return (c(im) + 6 * c(I) + c(ip)) / 8


@pytest.mark.parametrize("px", [False, True])
def test_round_trip_is_the_closed_form_smoother(px):
    """restrict(prolong(c)) on flat ground for r = 2 is S_x S_y with
    (S c)_I = (c_{I-1} + 6 c_I + c_{I+1}) / 8 in the interior and across a
    periodic seam, c_I next to a non-periodic face, and 1 along a nodal
    direction (Transfer.RoundTripIsTheClosedFormSmoother)."""
    faces = (abi.FACE_PERIODIC if px else abi.FACE_INFLOW, abi.FACE_INFLOW if px else abi.FACE_PERIODIC,
             abi.FACE_SLIP_WALL, abi.FACE_PERIODIC if px else abi.FACE_OUTFLOW,
             abi.FACE_OUTFLOW if px else abi.FACE_PERIODIC, abi.FACE_SLIP_WALL)
    inst = workloads.config1(16, 16, 4, turbulence=False)
    inst.grid = Grid(16, 16, 4, inst.grid.dx, inst.grid.dy, inst.grid.dzeta, px, not px)
    inst.ground = np.zeros((19, 19))
    inst.z = workloads.btf_heights(inst.grid, inst.zlevels[:5] if len(inst.zlevels) > 5 else inst.zlevels, inst.ground)
    inst.bc = abi.BC.make(faces, theta_ref=((0.0, 1500.0), (300.0, 300.0)))
    l0, l1 = hierarchy.build(inst, 2, 1)
    cc, cf, back = case_from_instance(l1.inst), case_from_instance(l0.inst), case_from_instance(l1.inst)
    g = cc.grid
    rng = np.random.default_rng(5)
    for f in FIELDS:
        v = g.valid(LOCS[f])
        cc.q[f][v] = 1.0 + 1e-5 * rng.standard_normal(cc.q[f][v].shape)
        seam_sync(g, LOCS[f], cc.q[f])
    oracle.prolong_fields(cc, cf, 2)
    for f in ("u", "v"):
        seam_sync(cf.grid, LOCS[f], cf.q[f])
        oracle.fill_periodic(cf.grid, LOCS[f], cf.q[f])
    oracle.restrict_state(cf, back, 2)
    G = g.ng
    for f in FIELDS:
        loc = LOCS[f]
        nx_, ny_ = (loc & 1) == 1, (loc & 2) == 2
        hc = cc.q[f]
        err = change = scale = 0.0
        for k in range(g.nz + ((loc >> 2) & 1)):
            for J in range(g.ny + ny_):
                for I in range(g.nx + nx_):
                    def sx(jj):
                        if nx_:
                            return hc[k + G, jj + G, I + G]
                        return _smooth1(lambda ii: hc[k + G, jj + G, ii + G], I, g.nx, px)
                    ex = sx(J) if ny_ else _smooth1(sx, J, g.ny, not px)
                    err = max(err, abs(back.q[f][k + G, J + G, I + G] - ex))
                    change = max(change, abs(ex - hc[k + G, J + G, I + G]))
                    scale = max(scale, abs(ex))
        assert err < 2e-14 * scale, (f, err)
        assert change > 1e-7, f


# ------------------------------------------------------------------ GPU ---

@pytest.mark.gpu
@pytest.mark.parametrize("hill", [False, True])
def test_gpu_prolong_matches_oracle(ctx, hill):
    """gb_simplec_prolong against the oracle's prolong_state: every field,
    the divergences and the clipped count (the surface layer, the closure)."""
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    faces = (abi.FACE_INFLOW, abi.FACE_PERIODIC, abi.FACE_SURFACE_LAYER, abi.FACE_OUTFLOW, abi.FACE_PERIODIC,
             abi.FACE_SLIP_WALL)
    l0, l1 = _two_levels(hill, turbulence=True, faces=faces, surface={"z0": 0.03})
    cc, cf = case_from_instance(l1.inst), case_from_instance(l0.inst)
    _smooth_state(cc, 11)
    cc.q["tke"][cc.grid.valid(0)] -= 0.02     # some cells below the floor
    reltol = 1e-11
    opts = abi.SimplecOptions.make(tke_floor=1e-3, pressure_reltol=reltol)
    dcc = DeviceCase.from_oracle(cc)
    dcf = DeviceCase.from_oracle(cf)
    stage = SimplecStage(ctx, dcf, l0.inst.bc, l0.inst.physics, opts)
    try:
        res = stage.prolong(dcc, reltol)
        st, info = oracle.prolong_state(cc, cf, 2, l0.inst.bc, l0.inst.physics, opts, reltol=reltol)
        assert st == 0
        assert res.tke_clipped == int(info[3]) and res.tke_clipped > 0
        assert abs(res.divergence_before - info[0]) <= 1e-10 * info[0]
        assert res.divergence_after <= 10 * max(info[1], 1e-12 * info[0])
        for f in FIELDS:
            vv = cf.grid.valid(LOCS[f])
            ref, got = cf.q[f][vv], dcf.host(f)[vv]
            assert np.abs(got - ref).max() <= 1e-8 * max(np.abs(ref).max(), 1e-300), f
    finally:
        stage.close()


@pytest.mark.gpu
def test_gpu_sequencing_runs_coarse_to_fine(ctx):
    """Three levels of a 32 x 32 x 16 hill with the closure and the surface
    layer: the coarse levels stop loosely (or at their iteration cap), each
    prolongation's projection leaves a small divergence, level 0's driver
    starts from the coarsest level's references and its first iterations
    are finite."""
    import torch

    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.sequencing import sequence_coarse_levels, sequencing_report
    from ablsteadyrans_b200.simplec import DeviceCase, NativeDriver, SimplecStage
    inst = workloads.config1(32, 32, 16, turbulence=True)
    inst.options.pressure_reltol = 1e-3
    g = inst.grid
    z = torch.from_numpy(inst.z).cuda()
    J, ax, ay, az, _ = gb.mesh_metrics(ctx, g, z)
    case = DeviceCase(g, z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
    stage = SimplecStage(ctx, case, inst.bc, inst.physics, inst.options)
    driver = NativeDriver(stage)
    seq = abi.SequencingOptions.make(enabled=1)
    try:
        levels = sequence_coarse_levels(ctx, inst, 3, seq, stage, driver, max_iterations=300)
        assert [s.level for s in levels] == [2, 1, 0]
        for s in levels[:-1]:
            assert s.iterations > 0 and s.stop, s
        for s in levels[1:]:
            assert s.prolonged and s.prolong.divergence_after < 1e-2 * s.prolong.divergence_before + 1e-12
        h = driver.criterion.history()
        assert h["count"] == 0 and h["res_ref"][:6] == pytest.approx(levels[0].res_ref, rel=0, abs=0)
        assert driver.status()[0] == 0      # the hold released
        for _ in range(5):
            verdict, info, _ = driver.step()
            assert verdict == "running" and all(math.isfinite(x) for x in info.residual_norms)
        print(sequencing_report(levels, 5, "not steady"))
    finally:
        driver.close()
        stage.close()


@pytest.mark.gpu
@pytest.mark.parametrize("hill", [False, True])
def test_gpu_restrict_matches_oracle(ctx, hill):
    """gb_restrict_state against the oracle's restrict_state, every field and
    the coarse Omega."""
    import ablsteadyrans_b200 as gb
    from ablsteadyrans_b200.simplec import DeviceCase
    inst, levels = _three_levels(hill)
    for lf, lc in ((0, 1), (0, 2)):
        cf, cc = case_from_instance(levels[lf].inst), case_from_instance(levels[lc].inst)
        _smooth_state(cf, 30 + lc)
        oracle.fill_ghosts(cf, inst.bc, inst.physics)
        dcf, dcc = DeviceCase.from_oracle(cf), DeviceCase.from_oracle(cc)
        om = gb.restrict_state(ctx, dcf, dcc).cpu().numpy()
        om_ref = oracle.restrict_state(cf, cc, 1 << (lc - lf))
        gc = cc.grid
        for f in FIELDS:
            v = gc.valid(LOCS[f])
            ref, got = cc.q[f][v], dcc.host(f)[v]
            assert np.abs(got - ref).max() <= 1e-13 * max(np.abs(ref).max(), 1e-300), (f, lf, lc)
        v = gc.valid(4)
        assert np.abs(om[v] - om_ref[v]).max() <= 1e-13 * np.abs(om_ref[v]).max()
