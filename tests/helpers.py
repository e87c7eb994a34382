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
