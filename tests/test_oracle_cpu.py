"""CPU checks of the oracle (the C restatement of the reference's path).

The reference ships no tests, fixtures or golden outputs; what pins the
restatement here is
* the reference's own test_mg right-hand side (CORE_POISSON.F90:565-674)
  with its closed-form all-Neumann solution: second-order convergence of
  the solve under grid refinement;
* manufactured discrete solutions: f = A phi for the reference operator
  with ghost and dead rows, so the converged solve must return phi;
* geometric invariants of the tagging (sphere volume and symmetry);
* the LAPACK semantics of the 8x8 inverse (GCM_SET_BOUNDARY.F90:769-773)
  and the Thomas algorithm (CORE_TDMA.F90:10-34) against numpy/scipy.
"""
import math

import numpy as np
import pytest
import scipy.linalg

from feicar_b200 import synth
import oracle as O


def test_invert8_matches_scipy():
    rng = np.random.default_rng(3)
    for _ in range(50):
        a = rng.standard_normal((8, 8)) + 4 * np.eye(8)
        inv, info = O.invert8(np.asfortranarray(a))
        assert info == 0
        ref = scipy.linalg.inv(a)
        assert np.allclose(inv, ref, rtol=1e-11, atol=1e-12)


def test_invert8_vandermonde_rows():
    """Trilinear Vandermonde rows of a stretched host cell, the matrices the
    ghost-cell weights invert."""
    xs, ys, zs = (0.3, 0.37), (1.1, 1.13), (2.0, 2.08)
    rows = []
    for (i, j, k) in [(0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0), (0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1)]:
        x, y, z = xs[i], ys[j], zs[k]
        rows.append([x * y * z, x * y, x * z, y * z, x, y, z, 1.0])
    a = np.array(rows)
    inv, info = O.invert8(np.asfortranarray(a))
    assert info == 0
    assert np.allclose(inv @ a, np.eye(8), atol=1e-8)


def test_tdma_matches_dense():
    rng = np.random.default_rng(4)
    n = 40
    a = rng.uniform(-1, 0, n)
    c = rng.uniform(-1, 0, n)
    b = 2.5 + rng.uniform(0, 1, n)
    r = rng.standard_normal(n)
    u = O.tdma(a, b, c, r, 0, n - 1)
    m = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
    assert np.allclose(u, np.linalg.solve(m, r), rtol=1e-12, atol=1e-12)


def _no_body_solve(grid, rhs, restol=1e-12):
    oc = O.OracleCase(grid)
    z = np.zeros(grid.shape, np.int8, order="F")
    p = np.zeros(grid.shape, order="F")
    rc, st = oc.solve_poisson(p, np.asfortranarray(rhs),
                              params=O.default_params(restol_pson=restol, restol_gcp=restol,
                                                      itermax_pson=400))
    return p, st


def test_mg_analytic_second_order():
    """test_mg of the reference: error against the closed form falls ~4x per
    halving of h."""
    errs = []
    for n in (16, 32):
        g = synth.Grid(synth.uniform_nodes(n, 0, 1), synth.uniform_nodes(n, 0, 1), synth.uniform_nodes(n, 0, 1))
        rhs = synth.test_mg_rhs(g)
        p, st = _no_body_solve(g, rhs)
        ex = synth.test_mg_exact(g)
        s = (slice(1, g.nx), slice(1, g.ny), slice(1, g.nz))
        e = (p[s] - p[s].mean()) - (ex[s] - ex[s].mean())
        errs.append(np.abs(e).max() / np.abs(ex[s]).max())
    ratio = errs[0] / errs[1]
    assert errs[1] < 0.05
    assert 3.0 < ratio < 5.5, errs


@pytest.mark.parametrize("stretch", [None, 2.0])
def test_manufactured_solution_recovered(stretch):
    g = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0), stretch=stretch)
    b = synth.sphere_body((1.0, 1.0, 1.0), 1.0, 3)
    oc = O.OracleCase(g)
    oc.add_body(b)
    oc.set_iblank()
    assert oc.gcm(2.0, 2.0) == 0
    G, D = oc.ghosts(), oc.deads()
    rows = [synth.Interp(D["ijk"], D["cell"], D["coefN"]), synth.Interp(G["ijk"], G["cell"], G["coefN"])]
    ib, gh, dd = oc.field(0), oc.field(1), oc.field(2)
    rhs, phi = synth.manufactured_rhs(g, ib, gh, dd, rows, seed=2)
    p = np.zeros(g.shape, order="F")
    rc, st = oc.solve_poisson(p, rhs, params=O.default_params(restol_pson=1e-13, restol_gcp=1e-13,
                                                               itermax_pson=400))
    m = np.zeros(g.shape, bool)
    m[1:g.nx, 1:g.ny, 1:g.nz] = ib[1:g.nx, 1:g.ny, 1:g.nz] == 0
    a = p[m] - p[m].mean()
    e = phi[m] - phi[m].mean()
    assert np.linalg.norm(a - e) / np.linalg.norm(e) < 1e-9, st


def test_sphere_volume_and_symmetry():
    n = 32
    g = synth.Grid(synth.uniform_nodes(n, 0, 2), synth.uniform_nodes(n, 0, 2), synth.uniform_nodes(n, 0, 2))
    r = 0.6
    oc = O.OracleCase(g)
    oc.add_body(synth.sphere_body((1.0, 1.0, 1.0), 2 * r, 4))
    oc.set_iblank()
    oc.gcm(2.0, 2.0)
    ib = oc.field(0)[1:g.nx, 1:g.ny, 1:g.nz].astype(np.int64)
    h = 2.0 / n
    vol = ib.sum() * h ** 3
    assert abs(vol - 4.0 / 3.0 * math.pi * r ** 3) / (4.0 / 3.0 * math.pi * r ** 3) < 0.05
    # the icosphere and the grid are symmetric about the centre planes
    assert np.array_equal(ib, ib[::-1, :, :])
    assert np.array_equal(ib, ib[:, ::-1, :])
    assert np.array_equal(ib, ib[:, :, ::-1])
    nghost = oc.counts()["nGhost"]
    area = 4 * math.pi * r ** 2
    assert 0.5 < nghost * h * h / area < 3.0


def test_ghost_and_dead_definitions():
    """ghost = fluid interior cell face-adjacent to iblank; dead = iblank
    cell face-adjacent to a ghost (GCM_SET_BOUNDARY.F90:800-876, :946-964)."""
    g = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0), stretch=2.0)
    oc = O.OracleCase(g)
    oc.add_body(synth.sphere_body((1.0, 1.0, 1.0), 1.0, 3))
    oc.set_iblank()
    oc.gcm(2.0, 2.0)
    ib, gh, dd = oc.field(0), oc.field(1), oc.field(2)
    nx, ny, nz = g.nx, g.ny, g.nz
    I = slice(1, nx), slice(1, ny), slice(1, nz)
    nb = np.zeros((nx - 1, ny - 1, nz - 1), bool)
    for ax in range(3):
        for d in (-1, 1):
            sl = [slice(1, nx), slice(1, ny), slice(1, nz)]
            sl[ax] = slice(1 + d, [nx, ny, nz][ax] + d)
            nb |= ib[tuple(sl)] == 1
    # i-neighbours at 0 and nx are not visited by the reference loop
    want = (ib[I] == 0) & nb
    assert np.array_equal(gh[I] == 1, want)
    ghosts = oc.ghosts()
    ijk = ghosts["ijk"]
    lin = ijk[:, 0] + (nx + 2) * (ijk[:, 1] + (ny + 2) * ijk[:, 2])
    assert np.all(np.diff(lin) > 0)  # (k,j,i) list order
    assert np.all(ib[dd == -1] == 1)


def test_slab_parallel_sweeps_reach_same_solution():
    """The timed CPU baseline runs the line sweeps on z-slabs, one per
    thread, as the reference runs them on MPI ranks (block-Jacobi across
    slab faces).  The iterates differ from the sequential sweeps, the
    converged solution does not: both recover the manufactured solution to
    1e-9."""
    g = synth.small_grid(32, 16, 24, (4.0, 2.0, 3.0), stretch=2.0)
    b = synth.sphere_body((1.0, 1.0, 1.5), 1.0, 3)
    oc = O.OracleCase(g)
    oc.add_body(b)
    oc.set_iblank()
    assert oc.gcm(2.0, 2.0) == 0
    G, D = oc.ghosts(), oc.deads()
    rows = [synth.Interp(D["ijk"], D["cell"], D["coefN"]), synth.Interp(G["ijk"], G["cell"], G["coefN"])]
    ib, gh, dd = oc.field(0), oc.field(1), oc.field(2)
    rhs, phi = synth.manufactured_rhs(g, ib, gh, dd, rows, seed=3)
    m = np.zeros(g.shape, bool)
    m[1:g.nx, 1:g.ny, 1:g.nz] = ib[1:g.nx, 1:g.ny, 1:g.nz] == 0
    e = phi[m] - phi[m].mean()
    sols = []
    try:
        for threads in (1, 3):
            O.set_threads(threads)
            p = np.zeros(g.shape, order="F")
            rc, st = oc.solve_poisson(p, rhs.copy(order="F"),
                                      params=O.default_params(restol_pson=1e-13, restol_gcp=1e-13,
                                                              itermax_pson=400))
            a = p[m] - p[m].mean()
            assert np.linalg.norm(a - e) / np.linalg.norm(e) < 1e-9, (threads, st)
            sols.append(a)
    finally:
        O.set_threads(1)
    assert np.linalg.norm(sols[0] - sols[1]) / np.linalg.norm(e) < 1e-9


def test_oracle_momentum_sweep_reaches_a_manufactured_solution():
    """With no convection (crank_nicolson off) the momentum system is
    (I - dt/2 nu L) v = r on the fluid cells (set_solve_ad's coefficients,
    CORE_SET_SOLVERS.F90:650-675) with v held on solid and ghost cells and
    on the boundary layers.  r is formed from a known v by that operator,
    so the line sweeps must return v."""
    grid = synth.small_grid(24, 16, 12, (3.0, 2.0, 1.5), stretch=1.5)
    oc = O.OracleCase(grid)
    oc.add_body(synth.sphere_body((1.5, 1.0, 0.75), 0.6, 2))
    oc.set_iblank()
    oc.gcm(2.0, 2.0)
    dt, reinv = 0.2, 1.0 / 10.0
    ad = oc.set_solve_ad(dt, reinv)
    rng = np.random.default_rng(3)
    vex = np.asfortranarray(rng.standard_normal(grid.shape))
    zero = np.zeros(grid.shape, order="F")
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    I, J, K = nx + 2, ny + 2, nz + 2
    amx, apx = ad[0:I], ad[I:2 * I]
    amy, apy = ad[2 * I:2 * I + J], ad[2 * I + J:2 * I + 2 * J]
    amz, apz = ad[2 * I + 2 * J:2 * I + 2 * J + K], ad[2 * I + 2 * J + K:]
    # r = A vex on the fluid cells, cell by cell from the coefficients
    r = np.zeros(grid.shape, order="F")
    ib, gh = oc.field(0), oc.field(1)
    for k in range(1, nz):
        for j in range(1, ny):
            for i in range(1, nx):
                ac = 1.0 - (amx[i] + apx[i]) - (amy[j] + apy[j]) - (amz[k] + apz[k])
                r[i, j, k] = (ac * vex[i, j, k] + amx[i] * vex[i - 1, j, k] + apx[i] * vex[i + 1, j, k]
                              + amy[j] * vex[i, j - 1, k] + apy[j] * vex[i, j + 1, k]
                              + amz[k] * vex[i, j, k - 1] + apz[k] * vex[i, j, k + 1])
    fluid = (ib == 0) & (gh == 0)
    interior = np.zeros(grid.shape, bool)
    interior[1:nx, 1:ny, 1:nz] = True
    var = np.where(fluid & interior, 0.0, vex).copy(order="F")  # held cells start at their values
    for _ in range(60):
        oc.itsolv_ad(ad, var, r, zero, zero, zero, 0.0, 1.0)
    m = fluid & interior
    assert np.abs(var[m] - vex[m]).max() <= 1e-11
    res, _ = oc.calc_residual_ad(ad, var, r, zero, zero, zero, 0.0)
    assert res <= 1e-11
