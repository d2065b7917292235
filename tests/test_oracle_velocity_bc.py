"""The oracle's outer velocity boundaries and momentum iteration without a
GPU: set_outer_velocity_bc (CORE_SET_OUTER_BC.F90:18-509) against a numpy
statement of each face type, set_outer_ghost_velocity (:739-823), and
solve_ad (CORE_SOLVE_AD.F90:11-127) on a channel past a sphere: Dirichlet
inflow, zero-gradient outflow, symmetry walls.

The face-by-face statement below writes each type's formula the way the
reference does (same operations, same order), so the arrays agree bit for
bit; the pulsatile values use Python's math.sin, the C library's sin.
"""
import math

import numpy as np

from feicar_b200 import synth
import oracle as O


def _case(nx=24, ny=12, nz=10):
    grid = synth.small_grid(nx, ny, nz, (4.0, 2.0, 2.0), stretch=1.3)
    oc = O.OracleCase(grid)
    return grid, oc


def _vb(types, time=1.7):
    vb = O.VelocityBC()
    rng = np.random.default_rng(5)
    for f in range(6):
        vb.type[f] = types[f]
        for a in range(3):
            vb.val[f][a] = float(rng.uniform(0.5, 1.5))
            vb.freq[f][a] = float(rng.uniform(0.05, 0.3))
    vb.time = time
    vb.yOrigin, vb.yout, vb.zOrigin, vb.zout = 0.0, 2.0, 0.0, 2.0
    return vb


def _expected(grid, u, v, w, vb, bc0):
    """The nine arrays after set_outer_velocity_bc, face by face."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    y, z = grid.y, grid.z  # node coordinates, reference indexing 0..n+1
    bc = [a.copy(order="F") for a in bc0]
    F = (u, v, w)
    pi = 4.0 * math.atan(1.0)
    t = vb.time

    def puls(f, a):
        return vb.val[f][a] * math.sin(2.0 * pi * vb.freq[f][a] * t)

    def chan(val, s, lo, hi):
        e = hi - lo
        return val * 6.0 * (s - lo) * (hi - s) / (e * e)

    for side in (0, 1):
        i, io, f = (1, nx - 1, 0) if side == 0 else (nx - 1, 1, 1)
        ty, val = vb.type[f], vb.val[f]
        for a in range(3):
            B = bc[a][side]
            if ty == 1:
                B[:, :] = val[a]
            elif ty == 2:
                B[:, :] = F[a][i]
            elif ty == 3:
                B[:, :] = (val[0] * t / 30.0) if (side == 0 and a == 0) else puls(f, a)
            elif ty == 4:
                B[:, :] = 0.0 if a == 0 else F[a][i]
            elif ty == 5:
                B[:, :] = 0.5 * (F[a][i] + F[a][io])
            elif ty == 6:
                if a == 0:
                    B[:, :] = np.array([chan(val[0], y[j], vb.yOrigin, vb.yout) for j in range(ny + 2)])[:, None]
                elif side == 1:
                    B[:, :] = val[a]
    for side in (0, 1):
        j, jo, f = (1, ny - 1, 2) if side == 0 else (ny - 1, 1, 3)
        ty, val = vb.type[f], vb.val[f]
        for a in range(3):
            B = bc[3 + a][:nx + 1, side, :]
            src = F[a][:nx + 1, j, :]
            if ty == 1:
                B[:, :] = val[a]
            elif ty == 2:
                B[:, :] = src
            elif ty == 3:
                B[:, :] = puls(f, a)
            elif ty == 4:
                B[:, :] = 0.0 if a == 1 else src
            elif ty == 5:
                B[:, :] = 0.5 * (src + F[a][:nx + 1, jo, :])
        if ty == 6:
            bc[0][1, j, :] = vb.val[f][0]
            bc[1][1, j, :] = [chan(vb.val[f][1], z[k], vb.zOrigin, vb.zout) for k in range(nz + 2)]
            bc[2][1, j, :] = vb.val[f][2]
    for side in (0, 1):
        k, ko, f = (1, nz - 1, 4) if side == 0 else (nz - 1, 1, 5)
        ty, val = vb.type[f], vb.val[f]
        for a in range(3):
            B = bc[6 + a][:nx + 1, :, side]
            src = F[a][:nx + 1, :, k]
            if ty == 1:
                B[:, :] = val[a]
            elif ty == 2:
                B[:, :] = src
            elif ty == 3:
                B[:, :] = puls(f, a)
            elif ty == 4:
                B[:, :] = 0.0 if a == 2 else src
            elif ty == 5:
                B[:, :] = 0.5 * (src + F[a][:nx + 1, :, ko])
        if ty == 6:
            bc[0][1, :, k] = vb.val[f][0]
            bc[1][1, :, k] = vb.val[f][1]
            bc[2][1, :, k] = [chan(vb.val[f][2], y[jj], vb.yOrigin, vb.yout) for jj in range(ny + 2)]
    return bc


TYPE_SETS = [(1, 2, 4, 4, 4, 4), (3, 2, 5, 5, 3, 3), (6, 6, 1, 2, 4, 5), (5, 5, 6, 6, 1, 1), (2, 1, 3, 4, 6, 6),
             (4, 3, 2, 1, 5, 2)]


def test_outer_velocity_bc_face_types():
    grid, oc = _case()
    rng = np.random.default_rng(3)
    u, v, w = (np.asfortranarray(rng.standard_normal(grid.shape)) for _ in range(3))
    for types in TYPE_SETS:
        vb = _vb(types)
        bc = oc.bc_arrays()
        for a in bc:
            a[...] = rng.standard_normal(a.shape)
        want = _expected(grid, u, v, w, vb, bc)
        assert oc.set_outer_velocity_bc(u, v, w, bc, vb) == 0
        for q in range(9):
            assert np.array_equal(bc[q], want[q]), (types, q)


def test_shear_face_is_rejected():
    grid, oc = _case()
    u = np.zeros(grid.shape, order="F")
    assert oc.set_outer_velocity_bc(u, u, u, oc.bc_arrays(), _vb((1, 2, 7, 4, 4, 4))) == 5  # OR_BAD_INPUT


def test_outer_ghost_layer_reflects_about_the_boundary_value():
    grid, oc = _case()
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    rng = np.random.default_rng(4)
    u, v, w = (np.asfortranarray(rng.standard_normal(grid.shape)) for _ in range(3))
    bc = oc.bc_arrays()
    for a in bc:
        a[...] = rng.standard_normal(a.shape)
    F0 = [a.copy() for a in (u, v, w)]
    oc.set_outer_ghost_velocity(u, v, w, bc)
    for a, f in enumerate((u, v, w)):
        # x faces away from the y and z ghost layers the later faces rewrite
        J, K = slice(1, ny), slice(1, nz)
        assert np.array_equal(f[0, J, K], 2.0 * bc[a][0, J, K] - F0[a][1, J, K])
        assert np.array_equal(f[nx, J, K], 2.0 * bc[a][1, J, K] - F0[a][nx - 1, J, K])
        # the z faces come last: every (i, j) of 0..nx x 0..ny+1
        assert np.array_equal(f[:nx + 1, :, 0], 2.0 * bc[6 + a][:nx + 1, :, 0] - f[:nx + 1, :, 1])
        assert np.array_equal(f[:nx + 1, :, nz], 2.0 * bc[6 + a][:nx + 1, :, 1] - f[:nx + 1, :, nz - 1])
        # the y faces over i = 0..nx, away from the z ghost planes
        assert np.array_equal(f[:nx + 1, 0, 1:nz], 2.0 * bc[3 + a][:nx + 1, 0, 1:nz] - f[:nx + 1, 1, 1:nz])
        # i = nx + 1 is no ghost cell of any face
        assert np.array_equal(f[nx + 1, 1:ny, 1:nz], F0[a][nx + 1, 1:ny, 1:nz])


def _channel():
    grid = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0), stretch=1.3)
    body = synth.sphere_body((1.5, 1.0, 1.0), 0.5, 3)
    oc = O.OracleCase(grid)
    oc.add_body(body)
    oc.set_iblank()
    assert oc.gcm(2.0, 2.0) == 0
    vb = O.VelocityBC()
    for f, ty in enumerate((1, 2, 4, 4, 4, 4)):
        vb.type[f] = ty
    vb.val[0][0] = 1.0
    return grid, oc, vb


def channel_state(grid, oc, vb, dt=0.05, reinv=0.01):
    """A time step's inputs: u = 1 with the outer boundaries and faces set."""
    u = np.asfortranarray(np.ones(grid.shape))
    v, w = np.zeros(grid.shape, order="F"), np.zeros(grid.shape, order="F")
    bc = oc.bc_arrays()
    assert oc.set_outer_velocity_bc(u, v, w, bc, vb) == 0
    oc.set_outer_ghost_velocity(u, v, w, bc)
    fu, fv, fw = oc.face_vel(u, v, w, bc[0], bc[4], bc[8])
    nl = [a.copy(order="F") for a in (u, v, w)]
    return u, v, w, nl, [np.asfortranarray(a) for a in (fu, fv, fw)], bc, oc.set_solve_ad(dt, reinv), dt


def net_flux(grid, oc, fu, fv, fw):
    ib, gh = oc.field(0), oc.field(1)
    dx, dy, dz = np.diff(grid.x), np.diff(grid.y), np.diff(grid.z)  # dx[i] = x(i+1) - x(i)
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    I, J, K = slice(1, nx), slice(1, ny), slice(1, nz)
    flag = (1.0 - ib[I, J, K]) * (1.0 - np.abs(gh[I, J, K]))
    f = ((fu[2:nx + 1, J, K] - fu[I, J, K]) * dy[None, 1:ny, None] * dz[None, None, 1:nz] +
         (fv[I, 2:ny + 1, K] - fv[I, J, K]) * dx[1:nx, None, None] * dz[None, None, 1:nz] +
         (fw[I, J, 2:nz + 1] - fw[I, J, K]) * dx[1:nx, None, None] * dy[None, 1:ny, None])
    return float((flag * f).sum())


def test_solve_ad_converges_on_a_channel_past_a_sphere():
    grid, oc, vb = _channel()
    u, v, w, nl, (fu, fv, fw), bc, ad, dt = channel_state(grid, oc, vb)
    ug, ud, _, _ = oc.body_intercept_values(1, dt)
    pld = 2.0
    rc, it, res, loc = oc.solve_ad(ad, u, v, w, *nl, fu, fv, fw, bc, ug, ud, 0.5 * dt, 1.0, vb, pld, 500, 1e-12,
                                   200, 1e-9)
    assert rc == 0 and 1 < it < 200 and res <= 1e-9
    assert all(1 <= x for x in loc)
    # the last face velocities carry no net mass flux out of the fluid cells
    assert abs(net_flux(grid, oc, fu, fv, fw)) <= 1e-12 * 4.0
    # the no-slip sphere slows the flow next to it: the first fluid cell
    # downstream of it on the centre line; the inflow face keeps u = 1
    j, k = grid.ny // 2, grid.nz // 2
    ib = oc.field(0)
    last_solid = int(np.nonzero(ib[:, j, k])[0].max())
    assert u[last_solid + 1, j, k] < 0.5
    J, K = slice(1, grid.ny), slice(1, grid.nz)
    assert np.array_equal(bc[0][0, J, K], np.ones((grid.ny - 1, grid.nz - 1)))


def test_solve_ad_stops_at_itermax_and_reports_it():
    grid, oc, vb = _channel()
    u, v, w, nl, (fu, fv, fw), bc, ad, dt = channel_state(grid, oc, vb)
    ug, ud, _, _ = oc.body_intercept_values(1, dt)
    rc, it, res, _ = oc.solve_ad(ad, u, v, w, *nl, fu, fv, fw, bc, ug, ud, 0.5 * dt, 1.0, vb, 2.0, 500, 1e-12, 3,
                                 0.0)
    assert rc == 0 and it == 3 and res > 0.0
