"""Properties that pin the oracle's prescribed rigid motion
(BOUNDARY_MARKER_VEL.F90:60-125 compute_marker_vel, BOUNDARY_MOVE.F90:151-186
compute_marker_poisition) without a GPU.

compute_marker_vel is the Crank-Nicolson (Cayley) rotation step: for a
constant angular velocity about one axis, x_{n+1} - c = R (x_n - c) with R
the rotation by 2 atan(dt |w| / 2), so every marker keeps its distance from
the centroid and turns by that angle each step.  A pure translation moves
every marker by dt * vcent.  dp/dn at the markers is zero on the first step
and -(du/dt . n) afterwards (BOUNDARY_MOVE.F90:96-110).
"""
import numpy as np

from feicar_b200 import synth
import oracle as O


def _case():
    grid = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0))
    body = synth.sphere_body((2.0, 1.0, 1.0), 0.8, 2)
    oc = O.OracleCase(grid)
    oc.add_body(body)
    return oc, body


def test_constant_rotation_is_a_cayley_step():
    oc, body = _case()
    m = O.RigidMotion()
    a = 0.3
    m.angv_init[2] = a
    m.angv_old[2] = a
    m.cent[:] = (2.0, 1.0, 1.0)
    dt = 0.1
    x0 = body.verts.copy()
    r0 = x0 - np.array(m.cent[:])
    theta = 2.0 * np.arctan(0.5 * dt * a)
    for n in range(1, 11):
        ds, _ = oc.move_body(0, m, n, n * dt, dt)
        x, u, p = oc.body_markers(0, body.nvert)
        r = x - np.array(m.cent[:])
        np.testing.assert_allclose(np.linalg.norm(r, axis=1), np.linalg.norm(r0, axis=1), rtol=0, atol=1e-13)
        c, s = np.cos(n * theta), np.sin(n * theta)
        want = np.stack([c * r0[:, 0] - s * r0[:, 1], s * r0[:, 0] + c * r0[:, 1], r0[:, 2]], axis=1)
        np.testing.assert_allclose(r, want, rtol=0, atol=1e-12)
        if n == 1:
            assert np.all(p == 0.0)
    # a constant angular velocity gives the markers a centripetal
    # acceleration: dp/dn = -(a . n) is nonzero on a sphere off its axis
    assert np.abs(p).max() > 0.0


def test_translation_moves_every_marker_by_dt_vcent():
    oc, body = _case()
    m = O.RigidMotion()
    m.vcent_trans[:] = (0.2, -0.1, 0.05)
    dt = 0.05
    for n in range(1, 6):
        oc.move_body(0, m, n, n * dt, dt)
    x, u, p = oc.body_markers(0, body.nvert)
    np.testing.assert_allclose(x - body.verts, np.tile(5 * dt * np.array([0.2, -0.1, 0.05]), (body.nvert, 1)),
                               rtol=0, atol=1e-14)
    np.testing.assert_array_equal(u, np.tile([0.2, -0.1, 0.05], (body.nvert, 1)))
    assert np.all(p == 0.0)  # no acceleration
    np.testing.assert_allclose(m.cent[:], 5 * dt * np.array([0.2, -0.1, 0.05]), rtol=0, atol=1e-15)


def test_retag_follows_the_displacement_since_the_last_snapshot():
    oc, body = _case()
    m = O.RigidMotion()
    g = oc.grid
    hmin = min(np.diff(g.xn).min(), np.diff(g.yn).min(), np.diff(g.zn).min())
    m.vcent_trans[0] = 0.02 * hmin  # 0.02 h per step: re-tag on the third step
    flags = [oc.move_body(0, m, n, float(n), 1.0)[1] for n in range(1, 7)]
    assert flags == [0, 0, 1, 0, 0, 1]
