"""Prescribed rigid body motion on the device (fg_move_body) against the
oracle's restatement of move_boundary / forced_motion / compute_marker_vel
/ compute_marker_poisition (BOUNDARY_MOVE.F90:3-186,
BOUNDARY_MARKER_VEL.F90:5-125): the config-2 membrane plate pitching about
its leading edge by a sinusoidal angular velocity, 30 time steps.

Bit for bit, every step: marker positions, velocities, dp/dn, the largest
displacement since the last re-tag and the re-tag decision.  At every tenth
step the device tagging of the device-moved plate (iblank, ghost and dead
lists) equals the oracle's tagging of its own moved plate.
"""
import importlib.util
import os

import numpy as np
import pytest

from feicar_b200 import fg, synth
import oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
_mg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_mg)


def _motion(cls):
    m = cls()
    m.ampang[2] = 2.0 * np.pi / 100.0 * np.radians(30.0)  # 30 deg amplitude over a 100-step period
    m.freqang[2] = 1.0 / 100.0
    m.angphase[2] = np.pi / 2.0
    m.vcent_trans[0] = 0.01
    m.cent[:] = (2.0, 2.0, 2.0)
    return m


def test_pitching_plate_moves_like_the_oracle():
    grid = synth.config2_grid()
    body = synth.config2_body(0)
    oc = O.OracleCase(grid)
    oc.add_body(body)
    c = fg.Case(grid, fg.default_config())
    c.add_body(body)
    mo, md = _motion(O.RigidMotion), _motion(fg.RigidMotion)
    dt = 1.0
    resets = 0
    for n in range(1, 31):
        t = n * dt
        ds_o, r_o = oc.move_body(0, mo, n, t, dt)
        ds_d, r_d = fg.move_body(c, 0, md, n, t, dt)
        xo, uo, po = oc.body_markers(0, body.nvert)
        xd, ud, pd = fg.body_markers(c, 0, body.nvert)
        assert np.array_equal(xd, xo), n
        assert np.array_equal(ud, uo), n
        assert np.array_equal(pd, po), n
        assert ds_d == ds_o and r_d == r_o, n
        assert list(md.cent) == list(mo.cent) and list(md.angv_old) == list(mo.angv_old)
        resets += r_d
        if n % 10 == 0:
            oc.set_iblank(ntime=n)
            assert oc.gcm(2.0, 2.0) == 0
            want = _mg.tagging_digests(oc.field(0), oc.field(1), oc.field(2), oc.ghosts(), oc.deads())
            c.set_iblank_body_fast()
            ib, gh, dd = c.gcm_set_internal_boundary()
            got = _mg.tagging_digests(ib, gh, dd, c.ghost_rows(), c.dead_rows())
            assert got == want, n
    assert resets > 0
    c.close()
