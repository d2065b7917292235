"""Body-intercept values and the velocity ghost cells on the device against
the oracle's restatement of GCM_SetBodyInterceptValues /
GCM_calc_BIVelocity_Unstruc (GCM_BODYINTERCEPT_VALUES.F90:22-388) and
GCM_ghostcell_velocity (GCM_GHOSTCELL_UPDATE.F90:1-359, iOpt = 2,
mix_GC_form = 0).

A sphere translating and rotating (prescribed rigid motion, two steps on
the device and in the oracle), re-tagged at its new position:
* the intercept velocities (this and the previous step's marker velocities
  interpolated over the closest element) and dp/dn at every ghost and dead
  row agree bit for bit (both compiled without FMA contraction);
* the velocity ghost and dead cells, iterated to restol_gcv 1e-14 (Jacobi
  sweeps on the device, the reference's in-place sweeps in the oracle),
  agree to 1e-12 of the field's largest value.
"""
import numpy as np
import pytest
import torch

from feicar_b200 import fg, synth
import oracle as O

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).transpose(*range(a.ndim)[::-1]))).cuda()


def _host(t):
    return t.cpu().numpy().transpose(*range(t.ndim)[::-1])


def _motion(cls):
    m = cls()
    m.angv_init[2] = 0.5
    m.vcent_trans[0] = 0.3
    m.ampang[1] = 0.4
    m.freqang[1] = 0.05
    m.cent[:] = (1.6, 1.0, 1.0)
    return m


def _cases():
    grid = synth.small_grid(40, 24, 24, (4.0, 2.0, 2.0), stretch=1.5)
    body = synth.sphere_body((1.6, 1.0, 1.0), 0.8, 3)
    oc = O.OracleCase(grid)
    oc.add_body(body)
    c = fg.Case(grid, fg.default_config())
    c.add_body(body)
    mo, md = _motion(O.RigidMotion), _motion(fg.RigidMotion)
    dt = 0.05
    for n in (1, 2):
        oc.move_body(0, mo, n, n * dt, dt)
        fg.move_body(c, 0, md, n, n * dt, dt)
    oc.set_iblank(ntime=2)
    assert oc.gcm(2.0, 2.0) == 0
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    assert (c.nGhost, c.nDead) == (oc.counts()["nGhost"], oc.counts()["nDead"])
    return grid, oc, c, dt


def test_body_intercept_values_match_oracle_bit_for_bit():
    grid, oc, c, dt = _cases()
    for ntime in (1, 2):
        ug, ud, pg, pd = oc.body_intercept_values(ntime, dt)
        d_ug = torch.zeros(3 * c.nGhost, dtype=torch.float64, device="cuda")
        d_ud = torch.zeros(3 * c.nDead, dtype=torch.float64, device="cuda")
        d_pg = torch.full((c.nGhost,), 7.0, dtype=torch.float64, device="cuda")
        d_pd = torch.full((c.nDead,), 7.0, dtype=torch.float64, device="cuda")
        fg.body_intercept_values_device(c, ntime, dt, d_ug.data_ptr(), d_ud.data_ptr(), d_pg.data_ptr(),
                                        d_pd.data_ptr())
        assert np.array_equal(d_ug.cpu().numpy().reshape(-1, 3), ug)
        assert np.array_equal(d_ud.cpu().numpy().reshape(-1, 3), ud)
        assert np.array_equal(d_pg.cpu().numpy(), pg) and np.array_equal(d_pd.cpu().numpy(), pd)
        if ntime == 1:
            assert not pg.any() and not pd.any()
        else:
            assert np.abs(pg).max() > 0 and np.abs(ug).max() > 0.2  # the body moves
    c.close()


def test_ghostcell_velocity_matches_oracle():
    grid, oc, c, dt = _cases()
    ug, ud, _, _ = oc.body_intercept_values(2, dt)
    rng = np.random.default_rng(12)
    u, v, w = (np.asfortranarray(synth.box_smooth(rng.standard_normal(grid.shape))) for _ in range(3))
    du, dv, dw = _dev(u), _dev(v), _dev(w)
    pld = fg.default_config().probe_length_dead
    rc, it = oc.ghostcell_velocity(u, v, w, ug, ud, pld, 500, 1e-14)
    assert rc == 0 and it > 1
    d_ug = torch.from_numpy(np.ascontiguousarray(ug).ravel()).cuda()
    d_ud = torch.from_numpy(np.ascontiguousarray(ud).ravel()).cuda()
    sweeps = fg.ghostcell_velocity_device(c, du.data_ptr(), dv.data_ptr(), dw.data_ptr(), d_ug.data_ptr(),
                                          d_ud.data_ptr(), 500, 1e-14)
    assert sweeps > 1
    for a, t in ((u, du), (v, dv), (w, dw)):
        h = _host(t)
        assert np.abs(h - a).max() <= 1e-12 * np.abs(a).max()
    c.close()
