"""The outer velocity boundaries and the momentum iteration on the device
(fg_set_outer_velocity_bc_device, fg_set_outer_ghost_velocity_device,
fg_enforce_global_mass_consv_device, fg_solve_ad_device) against the
oracle's restatement of set_outer_velocity_bc / set_outer_ghost_velocity /
enforce_global_mass_consv (CORE_SET_OUTER_BC.F90:18-823) and solve_ad
(CORE_SOLVE_AD.F90:11-127).

* Every face type on every face: the nine boundary arrays bit for bit
  (the file that forms them is compiled without FMA contraction, the
  pulsatile values use the host's sin as the oracle does).
* The outer ghost layer bit for bit.
* Mass conservation: the same correction to 1e-14 (the flux sum is a
  parallel reduction on the device).
* solve_ad on a channel past a sphere (Dirichlet inflow, zero-gradient
  outflow, symmetry walls): after three fixed iterations and at
  convergence the velocities agree with the oracle's to 1e-10 of the
  inflow speed (the velocity ghost cells are Jacobi sweeps on the device
  and in-place sweeps in the oracle, both to restol_gcv 1e-13), the
  converged iteration counts within one, and the last face velocities
  carry no net mass flux.
"""
import numpy as np
import pytest
import torch

from feicar_b200 import fg, synth
import oracle as O
from test_oracle_velocity_bc import TYPE_SETS, _channel, _vb, channel_state, net_flux

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).transpose(*range(a.ndim)[::-1]))).cuda()


def _host(t):
    return t.cpu().numpy().transpose(*range(t.ndim)[::-1])


def _fvb(ovb):
    vb = fg.VelocityBC()
    for f in range(6):
        vb.type[f] = ovb.type[f]
        for a in range(3):
            vb.val[f][a] = ovb.val[f][a]
            vb.freq[f][a] = ovb.freq[f][a]
    for n in ("time", "yOrigin", "yout", "zOrigin", "zout"):
        setattr(vb, n, getattr(ovb, n))
    return vb


def _device_case(grid, body=None):
    c = fg.Case(grid, fg.default_config())
    if body is not None:
        c.add_body(body)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    return c


def test_outer_velocity_bc_and_ghost_layer_bit_for_bit():
    grid = synth.small_grid(24, 12, 10, (4.0, 2.0, 2.0), stretch=1.3)
    body = synth.sphere_body((2.0, 1.0, 1.0), 0.4, 2)
    oc = O.OracleCase(grid)
    c = _device_case(grid, body)
    rng = np.random.default_rng(3)
    u, v, w = (np.asfortranarray(rng.standard_normal(grid.shape)) for _ in range(3))
    du, dv, dw = _dev(u), _dev(v), _dev(w)
    for types in TYPE_SETS:
        ovb = _vb(types)
        bc = oc.bc_arrays()
        for a in bc:
            a[...] = rng.standard_normal(a.shape)
        dbc = [_dev(a) for a in bc]
        assert oc.set_outer_velocity_bc(u, v, w, bc, ovb) == 0
        fg.set_outer_velocity_bc_device(c, du.data_ptr(), dv.data_ptr(), dw.data_ptr(),
                                        [t.data_ptr() for t in dbc], _fvb(ovb))
        for q in range(9):
            assert np.array_equal(_host(dbc[q]), bc[q]), (types, q)
        uu, vv, ww = (a.copy(order="F") for a in (u, v, w))
        du2, dv2, dw2 = _dev(uu), _dev(vv), _dev(ww)
        oc.set_outer_ghost_velocity(uu, vv, ww, bc)
        fg.set_outer_ghost_velocity_device(c, du2.data_ptr(), dv2.data_ptr(), dw2.data_ptr(),
                                           [t.data_ptr() for t in dbc])
        for a, t in ((uu, du2), (vv, dv2), (ww, dw2)):
            assert np.array_equal(_host(t), a), types
    with pytest.raises(fg.FGError):
        fg.set_outer_velocity_bc_device(c, du.data_ptr(), dv.data_ptr(), dw.data_ptr(),
                                        [t.data_ptr() for t in dbc], _fvb(_vb((1, 2, 7, 4, 4, 4))))
    c.close()


def test_enforce_global_mass_consv_matches_oracle():
    grid, oc, ovb = _channel()
    u, v, w, nl, (fu, fv, fw), bc, ad, dt = channel_state(grid, oc, ovb)
    c = _device_case(grid, synth.sphere_body((1.5, 1.0, 1.0), 0.5, 3))
    rng = np.random.default_rng(9)
    fu = np.asfortranarray(fu + 0.01 * rng.standard_normal(fu.shape))  # a net outflow to remove
    vzg = [0, 1, 0, 0, 1, 0]
    d = [_dev(a) for a in (fu, fv, fw, bc[0], bc[4], bc[8])]
    oc.enforce_global_mass_consv(fu, fv, fw, bc[0], bc[4], bc[8], vzg)
    fg.enforce_global_mass_consv_device(c, *[t.data_ptr() for t in d], vzg)
    for a, t in zip((fu, fv, fw, bc[0], bc[4], bc[8]), d):
        assert np.abs(_host(t) - a).max() <= 1e-14 * max(1.0, np.abs(a).max())
    assert abs(net_flux(grid, oc, fu, fv, fw)) <= 1e-12
    c.close()


@pytest.mark.parametrize("converge", [False, True])
def test_solve_ad_matches_oracle(converge):
    grid, oc, ovb = _channel()
    u, v, w, nl, (fu, fv, fw), bc, ad, dt = channel_state(grid, oc, ovb)
    c = _device_case(grid, synth.sphere_body((1.5, 1.0, 1.0), 0.5, 3))
    assert (c.nGhost, c.nDead) == (oc.counts()["nGhost"], oc.counts()["nDead"])
    ug, ud, _, _ = oc.body_intercept_values(1, dt)
    pld = fg.default_config().probe_length_dead
    itermax, restol = (200, 1e-9) if converge else (3, 0.0)
    d = {k: _dev(a) for k, a in dict(u=u, v=v, w=w, nlu=nl[0], nlv=nl[1], nlw=nl[2], fu=fu, fv=fv, fw=fw).items()}
    dbc = [_dev(a) for a in bc]
    d_ug = torch.from_numpy(np.ascontiguousarray(ug).ravel()).cuda()
    d_ud = torch.from_numpy(np.ascontiguousarray(ud).ravel()).cuda()
    rc, it_o, res_o, _ = oc.solve_ad(ad, u, v, w, *nl, fu, fv, fw, bc, ug, ud, 0.5 * dt, 1.0, ovb, pld, 500, 1e-13,
                                     itermax, restol)
    assert rc == 0
    prm = fg.AdParams(dt=dt, reinv=0.01, omega_ad=1.0, crank_nicolson=1)
    it_d, res_d, loc_d = fg.solve_ad_device(c, *[d[k].data_ptr() for k in ("u", "v", "w", "nlu", "nlv", "nlw", "fu",
                                                                            "fv", "fw")],
                                            [t.data_ptr() for t in dbc], d_ug.data_ptr(), d_ud.data_ptr(), prm,
                                            _fvb(ovb), 500, 1e-13, itermax, restol)
    if converge:
        assert abs(it_d - it_o) <= 1 and res_d <= restol and 1 < it_d < itermax
    else:
        assert it_d == it_o == 3 and res_d == pytest.approx(res_o, rel=1e-6)
    for k, a in (("u", u), ("v", v), ("w", w)):
        assert np.abs(_host(d[k]) - a).max() <= 1e-10, k
    hf = [_host(d[k]) for k in ("fu", "fv", "fw")]
    assert abs(net_flux(grid, oc, *hf)) <= 1e-12
    c.close()
