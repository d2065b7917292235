"""The momentum line SOR on the device (fg_itsolv_ad_device,
fg_calc_residual_ad_device) against the oracle's restatement of
set_solve_ad, itsolv_ad_x/y/z and calc_residual_ad (CORE_SET_SOLVERS.F90:
591-677, CORE_SOLVE_AD.F90:131-964).

The device solves each direction's lines one anti-diagonal at a time, which
is the reference's lexicographic Gauss-Seidel order, and forms every
coefficient in the reference's operation order without FMA contraction:
the swept field is compared bit for bit after each pass, and the residual
with its location exactly.  Face velocities of both signs exercise the
upwind and central branches (the reference switches on 25 <= i <= 375; the
long x axis of the second case reaches past 375).
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


@pytest.mark.parametrize("case", ["sphere", "long_x"])
@pytest.mark.parametrize("cn", [1, 0])
def test_itsolv_ad_matches_oracle_bit_for_bit(case, cn):
    if case == "sphere":
        grid = synth.small_grid(40, 24, 20, (4.0, 2.0, 2.0), stretch=1.5)
        body = synth.sphere_body((1.2, 1.0, 1.0), 0.8, 3)
    else:
        grid = synth.small_grid(400, 8, 8, (40.0, 1.0, 1.0))
        body = synth.sphere_body((38.0, 0.5, 0.5), 0.6, 2)
    oc = O.OracleCase(grid)
    oc.add_body(body)
    oc.set_iblank()
    assert oc.gcm(2.0, 2.0) == 0
    c = fg.Case(grid, fg.default_config())
    c.add_body(body)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    dt, reinv = 0.01, 1.0 / 200.0
    prm = fg.AdParams(dt=dt, reinv=reinv, omega_ad=1.1, crank_nicolson=cn)
    ad = oc.set_solve_ad(dt, reinv)
    half_dt = 0.5 * dt if cn else 0.0
    rng = np.random.default_rng(7)
    sh = grid.shape
    fu, fv, fw = (np.asfortranarray(synth.box_smooth(rng.standard_normal(sh)) * 3.0) for _ in range(3))
    assert (fu < 0).any() and (fu > 0).any()
    r = np.asfortranarray(synth.box_smooth(rng.standard_normal(sh)))
    var = np.asfortranarray(0.1 * rng.standard_normal(sh))
    d = {k: _dev(a) for k, a in dict(fu=fu, fv=fv, fw=fw, r=r, var=var).items()}
    ptr = [d[k].data_ptr() for k in ("var", "r", "fu", "fv", "fw")]
    for it in range(3):
        oc.itsolv_ad(ad, var, r, fu, fv, fw, half_dt, 1.1)
        fg.itsolv_ad_device(c, *ptr, prm)
        assert np.array_equal(_host(d["var"]), var), it
        mo, lo = oc.calc_residual_ad(ad, var, r, fu, fv, fw, half_dt)
        md, ld = fg.calc_residual_ad_device(c, *ptr, prm)
        assert md == mo and ld == lo, (it, md, mo, ld, lo)
    c.close()


def test_itsolv_ad_converges_on_the_device():
    """Repeated passes drive the momentum residual to rounding level."""
    grid = synth.small_grid(48, 32, 32, (3.0, 2.0, 2.0), stretch=1.5)
    body = synth.sphere_body((1.5, 1.0, 1.0), 0.7, 3)
    c = fg.Case(grid, fg.default_config())
    c.add_body(body)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    rng = np.random.default_rng(8)
    sh = grid.shape
    f = [_dev(synth.box_smooth(rng.standard_normal(sh))) for _ in range(3)]
    r = _dev(synth.box_smooth(rng.standard_normal(sh)))
    var = torch.zeros_like(r)
    prm = fg.AdParams(dt=0.005, reinv=1.0 / 100.0, omega_ad=1.0, crank_nicolson=1)
    ptr = [var.data_ptr(), r.data_ptr()] + [t.data_ptr() for t in f]
    m0, _ = fg.calc_residual_ad_device(c, *ptr, prm)
    for _ in range(12):
        fg.itsolv_ad_device(c, *ptr, prm)
    m, _ = fg.calc_residual_ad_device(c, *ptr, prm)
    assert m <= 1e-12 * m0
    c.close()
