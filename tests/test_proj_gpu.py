"""The projection steps either side of the pressure solve, on device
fields, against the oracle's restatement of the reference routines:
face_vel (CORE_FRAC_STEP_ROUTINES.F90:1-130), enforce_global_mass_consv +
rhs_poisson (CORE_SET_OUTER_BC.F90:515-735, CORE_POISSON.F90:9-79),
correct_vel / calc_pres_grad (CORE_FRAC_STEP_ROUTINES.F90:132-320), and a
whole time step's chain (face velocities -> div -> pressure solve ->
corrected velocity) kept on the device.

Tolerances: 1e-13 relative for the stencil steps (the device contracts
multiply-adds, the oracle does not), 1e-12 for the sums, 1e-8 for the
corrected velocity after a solve to rtol 1e-12 against the oracle's
converged solve.
"""
import numpy as np
import pytest
import torch

from feicar_b200 import fg, synth
import oracle as O

pytestmark = pytest.mark.gpu

GRID = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0), stretch=1.5)
BODY = synth.sphere_body((1.2, 1.0, 1.0), 0.8, 3)


def _dev(a):
    """Device copy of a Fortran-ordered array (the C layout of the reversed shape)."""
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).transpose(*range(a.ndim)[::-1]))).cuda()


def _host(t):
    return t.cpu().numpy().transpose(*range(t.ndim)[::-1])


def _setup():
    oc = O.OracleCase(GRID)
    oc.add_body(BODY)
    oc.set_iblank()
    oc.gcm(2.0, 2.0)
    c = fg.Case(GRID, fg.default_config())
    c.add_body(BODY)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    return oc, c


def _fields(rng):
    sh = GRID.shape
    NX, NY, NZ = sh
    u, v, w = (np.asfortranarray(synth.box_smooth(rng.standard_normal(sh))) for _ in range(3))
    bcxu = np.asfortranarray(0.1 * rng.standard_normal((2, NY, NZ)) + 1.0)
    bcyv = np.asfortranarray(0.1 * rng.standard_normal((NX, 2, NZ)))
    bczw = np.asfortranarray(0.1 * rng.standard_normal((NX, NY, 2)))
    return u, v, w, bcxu, bcyv, bczw


def _close(got, want, tol):
    scale = max(1e-300, float(np.abs(want).max()))
    return float(np.abs(got - want).max()) <= tol * scale


@pytest.mark.parametrize("vzg", [[0, 0, 0, 0, 0, 0], [0, 1, 0, 0, 0, 0], [0, 1, 0, 1, 0, 1]])
def test_face_vel_and_rhs_poisson_match_oracle(vzg):
    oc, c = _setup()
    rng = np.random.default_rng(2)
    u, v, w, bcxu, bcyv, bczw = _fields(rng)
    fo = oc.face_vel(u, v, w, bcxu, bcyv, bczw)
    d = {k: _dev(a) for k, a in dict(u=u, v=v, w=w, bcxu=bcxu, bcyv=bcyv, bczw=bczw).items()}
    fd = [torch.zeros_like(d["u"]) for _ in range(3)]
    fg.face_vel_device(c, d["u"].data_ptr(), d["v"].data_ptr(), d["w"].data_ptr(), d["bcxu"].data_ptr(),
                       d["bcyv"].data_ptr(), d["bczw"].data_ptr(), *[t.data_ptr() for t in fd])
    for a, t in zip(fo, fd):
        assert _close(_host(t), a, 1e-13)
    dt = 0.01
    bco = [bcxu.copy(order="F"), bcyv.copy(order="F"), bczw.copy(order="F")]
    fo2 = [a.copy(order="F") for a in fo]
    div_o, sd_o, rd_o = oc.rhs_poisson(*fo2, *bco, vzg, dt)
    div_d = torch.zeros_like(d["u"])
    sd_d, rd_d = fg.rhs_poisson_device(c, *[t.data_ptr() for t in fd], d["bcxu"].data_ptr(), d["bcyv"].data_ptr(),
                                       d["bczw"].data_ptr(), vzg, dt, div_d.data_ptr())
    assert _close(_host(div_d), div_o, 1e-12)
    for a, t in zip(fo2, fd):  # boundary face velocities corrected alike
        assert _close(_host(t), a, 1e-13)
    for a, k in zip(bco, ("bcxu", "bcyv", "bczw")):
        assert _close(_host(d[k]), a, 1e-13)
    assert abs(sd_d - sd_o) <= 1e-11 * max(1.0, abs(sd_o))
    assert abs(rd_d - rd_o) <= 1e-12 * rd_o
    if any(vzg):  # the correction leaves no net mass flux
        assert abs(sd_o) < 1e-10
    c.close()


def test_correct_vel_matches_oracle():
    oc, c = _setup()
    rng = np.random.default_rng(4)
    u, v, w, _, _, _ = _fields(rng)
    pp = np.asfortranarray(synth.box_smooth(rng.standard_normal(GRID.shape)))
    uo, vo, wo = u.copy(order="F"), v.copy(order="F"), w.copy(order="F")
    go = oc.correct_vel(pp, 0.02, uo, vo, wo)
    du, dv, dw, dpp = _dev(u), _dev(v), _dev(w), _dev(pp)
    g = [torch.zeros_like(du) for _ in range(3)]
    fg.correct_vel_device(c, dpp.data_ptr(), 0.02, du.data_ptr(), dv.data_ptr(), dw.data_ptr(),
                          *[t.data_ptr() for t in g])
    for a, t in zip((uo, vo, wo), (du, dv, dw)):
        assert _close(_host(t), a, 1e-13)
    for a, t in zip(go, g):
        assert _close(_host(t), a, 1e-13)
    c.close()


def test_time_step_stays_on_device():
    """face velocities -> div (with an outflow face made mass-conserving)
    -> the pressure solve on the device div -> corrected velocity, against
    the same chain through the oracle.  The outflow face carries p = 0
    (Dirichlet), which makes the pressure system nonsingular for any div."""
    oc, c = _setup()
    c.close()
    pbc = [fg.FG_PBC_NEUMANN] * 6
    pbc[1] = fg.FG_PBC_DIRICHLET
    c = fg.Case(GRID, fg.default_config(rtol=1e-12, max_cycles=200, pbc=pbc))
    c.add_body(BODY)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    rng = np.random.default_rng(9)
    u, v, w, bcxu, bcyv, bczw = _fields(rng)
    vzg = [0, 1, 0, 0, 0, 0]
    dt = 0.05
    # oracle chain
    fo = oc.face_vel(u, v, w, bcxu, bcyv, bczw)
    bco = [bcxu.copy(order="F"), bcyv.copy(order="F"), bczw.copy(order="F")]
    div_o, _, _ = oc.rhs_poisson(*fo, *bco, vzg, dt)
    po = np.zeros(GRID.shape, order="F")
    oc.solve_poisson(po, div_o, params=O.default_params(restol_pson=1e-14, restol_gcp=1e-14, itermax_pson=4000,
                                                        pbc=pbc))
    uo, vo, wo = u.copy(order="F"), v.copy(order="F"), w.copy(order="F")
    oc.correct_vel(po, dt, uo, vo, wo)
    # device chain
    d = {k: _dev(a) for k, a in dict(u=u, v=v, w=w, bcxu=bcxu, bcyv=bcyv, bczw=bczw).items()}
    fd = [torch.zeros_like(d["u"]) for _ in range(3)]
    fg.face_vel_device(c, d["u"].data_ptr(), d["v"].data_ptr(), d["w"].data_ptr(), d["bcxu"].data_ptr(),
                       d["bcyv"].data_ptr(), d["bczw"].data_ptr(), *[t.data_ptr() for t in fd])
    div_d = torch.zeros_like(d["u"])
    fg.rhs_poisson_device(c, *[t.data_ptr() for t in fd], d["bcxu"].data_ptr(), d["bcyv"].data_ptr(),
                          d["bczw"].data_ptr(), vzg, dt, div_d.data_ptr())
    p_d = torch.zeros_like(d["u"])
    st = c.solve_poisson_device(p_d.data_ptr(), div_d.data_ptr())
    assert st["relres"] <= 1e-12
    fg.correct_vel_device(c, p_d.data_ptr(), dt, d["u"].data_ptr(), d["v"].data_ptr(), d["w"].data_ptr())
    ib = oc.field(0)
    m = np.zeros(GRID.shape, bool)
    m[1:GRID.nx, 1:GRID.ny, 1:GRID.nz] = ib[1:GRID.nx, 1:GRID.ny, 1:GRID.nz] == 0
    for a, k in zip((uo, vo, wo), ("u", "v", "w")):
        h = _host(d[k])
        assert np.abs(h[m] - a[m]).max() <= 1e-8 * np.abs(a[m]).max()
    c.close()


def test_update_pressure_matches_oracle():
    """update_pressure zeroes p' on the solid cells that are not dead-marked
    -1 and on the domain edge lines, then copies it to p: bit for bit."""
    oc, c = _setup()
    rng = np.random.default_rng(6)
    pp = np.asfortranarray(rng.standard_normal(GRID.shape))
    assert (oc.field(2) == -1).any() and (oc.field(0) == 1).any()
    po = pp.copy(order="F")
    p_o = oc.update_pressure(po)
    d_pp = _dev(pp)
    d_p = torch.full_like(d_pp, 7.0)
    fg.update_pressure_device(c, d_pp.data_ptr(), d_p.data_ptr())
    assert np.array_equal(_host(d_pp), po)
    assert np.array_equal(_host(d_p), p_o)
    c.close()
