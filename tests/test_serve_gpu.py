"""The serving engine (fg_server_*): continuous admission of solve requests
and overlapped steps.

Each request is a problem (grid, body) with a run of time steps, as the
reference's time loop calls solve_poisson once per step with the pressure
kept between steps (CORE_TIME_STEP.F90:171-178).  The tests check that

* a request's results are the same whether it runs alone or in a mix of
  requests arriving while others are on the device (bit for bit: every
  case has its own stream, buffers and graph; nothing is shared);
* the mix really overlapped (several cases resident at once);
* a request served equals the same steps through the plain case API, and
  reaches the exact discrete solution of its manufactured right-hand side
  within 1e-9 (rtol 1e-12);
* admission respects the memory budget, and a request larger than the
  budget is rejected.
"""
import time

import numpy as np
import pytest

from feicar_b200 import fg, synth

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _templates():
    """Five small problems of the serving shapes: edges 24..40 cells, aspect
    1:1:1 or 2:1:1, sphere or rotated ellipsoid."""
    out = []
    rng = np.random.default_rng(21)
    for i, (edge, a) in enumerate([(24, 1), (32, 2), (28, 1), (40, 1), (24, 2)]):
        g = synth.Grid(synth.uniform_nodes(a * edge, 0, float(a)), synth.uniform_nodes(edge, 0, 1.0),
                       synth.uniform_nodes(edge, 0, 1.0))
        if i % 2 == 0:
            b = synth.sphere_body((0.5, 0.5, 0.5), rng.uniform(0.3, 0.5), 3)
        else:
            b = synth.ellipsoid_body((0.5, 0.5, 0.5), rng.uniform(0.15, 0.3, size=3),
                                     synth.random_rotation(rng), 3)
        out.append((g, b))
    return out


def _rhs_steps(g, b, nsteps, seed):
    c = fg.Case(g, fg.default_config())
    c.add_body(b)
    c.set_iblank_body_fast()
    ib, gh, dd = c.gcm_set_internal_boundary()
    G, D = c.ghost_rows(), c.dead_rows()
    c.close()
    rows = [synth.Interp(D["ijk"], D["cell"], D["coefN"]), synth.Interp(G["ijk"], G["cell"], G["coefN"])]
    out = []
    for s in range(nsteps):
        rhs, phi = synth.manufactured_rhs(g, ib, gh, dd, rows, seed=seed + s)
        out.append((np.asfortranarray(rhs), phi))
    m = np.zeros(g.shape, bool)
    m[1:g.nx, 1:g.ny, 1:g.nz] = ib[1:g.nx, 1:g.ny, 1:g.nz] == 0
    return out, m


PROBS = None


def _probs():
    global PROBS
    if PROBS is None:
        PROBS = []
        for i, (g, b) in enumerate(_templates()):
            steps, m = _rhs_steps(g, b, 2 + i % 3, seed=100 * i)
            PROBS.append((g, b, steps, m))
    return PROBS


def _cfg():
    return fg.default_config(precision=fg.FG_PREC_MIXED, rtol=1e-12, max_cycles=120)


def _run(server, order, delays=None):
    outs = {}
    for n, i in enumerate(order):
        g, b, steps, _ = _probs()[i]
        outs[i] = [np.zeros(g.shape, order="F") for _ in steps]
        server.submit(i, g, b, [s[0] for s in steps], outs[i])
        if delays is not None:
            time.sleep(delays[n])
    server.wait_idle(300.0)
    res = {r["id"]: r for r in server.poll()}
    return outs, res


def test_alone_equals_mixed_and_mix_overlaps():
    alone = {}
    for i in range(len(_probs())):
        s = fg.Server(_cfg(), max_active=1)
        outs, res = _run(s, [i])
        assert res[i]["status"] == fg.FG_OK and res[i]["steps_done"] == len(outs[i])
        alone[i] = outs[i]
        s.close()
    s = fg.Server(_cfg(), max_active=4)
    order = [3, 0, 4, 1, 2]
    outs, res = _run(s, order, delays=[0.0, 0.002, 0.0, 0.004, 0.0])
    info = s.info()
    s.close()
    assert info["active_peak"] > 1  # requests were resident together
    for i in order:
        assert res[i]["status"] == fg.FG_OK
        for a, m in zip(alone[i], outs[i]):
            assert np.array_equal(a, m)


def test_served_steps_match_case_api_and_exact_solution():
    g, b, steps, m = _probs()[1]
    s = fg.Server(_cfg(), max_active=2)
    outs, res = _run(s, [1])
    s.close()
    c = fg.Case(g, _cfg())
    c.add_body(b)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    p = np.zeros(g.shape, order="F")
    for (rhs, phi), o in zip(steps, outs[1]):
        c.solve_poisson(p, rhs)  # warm start from the previous step, as the server
        assert np.array_equal(p, o)
        a = o[m] - o[m].mean()
        e = phi[m] - phi[m].mean()
        assert np.linalg.norm(a - e) / np.linalg.norm(e) <= TOL
    c.close()


def test_budget_admission_and_rejection():
    probs = _probs()
    need = [fg.estimate_bytes(g, _cfg()) for g, _, _, _ in probs]
    # room for the largest request but not for two
    s = fg.Server(_cfg(), budget_bytes=max(need) + min(need) // 2, max_active=4)
    outs, res = _run(s, list(range(len(probs))))
    info = s.info()
    assert info["active_peak"] == 1 and info["finished"] == len(probs)
    assert all(r["status"] == fg.FG_OK for r in res.values())
    g, b, steps, _ = probs[3]
    with pytest.raises(fg.FGError) as e:
        tiny = fg.Server(_cfg(), budget_bytes=need[3] // 2, max_active=4)
        try:
            tiny.submit(99, g, b, [steps[0][0]])
        finally:
            tiny.close()
    assert e.value.status == 9  # FG_REJECTED
    s.close()
