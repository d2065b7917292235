"""bench.py's CPU baseline and reference arm: one measured solve of the
oracle from the zero initial guess, to the tolerance or to a time budget
(then reported as an upper bound, never extrapolated), with the same rule
in the main line's cpu_baseline and in ``--impl reference``."""
import importlib.util
import io
import json
import os
import types
from contextlib import redirect_stdout

import numpy as np

from feicar_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
_spec = importlib.util.spec_from_file_location("fg_bench", os.path.join(HERE, "..", "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def _tiny():
    grid = synth.small_grid(16, 8, 8, (4.0, 2.0, 2.0))
    body = synth.sphere_body((1.0, 1.0, 1.0), 1.0, 2)
    O = bench._oracle()
    oc = O.OracleCase(grid)
    oc.add_body(body)
    oc.set_iblank()
    oc.gcm(2.0, 2.0)
    G, D = oc.ghosts(), oc.deads()
    rows = [synth.Interp(D["ijk"], D["cell"], D["coefN"]), synth.Interp(G["ijk"], G["cell"], G["coefN"])]
    rhs, _ = synth.manufactured_rhs(grid, oc.field(0), oc.field(1), oc.field(2), rows, seed=0)
    return grid, body, rhs


def test_measured_solve_converges_and_is_timed():
    grid, body, rhs = _tiny()
    out = bench.cpu_measured_solve(grid, body, rhs, budget_s=60.0, warm_iters=0)
    assert out["converged"] and not out["value_is_upper_bound"]
    assert out["relres_last"] <= bench.RTOL
    assert np.isclose(out["value"], 1.0 / out["seconds"])
    assert "extrapolat" not in out["sample"]


def test_budget_gives_an_upper_bound_not_an_estimate():
    grid, body, rhs = _tiny()
    out = bench.cpu_measured_solve(grid, body, rhs, budget_s=0.0, warm_iters=0)
    assert out["iterations"] == 1
    assert not out["converged"] and out["value_is_upper_bound"]
    assert out["relres_last"] > bench.RTOL
    assert np.isclose(out["value"], 1.0 / out["seconds"])


def test_reference_arm_line(monkeypatch):
    grid, body, _ = _tiny()
    monkeypatch.setattr(bench, "workload", lambda name: (grid, body, "tiny"))
    args = types.SimpleNamespace(workload="tiny", steps=5, warmup=3, cpu_budget_s=60.0)
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    line = json.loads(buf.getvalue().strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["cpu_baseline"]["converged"]
    assert line["value"] == line["cpu_baseline"]["value"] == line["e2e"]["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["value"] > 0
