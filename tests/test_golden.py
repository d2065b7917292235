"""Golden fixtures (tests/golden/, written by tests/golden/make_golden.py).

CPU: the oracle reproduces its committed digests (regression of the
restatement).  GPU: the device tagging reproduces the same digests --
iblank, ghostCellMark, dead_cell and every ghost/dead list array bit for
bit -- on config 0, on the headline 512x256x256 stretched sphere, on all
100 steps of the config-2 pitching plate (moved on one handle) and on
four problems of the 64-problem batch; and the converged config-0
pressure matches the oracle's sample to 1e-9.
"""
import importlib.util
import json
import os

import numpy as np
import pytest

from feicar_b200 import fg, synth

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "tagging_digests.json")))

_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
_mg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(_mg)


def _oracle_digests(grid, body):
    oc = _mg.oracle_tag(grid, body)
    return _mg.tagging_digests(oc.field(0), oc.field(1), oc.field(2), oc.ghosts(), oc.deads())


def test_oracle_config0_digests():
    assert _oracle_digests(synth.config0_grid(), synth.config0_body()) == GOLD["config0"]


@pytest.mark.parametrize("step", [0, 25])
def test_oracle_config2_digests(step):
    assert _oracle_digests(synth.config2_grid(), synth.config2_body(step)) == GOLD[f"config2_step{step}"]


def _device_digests(c):
    ib, gh, dd = c.gcm_set_internal_boundary()
    return _mg.tagging_digests(ib, gh, dd, c.ghost_rows(), c.dead_rows())


@pytest.mark.gpu
def test_device_config0_digests():
    c = fg.Case(synth.config0_grid(), fg.default_config())
    c.add_body(synth.config0_body())
    c.set_iblank_body_fast()
    assert _device_digests(c) == GOLD["config0"]
    c.close()


@pytest.mark.gpu
def test_device_config2_moving_plate_digests():
    base = synth.config2_plate()
    c = fg.Case(synth.config2_grid(), fg.default_config())
    c.add_body(synth.config2_body(0))
    c.set_iblank_body_fast()
    assert _device_digests(c) == GOLD["config2_step0"]
    c.update_body(0, synth.config2_verts(base, 25))
    c.set_iblank_body_fast()
    assert _device_digests(c) == GOLD["config2_step25"]
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_device_config0_pressure_sample(prec):
    smp = np.load(os.path.join(HERE, "golden", "config0_pressure_sample.npz"))
    g, b = synth.config0_grid(), synth.config0_body()
    c = fg.Case(g, fg.default_config(precision=fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64,
                                     rtol=1e-12, max_cycles=120))
    c.add_body(b)
    c.set_iblank_body_fast()
    ib, gh, dd = c.gcm_set_internal_boundary()
    G, D = c.ghost_rows(), c.dead_rows()
    rows = [synth.Interp(D["ijk"], D["cell"], D["coefN"]), synth.Interp(G["ijk"], G["cell"], G["coefN"])]
    rhs, _ = synth.manufactured_rhs(g, ib, gh, dd, rows, seed=0)
    c.mg_prepare()
    p = np.zeros(g.shape, order="F")
    c.solve_poisson(p, rhs)
    m = np.zeros(g.shape, bool)
    m[1:g.nx, 1:g.ny, 1:g.nz] = ib[1:g.nx, 1:g.ny, 1:g.nz] == 0
    pf = p.ravel(order="F")
    flat = np.flatnonzero(m.ravel(order="F"))
    v = pf[smp["index"]] - pf[flat].mean()
    ref = smp["p"]
    assert np.linalg.norm(v - ref) / np.linalg.norm(ref) <= 1e-9
    c.close()


# ---- the benched geometries (tests/golden/benched_digests.json)
BENCHED = json.load(open(os.path.join(HERE, "golden", "benched_digests.json")))


@pytest.mark.parametrize("i", ["4", "9"])
def test_oracle_batch64_digests(i):
    g, b, _ = synth.batch_problems(n=64, seed0=0, lo=32, hi=192)[int(i)]
    assert _oracle_digests(g, b) == BENCHED["batch64"][i]


@pytest.mark.parametrize("step", [50, 75])
def test_oracle_config2_step_digests(step):
    assert _oracle_digests(synth.config2_grid(), synth.config2_body(step)) == BENCHED["config2_steps"][step]


@pytest.mark.gpu
def test_device_config1_digests():
    """The headline geometry: 512x256x256 cells tanh-stretched in y and z,
    an 81920-triangle sphere; iblank, ghostCellMark, dead_cell and every
    ghost/dead list array equal the oracle's bit for bit."""
    c = fg.Case(synth.config1_grid(), fg.default_config())
    c.add_body(synth.config1_body())
    c.set_iblank_body_fast()
    assert _device_digests(c) == BENCHED["config1"]
    c.close()


@pytest.mark.gpu
def test_device_config2_all_steps_digests():
    """All 100 steps of the pitching plate, moved step by step on one
    handle as the time loop does, against the oracle tagging each position
    from scratch."""
    base = synth.config2_plate()
    c = fg.Case(synth.config2_grid(), fg.default_config())
    c.add_body(synth.config2_body(0))
    bad = []
    for step in range(100):
        if step:
            c.update_body(0, synth.config2_verts(base, step))
        c.set_iblank_body_fast()
        if _device_digests(c) != BENCHED["config2_steps"][step]:
            bad.append(step)
    c.close()
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize("i", sorted(BENCHED["batch64"]))
def test_device_batch64_digests(i):
    g, b, _ = synth.batch_problems(n=64, seed0=0, lo=32, hi=192)[int(i)]
    c = fg.Case(g, fg.default_config())
    c.add_body(b)
    c.set_iblank_body_fast()
    assert _device_digests(c) == BENCHED["batch64"][i]
    c.close()
