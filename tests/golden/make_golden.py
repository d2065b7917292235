"""Writes the oracle's golden fixtures (run from the repository root):

    python tests/golden/make_golden.py          # everything
    python tests/golden/make_golden.py more     # benched_digests.json only

For config 0 (128x64x64, sphere) and config 2 (256x128x128, pitching
membrane plate) at steps 0 and 25: SHA-256 digests of iblank,
ghostCellMark and dead_cell and of every ghost/dead list array (exact
bytes, little-endian), plus row counts; for config 0 also a seeded sample
of 4096 fluid-cell values of the converged pressure (mean removed) for the
seed-0 manufactured RHS.  The reference ships no golden outputs; these
fixtures are regression anchors of the oracle and the device path.
"""
import hashlib
import importlib.util
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
PKG = os.path.join(ROOT, "feicar3d_3.0_febio_b200")
if "feicar_b200" not in sys.modules:
    spec = importlib.util.spec_from_file_location("feicar_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["feicar_b200"] = mod
    spec.loader.exec_module(mod)
from feicar_b200 import synth  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
GHOST_KEYS = ["ijk", "cell", "closest", "bi", "ip", "probe", "alpha", "coefN", "coefD"]
DEAD_KEYS = ["ijk", "cell", "closest", "bi", "ip", "probe", "coefN", "coefD"]


def digest(a):
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes()).hexdigest()


def tagging_digests(ib, gh, dd, G, D):
    return {
        "iblank": digest(ib), "ghostCellMark": digest(gh), "dead_cell": digest(dd),
        "nGhost": int(len(G["ijk"])), "nDead": int(len(D["ijk"])),
        "ghost": {k: digest(G[k]) for k in GHOST_KEYS},
        "dead": {k: digest(D[k]) for k in DEAD_KEYS},
    }


def oracle_tag(grid, body):
    oc = O.OracleCase(grid)
    oc.add_body(body)
    oc.set_iblank()
    rc = oc.gcm(2.0, 2.0)
    assert rc == 0, rc
    return oc


def main():
    gold = {}
    g0, b0 = synth.config0_grid(), synth.config0_body()
    oc = oracle_tag(g0, b0)
    G, D = oc.ghosts(), oc.deads()
    ib, gh, dd = oc.field(0), oc.field(1), oc.field(2)
    gold["config0"] = tagging_digests(ib, gh, dd, G, D)
    rows = [synth.Interp(D["ijk"], D["cell"], D["coefN"]), synth.Interp(G["ijk"], G["cell"], G["coefN"])]
    rhs, phi = synth.manufactured_rhs(g0, ib, gh, dd, rows, seed=0)
    p = np.zeros(g0.shape, order="F")
    rc, st = oc.solve_poisson(p, rhs, params=O.default_params(restol_pson=1e-13, restol_gcp=1e-13,
                                                               itermax_pson=400))
    m = np.zeros(g0.shape, bool)
    m[1:g0.nx, 1:g0.ny, 1:g0.nz] = ib[1:g0.nx, 1:g0.ny, 1:g0.nz] == 0
    flat = np.flatnonzero(m.ravel(order="F"))
    pick = np.sort(np.random.default_rng(123).choice(flat, 4096, replace=False))
    pf = p.ravel(order="F")
    pv = pf[pick] - pf[flat].mean()
    np.savez_compressed(os.path.join(OUT, "config0_pressure_sample.npz"), index=pick, p=pv,
                        relres=np.array([st["relres"]]))
    for step in (0, 25):
        oc2 = oracle_tag(synth.config2_grid(), synth.config2_body(step))
        gold[f"config2_step{step}"] = tagging_digests(oc2.field(0), oc2.field(1), oc2.field(2),
                                                      oc2.ghosts(), oc2.deads())
    with open(os.path.join(OUT, "tagging_digests.json"), "w") as f:
        json.dump(gold, f, indent=1, sort_keys=True)
    print(json.dumps({k: (v["nGhost"], v["nDead"]) for k, v in gold.items()}))
    more_goldens()


# problems of the 64-problem batch whose tagging is pinned (edges 32, 35,
# 45 and 81 cells)
BATCH_PICK = (4, 9, 3, 0)


def more_goldens():
    """Digests of the benched geometries: config 1 (512x256x256 stretched,
    81920-triangle sphere), all 100 steps of the config-2 pitching plate
    (each tagged from scratch at its position), and four problems of the
    64-problem batch."""
    gold = {}
    oc = oracle_tag(synth.config1_grid(), synth.config1_body())
    gold["config1"] = tagging_digests(oc.field(0), oc.field(1), oc.field(2), oc.ghosts(), oc.deads())
    del oc
    steps = []
    for step in range(100):
        oc2 = oracle_tag(synth.config2_grid(), synth.config2_body(step))
        steps.append(tagging_digests(oc2.field(0), oc2.field(1), oc2.field(2), oc2.ghosts(), oc2.deads()))
    gold["config2_steps"] = steps
    probs = synth.batch_problems(n=64, seed0=0, lo=32, hi=192)
    gold["batch64"] = {}
    for i in BATCH_PICK:
        g, b, _ = probs[i]
        ocb = oracle_tag(g, b)
        gold["batch64"][str(i)] = tagging_digests(ocb.field(0), ocb.field(1), ocb.field(2), ocb.ghosts(),
                                                  ocb.deads())
    with open(os.path.join(OUT, "benched_digests.json"), "w") as f:
        json.dump(gold, f, indent=1, sort_keys=True)
    print(json.dumps({"config1": (gold["config1"]["nGhost"], gold["config1"]["nDead"]),
                      "batch64": {k: (v["nGhost"], v["nDead"]) for k, v in gold["batch64"].items()}}))


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "more":
    more_goldens()
    sys.exit(0)


if __name__ == "__main__":
    main()
