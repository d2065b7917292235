"""Pressure-Poisson solve on the device against the oracle.

The right-hand side is manufactured: f = A phi for a smooth random potential
phi, with A the reference operator (7-point stencil on fluid cells, the
ghost rows of GCM_SET_BOUNDARY.F90:521-537 and dead rows of :1451-1489 with
homogeneous Neumann data).  The discrete solution is phi up to a constant,
so the converged pressure of the device path is compared with phi and with
the oracle's own converged solve_poisson (CORE_POISSON.F90:83-200).

Tolerances: FP64 and mixed paths within 1e-9 relative L2 (mean removed,
fluid cells) of the exact discrete solution when run to rtol 1e-12.
"""
import numpy as np
import pytest
import torch

from feicar_b200 import fg, synth
import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _fluid(grid, ib):
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    m = np.zeros(grid.shape, bool)
    m[1:nx, 1:ny, 1:nz] = ib[1:nx, 1:ny, 1:nz] == 0
    return m


def _relerr(p, ref, mask):
    a = p[mask] - p[mask].mean()
    b = ref[mask] - ref[mask].mean()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _problem(grid, bodies, seed=0):
    """Device case tagged on the GPU, RHS from the oracle's rows."""
    if not bodies:
        z = np.zeros(grid.shape, np.int8, order="F")
        rhs, phi = synth.manufactured_rhs(grid, z, z, z, [], seed=seed)
        return None, z, rhs, phi
    oc = O.OracleCase(grid)
    for b in bodies:
        oc.add_body(b)
    oc.set_iblank()
    oc.gcm(2.0, 2.0)
    G, D = oc.ghosts(), oc.deads()
    rows = [synth.Interp(D["ijk"], D["cell"], D["coefN"]), synth.Interp(G["ijk"], G["cell"], G["coefN"])]
    ib, gh, dd = oc.field(0), oc.field(1), oc.field(2)
    rhs, phi = synth.manufactured_rhs(grid, ib, gh, dd, rows, seed=seed)
    return oc, ib, rhs, phi


def _case(grid, bodies, **kw):
    cfg = fg.default_config(**kw)
    c = fg.Case(grid, cfg)
    if bodies:
        for b in bodies:
            c.add_body(b)
        c.set_iblank_body_fast()
        c.gcm_set_internal_boundary()
    else:
        z = np.zeros(grid.shape, np.int8, order="F")
        e3 = np.zeros((0, 3), np.int32)
        c.set_geometry(z, z, z, dict(ijk=e3, cell=e3, coefN=np.zeros((0, 8))),
                       dict(ijk=e3, cell=e3, coefN=np.zeros((0, 8)), probe=np.zeros(0),
                            ip=np.zeros((0, 3))))
    c.mg_prepare()
    return c


def _grids():
    return {
        "sphere_small": (synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0)),
                         [synth.sphere_body((1.0, 1.0, 1.0), 1.0, 3)]),
        "sphere_stretched": (synth.Grid(synth.uniform_nodes(64, 0, 4), synth.tanh_nodes(32, 0, 2, 2.0),
                                        synth.tanh_nodes(32, 0, 2, 2.0)),
                             [synth.sphere_body((1.0, 1.0, 1.0), 1.0, 4)]),
        "two_spheres": (synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0)),
                        [synth.sphere_body((1.0, 1.0, 1.0), 0.8, 3),
                         synth.sphere_body((2.6, 0.9, 1.1), 0.7, 3)]),
        "ragged_no_body": (synth.Grid(synth.uniform_nodes(37, 0, 1.3), synth.uniform_nodes(23, 0, 0.9),
                                      synth.tanh_nodes(19, 0, 0.7, 1.5)), []),
        "config0": (synth.config0_grid(), [synth.config0_body()]),
    }


GRIDS = _grids()


@pytest.mark.parametrize("outer", ["fgmres", "richardson"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(GRIDS))
def test_converges_to_discrete_solution(name, prec, outer):
    grid, bodies = GRIDS[name]
    _, ib, rhs, phi = _problem(grid, bodies)
    p_ = fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64
    o_ = fg.FG_OUTER_FGMRES if outer == "fgmres" else fg.FG_OUTER_RICHARDSON
    c = _case(grid, bodies, precision=p_, outer=o_, rtol=1e-12, max_cycles=120)
    p = np.zeros(grid.shape, order="F")
    st = c.solve_poisson(p, rhs)
    assert st["relres"] <= 1e-12
    err = _relerr(p, phi, _fluid(grid, ib))
    assert err <= TOL, (name, prec, err, st)
    c.close()


@pytest.mark.parametrize("name", ["sphere_small", "two_spheres"])
def test_matches_oracle_solve(name):
    grid, bodies = GRIDS[name]
    oc, ib, rhs, phi = _problem(grid, bodies)
    po = np.zeros(grid.shape, order="F")
    rc, ost = oc.solve_poisson(po, rhs.copy(order="F"),
                               params=O.default_params(restol_pson=1e-13, restol_gcp=1e-13, itermax_pson=400))
    c = _case(grid, bodies, rtol=1e-12, max_cycles=120)
    p = np.zeros(grid.shape, order="F")
    c.solve_poisson(p, rhs)
    m = _fluid(grid, ib)
    assert _relerr(po, phi, m) <= TOL, ost
    assert _relerr(p, po, m) <= TOL
    c.close()


def test_device_entry_matches_host_entry():
    grid, bodies = GRIDS["sphere_stretched"]
    _, ib, rhs, phi = _problem(grid, bodies)
    c = _case(grid, bodies, rtol=1e-10, max_cycles=60)
    p = np.zeros(grid.shape, order="F")
    st_h = c.solve_poisson(p, rhs)
    # Fortran (i fastest) layout == C layout of the reversed shape
    rev = grid.shape[::-1]
    d_p = torch.zeros(rev, dtype=torch.float64, device="cuda")
    d_f = torch.from_numpy(np.ascontiguousarray(rhs.transpose(2, 1, 0))).cuda()
    st_d = c.solve_poisson_device(d_p.data_ptr(), d_f.data_ptr())
    torch.cuda.synchronize()
    pd = d_p.cpu().numpy().transpose(2, 1, 0)
    assert st_d["cycles"] == st_h["cycles"]
    # same kernels, same gauge and outer boundary layers: identical fields
    assert np.array_equal(pd, p)
    c.close()


def test_batch_matches_solo():
    probs = synth.batch_problems(n=3, seed0=5, lo=24, hi=48)
    cases, rhss, solo = [], [], []
    for g, b, s in probs:
        _, ib, rhs, phi = _problem(g, [b], seed=s)
        c = _case(g, [b], rtol=1e-11, max_cycles=80)
        p = np.zeros(g.shape, order="F")
        c.solve_poisson(p, rhs)
        solo.append((p, _fluid(g, ib)))
        cases.append(c)
        rhss.append(rhs)
    bt = fg.Batch(fg.default_config(rtol=1e-11, max_cycles=80))
    for c in cases:
        bt.add(c)
    d_ps, d_fs = [], []
    for (g, _, _), rhs in zip(probs, rhss):
        d_ps.append(torch.zeros(g.shape[::-1], dtype=torch.float64, device="cuda"))
        d_fs.append(torch.from_numpy(np.ascontiguousarray(rhs.transpose(2, 1, 0))).cuda())
    bt.solve_device([t.data_ptr() for t in d_ps], [t.data_ptr() for t in d_fs])
    torch.cuda.synchronize()
    for (p, m), t in zip(solo, d_ps):
        pb = t.cpu().numpy().transpose(2, 1, 0)
        assert _relerr(pb, p, m) <= 1e-10
    bt.close()
    for c in cases:
        c.close()


def test_warm_start_reaches_same_solution():
    """A second solve started from the converged pressure (the next time
    step's initial guess in CORE_POISSON.F90) needs at most one cycle."""
    grid, bodies = GRIDS["sphere_small"]
    _, ib, rhs, phi = _problem(grid, bodies)
    c = _case(grid, bodies, rtol=1e-10, max_cycles=60)
    p = np.zeros(grid.shape, order="F")
    c.solve_poisson(p, rhs)
    st2 = c.solve_poisson(p, rhs)
    assert st2["cycles"] <= 1
    assert _relerr(p, phi, _fluid(grid, ib)) <= 1e-8
    c.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_graph_replay_matches_direct_launches(prec):
    """The whole FGMRES solve is captured once as a CUDA graph (its restart
    and inner loops as conditional nodes decided on the device) and
    replayed as one launch; with launch-class timing on, the host drives
    the same kernels step by step.  Same kernels in the same order: the two
    solves give identical fields and histories, and the launch counter
    counts the kernels the graph ran."""
    grid, bodies = GRIDS["sphere_stretched"]
    _, ib, rhs, phi = _problem(grid, bodies)
    p_ = fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64
    c = _case(grid, bodies, precision=p_, rtol=1e-10, max_cycles=60)
    p_graph = np.zeros(grid.shape, order="F")
    c.solve_poisson(p_graph, rhs)  # captures
    assert c.solve_mode() == 1
    p_graph[...] = 0.0
    n0 = fg.launch_count()
    st_g = c.solve_poisson(p_graph, rhs)  # replays
    n_graph = fg.launch_count() - n0
    h_graph = c.history()
    assert c.solve_mode() == 1
    c.profile(True)
    p_direct = np.zeros(grid.shape, order="F")
    n0 = fg.launch_count()
    st_d = c.solve_poisson(p_direct, rhs)
    n_direct = fg.launch_count() - n0
    assert c.solve_mode() == 0
    c.profile(False)
    assert st_g["cycles"] == st_d["cycles"]
    assert np.array_equal(h_graph, c.history())
    assert np.array_equal(p_graph, p_direct)
    assert n_graph == n_direct
    assert _relerr(p_graph, phi, _fluid(grid, ib)) <= 1e-8
    c.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_moved_body_matches_fresh_case(prec):
    """A body moved on a live case (update_body, re-tag, prepare) keeps the
    case's level tables and V-cycle graph and only replaces its rows and
    coarsest inverse; the solve must equal that of a case built directly
    at the new position, field for field."""
    grid = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0))
    b0 = synth.sphere_body((1.0, 1.0, 1.0), 0.8, 3)
    b1 = synth.sphere_body((1.4, 0.95, 1.05), 0.8, 3)
    p_ = fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64
    _, ib0, rhs0, _ = _problem(grid, [b0], seed=1)
    _, ib1, rhs1, phi1 = _problem(grid, [b1], seed=2)
    live = _case(grid, [b0], precision=p_, rtol=1e-10, max_cycles=60)
    p = np.zeros(grid.shape, order="F")
    live.solve_poisson(p, rhs0)
    live.update_body(0, b1.verts)
    live.set_iblank_body_fast()
    live.gcm_set_internal_boundary()
    live.mg_prepare()
    p_live = np.zeros(grid.shape, order="F")
    st_live = live.solve_poisson(p_live, rhs1)
    live.close()
    fresh = _case(grid, [b1], precision=p_, rtol=1e-10, max_cycles=60)
    p_fresh = np.zeros(grid.shape, order="F")
    st_fresh = fresh.solve_poisson(p_fresh, rhs1)
    fresh.close()
    assert st_live["cycles"] == st_fresh["cycles"]
    assert np.array_equal(p_live, p_fresh)
    assert _relerr(p_fresh, phi1, _fluid(grid, ib1)) <= 1e-8


def test_reused_device_blocks_give_identical_solves():
    """Device memory freed by a closed case is handed to the next one
    without being cleared; a case made again after another of a different
    size must solve exactly as the first time."""
    grid, bodies = GRIDS["sphere_small"]
    _, _, rhs, _ = _problem(grid, bodies)
    g2, b2 = GRIDS["two_spheres"]
    _, _, rhs2, _ = _problem(g2, b2, seed=3)
    runs = []
    for _ in range(2):
        c = _case(grid, bodies, precision=fg.FG_PREC_MIXED, rtol=1e-10, max_cycles=60)
        p = np.zeros(grid.shape, order="F")
        st = c.solve_poisson(p, rhs)
        c.close()
        runs.append((st["cycles"], p))
        o = _case(g2, b2, precision=fg.FG_PREC_MIXED, rtol=1e-10, max_cycles=60)
        o.solve_poisson(np.zeros(g2.shape, order="F"), rhs2)
        o.close()
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1])


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_batch64_problems_each_reach_their_solution(prec):
    """Four problems of the 64-problem batched workload (edges 32, 35, 45
    and 81 cells, seeded 5120-triangle ellipsoids), solved together by one
    batch: each pressure within 1e-9 of its own exact discrete solution
    (manufactured from the oracle's rows), not of another solve."""
    allp = synth.batch_problems(n=64, seed0=0, lo=32, hi=192)
    p_ = fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64
    cfg = fg.default_config(precision=p_, rtol=1e-12, max_cycles=120)
    cases, refs, d_ps, d_fs = [], [], [], []
    for i in (4, 9, 3, 0):
        g, b, seed = allp[i]
        _, ib, rhs, phi = _problem(g, [b], seed=seed)
        c = fg.Case(g, cfg)
        c.add_body(b)
        c.set_iblank_body_fast()
        c.gcm_set_internal_boundary()
        c.mg_prepare()
        cases.append(c)
        refs.append((g, phi, _fluid(g, ib)))
        d_ps.append(torch.zeros(g.shape[::-1], dtype=torch.float64, device="cuda"))
        d_fs.append(torch.from_numpy(np.ascontiguousarray(rhs.transpose(2, 1, 0))).cuda())
    bt = fg.Batch(cfg)
    for c in cases:
        bt.add(c)
    st = bt.solve_device([t.data_ptr() for t in d_ps], [t.data_ptr() for t in d_fs])
    torch.cuda.synchronize()
    assert st["relres"] <= 1e-12
    for (g, phi, m), t in zip(refs, d_ps):
        p = t.cpu().numpy().transpose(2, 1, 0)
        assert _relerr(p, phi, m) <= TOL
    bt.close()
    for c in cases:
        c.close()


def test_line_sor_solver_reaches_the_same_solution():
    """The reference's single-grid solver type 1 (line SOR on the fine
    grid, CORE_POISSON.F90:205-456): on the device it converges to the
    same discrete solution as the multigrid path and as the oracle's own
    line-SOR solve."""
    grid, bodies = GRIDS["sphere_small"]
    oc, ib, rhs, phi = _problem(grid, bodies)
    m = _fluid(grid, ib)
    c = _case(grid, bodies, outer=fg.FG_OUTER_LSOR, omega=1.6, rtol=1e-11, max_cycles=40000)
    p = np.zeros(grid.shape, order="F")
    st = c.solve_poisson(p, rhs)
    assert st["relres"] <= 1e-11
    assert _relerr(p, phi, m) <= 1e-8
    po = np.zeros(grid.shape, order="F")
    oc.solve_poisson(po, rhs.copy(order="F"), params=O.default_params(
        lsor=True, omega_pson=1.6, restol_pson=1e-13, restol_gcp=1e-13, itermax_pson=40000))
    assert _relerr(p, po, m) <= 1e-8
    c.close()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_autotuned_batch_reaches_each_solution(prec):
    """The autotuner measures the line-kernel families of every level set
    and the (nu1, nu2) candidates on the batch itself and keeps the
    fastest; the tuned batch still solves each problem to its own exact
    discrete solution."""
    allp = synth.batch_problems(n=64, seed0=0, lo=32, hi=192)
    p_ = fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64
    cfg = fg.default_config(precision=p_, rtol=1e-12, max_cycles=120)
    cases, refs, d_ps, d_fs = [], [], [], []
    for i in (4, 9, 0):
        g, b, seed = allp[i]
        _, ib, rhs, phi = _problem(g, [b], seed=seed)
        c = fg.Case(g, cfg)
        c.add_body(b)
        c.set_iblank_body_fast()
        c.gcm_set_internal_boundary()
        c.mg_prepare()
        cases.append(c)
        refs.append((phi, _fluid(g, ib)))
        d_ps.append(torch.zeros(g.shape[::-1], dtype=torch.float64, device="cuda"))
        d_fs.append(torch.from_numpy(np.ascontiguousarray(rhs.transpose(2, 1, 0))).cuda())
    bt = fg.Batch(cfg)
    for c in cases:
        bt.add(c)
    tun = fg.batch_autotune(bt, [t.data_ptr() for t in d_ps], [t.data_ptr() for t in d_fs])
    assert tun["tuned"] and (tun["nu1"], tun["nu2"]) in [(1, 1), (2, 1), (2, 2), (3, 3)]
    assert tun["levels"][0]["x"]["us"] > 0
    for t in d_ps:
        t.zero_()
    st = bt.solve_device([t.data_ptr() for t in d_ps], [t.data_ptr() for t in d_fs])
    torch.cuda.synchronize()
    assert st["relres"] <= 1e-12
    for (phi, m), t in zip(refs, d_ps):
        assert _relerr(t.cpu().numpy().transpose(2, 1, 0), phi, m) <= TOL
    bt.close()
    for c in cases:
        c.close()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("fam", [(1, 1), (2, 2), (3, 3), (3, 4), (3, 5), (1, 4), (2, 5), (3, 6), (1, 6)])
def test_every_line_family_reaches_the_solution(prec, fam):
    """Each line-kernel family the autotuner may pick, forced on every
    level (a family that cannot take a level's lines falls back to the
    default there), solves to the exact discrete solution: the families
    differ only in how a line's tridiagonal system is split over threads."""
    grid = synth.small_grid(128, 96, 80, (4.0, 3.0, 2.5), stretch=1.5)
    body = synth.sphere_body((1.7, 1.4, 1.2), 0.9, 3)
    _, ib, rhs, phi = _problem(grid, [body], seed=11)
    p_ = fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64
    c = fg.Case(grid, fg.default_config(precision=p_, rtol=1e-12, max_cycles=150))
    c.add_body(body)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    fg.case_set_tuning(c, {"x": fam[0], "y": fam[1], "z": fam[1]}, nu=(2, 1))
    d_p = torch.zeros(grid.shape[::-1], dtype=torch.float64, device="cuda")
    d_f = torch.from_numpy(np.ascontiguousarray(rhs.transpose(2, 1, 0))).cuda()
    st = c.solve_poisson_device(d_p.data_ptr(), d_f.data_ptr())
    assert st["relres"] <= 1e-12
    assert _relerr(d_p.cpu().numpy().transpose(2, 1, 0), phi, _fluid(grid, ib)) <= TOL
    c.close()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("cfrom", [2, 1])
def test_coarse_level_smoothing_steps_reach_the_solution(prec, cfrom):
    """V(2,1) on the finest levels and V(1,1) from level cfrom down (the
    autotuner's coarse candidates) solves to the exact discrete solution."""
    grid = synth.small_grid(128, 96, 80, (4.0, 3.0, 2.5), stretch=1.5)
    body = synth.sphere_body((1.7, 1.4, 1.2), 0.9, 3)
    _, ib, rhs, phi = _problem(grid, [body], seed=12)
    p_ = fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64
    c = fg.Case(grid, fg.default_config(precision=p_, rtol=1e-12, max_cycles=150))
    c.add_body(body)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    fg.case_set_tuning(c, {}, nu=(2, 1), nu_coarse=(1, 1), coarse_from=cfrom)
    d_p = torch.zeros(grid.shape[::-1], dtype=torch.float64, device="cuda")
    d_f = torch.from_numpy(np.ascontiguousarray(rhs.transpose(2, 1, 0))).cuda()
    st = c.solve_poisson_device(d_p.data_ptr(), d_f.data_ptr())
    assert st["relres"] <= 1e-12
    assert _relerr(d_p.cpu().numpy().transpose(2, 1, 0), phi, _fluid(grid, ib)) <= TOL
    c.close()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_both_colour_sweep_equals_two_launches(prec):
    """The both-colour y/z sweep (one launch, plane-ordered tickets) runs
    the tile of the two colour launches of the block-PCR family on the same
    values (its colour-1 tiles read x from L2, where the colour-0 tiles of
    the launch left it), so whole solves take the same cycles and agree to
    rounding: the two kernels are compiled separately, and the compiler may
    contract a multiply-add in one and not in the other.  In FP64 the two
    solutions agree to 1e-11; the FP32 V-cycles of the mixed path carry
    that rounding into the Krylov iterates, so there the two converged
    solutions agree to the solve's own accuracy (1e-9)."""
    grid = synth.small_grid(96, 80, 72, (4.0, 3.0, 2.5), stretch=1.5)
    body = synth.sphere_body((1.7, 1.4, 1.2), 0.9, 3)
    _, ib, rhs, phi = _problem(grid, [body], seed=12)
    p_ = fg.FG_PREC_MIXED if prec == "mixed" else fg.FG_PREC_FP64
    c = fg.Case(grid, fg.default_config(precision=p_, rtol=1e-12, max_cycles=150))
    c.add_body(body)
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    d_f = torch.from_numpy(np.ascontiguousarray(rhs.transpose(2, 1, 0))).cuda()
    out = []
    for fam in (2, 6, 2):
        fg.case_set_tuning(c, {"x": 3, "y": fam, "z": fam}, nu=(2, 1))
        d_p = torch.zeros(grid.shape[::-1], dtype=torch.float64, device="cuda")
        st = c.solve_poisson_device(d_p.data_ptr(), d_f.data_ptr())
        out.append((d_p.cpu().numpy(), st["cycles"]))
    assert out[0][1] == out[1][1] == out[2][1]
    assert np.array_equal(out[0][0], out[2][0])  # the solve itself is deterministic
    # the all-Neumann solution is fixed up to a constant: compare the fluid
    # cells without it (solid cells keep values the solve does not define)
    m = _fluid(grid, ib)
    a = out[0][0].transpose(2, 1, 0)
    b = out[1][0].transpose(2, 1, 0)
    assert _relerr(b, a, m) <= (1e-9 if prec == "mixed" else 1e-11)
    assert _relerr(out[1][0].transpose(2, 1, 0), phi, _fluid(grid, ib)) <= TOL
    c.close()
