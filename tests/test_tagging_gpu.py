"""Immersed-boundary tagging on the device against the oracle.

The device path (fg_set_iblank_body_fast + fg_gcm_set_internal_boundary)
follows BOUNDARY_IBLANK_FAST.F90:2-854 and GCM_SET_BOUNDARY.F90:2-1697;
it is compiled without FMA contraction, so every output is compared bit for
bit: iblank, ghostCellMark and dead_cell fields, the ghost and dead lists in
(k,j,i) order, host cells, closest elements, body intercepts, image points,
probe lengths, alphaGhost and both 8-point weight sets.
"""
import math

import numpy as np
import pytest

from feicar_b200 import fg, synth
import oracle as O

pytestmark = pytest.mark.gpu

GHOST_KEYS = ["ijk", "cell", "closest", "bi", "ip", "probe", "alpha", "coefN", "coefD"]
DEAD_KEYS = ["ijk", "cell", "closest", "bi", "ip", "probe", "coefN", "coefD"]


def _plate(grid_h, pivot, angle):
    b = synth.plate_body(n=24, size=1.0, tkns_factor=1.0, grid_h=grid_h)
    b.verts = synth.pitch_plate(b, pivot, angle)
    return b


def _cases():
    rng = np.random.default_rng(7)
    g_small = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0))
    g_str = synth.Grid(synth.uniform_nodes(64, 0, 4), synth.tanh_nodes(32, 0, 2, 2.0),
                       synth.tanh_nodes(32, 0, 2, 2.0))
    g_cube = synth.Grid(synth.uniform_nodes(48, 0, 1), synth.uniform_nodes(48, 0, 1),
                        synth.uniform_nodes(48, 0, 1))
    ell = synth.ellipsoid_body((0.5, 0.5, 0.5), (0.3, 0.18, 0.22), synth.random_rotation(rng), 4)
    g_plate = synth.small_grid(64, 32, 32, (4.0, 2.0, 2.0))
    return {
        "sphere_small": (g_small, [synth.sphere_body((1.0, 1.0, 1.0), 1.0, 3)]),
        "sphere_stretched": (g_str, [synth.sphere_body((1.0, 1.0, 1.0), 1.0, 4)]),
        "ellipsoid_rotated": (g_cube, [ell]),
        "two_spheres": (g_small, [synth.sphere_body((1.0, 1.0, 1.0), 0.8, 3),
                                  synth.sphere_body((2.6, 0.9, 1.1), 0.7, 3)]),
        "membrane_plate": (g_plate, [_plate(1.0 / 16.0, (1.2, 1.0, 1.0), math.radians(20.0))]),
    }


CASES = _cases()


def _oracle(grid, bodies):
    oc = O.OracleCase(grid)
    for b in bodies:
        oc.add_body(b)
    oc.set_iblank()
    rc = oc.gcm(2.0, 2.0)
    return oc, rc


def _device(grid, bodies):
    c = fg.Case(grid, fg.default_config())
    for b in bodies:
        c.add_body(b)
    ib0 = c.set_iblank_body_fast()
    return c, ib0


def _compare_rows(name, got, want, keys):
    for k in keys:
        a, b = got[k], want[k]
        assert a.shape == b.shape, (name, k, a.shape, b.shape)
        if a.size:
            bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))) if a.dtype.kind == "f"
                              else a != b)
            assert bad.size == 0, (name, k, bad[:5].tolist(), a[tuple(bad[0])], b[tuple(bad[0])])


@pytest.mark.parametrize("name", list(CASES))
def test_tagging_bit_exact(name):
    grid, bodies = CASES[name]
    oc, orc = _oracle(grid, bodies)
    c, _ = _device(grid, bodies)
    # band and the committed iblank before smoothing
    band_o = oc.field(4)
    assert np.array_equal(c.band(), band_o), name
    ib, gh, dd = c.gcm_set_internal_boundary()
    assert np.array_equal(ib, oc.field(0)), name
    assert np.array_equal(gh, oc.field(1)), name
    assert np.array_equal(dd, oc.field(2)), name
    cnt = oc.counts()
    assert (c.nGhost, c.nDead) == (cnt["nGhost"], cnt["nDead"])
    assert c.nGhost > 0 and c.nDead > 0
    _compare_rows(name + "/ghost", c.ghost_rows(), oc.ghosts(), GHOST_KEYS)
    _compare_rows(name + "/dead", c.dead_rows(), oc.deads(), DEAD_KEYS)
    c.close()


def test_iblank_before_smoothing_bit_exact():
    grid, bodies = CASES["sphere_stretched"]
    oc = O.OracleCase(grid)
    for b in bodies:
        oc.add_body(b)
    oc.set_iblank()
    c, ib0 = _device(grid, bodies)
    assert np.array_equal(ib0, oc.field(0))
    c.close()


def test_moving_body_retag():
    """A pitching membrane moved through three positions: each re-tag of the
    same handle matches a fresh oracle tagging (BOUNDARY_MOVE.F90 then
    set_iblank_body_fast and GCM_set_internal_boundary every step)."""
    grid = synth.small_grid(64, 32, 32, (4.0, 2.0, 2.0))
    base = synth.plate_body(n=24, size=1.0, tkns_factor=1.0, grid_h=1.0 / 16.0)
    c = fg.Case(grid, fg.default_config())
    first = True
    for ang in (10.0, 17.5, 25.0):
        verts = synth.pitch_plate(base, (1.2, 1.0, 1.0), math.radians(ang))
        body = synth.Body(verts=verts, tri=base.tri, surface=2, membrane_tkns=base.membrane_tkns)
        if first:
            c.add_body(body)
            first = False
        else:
            c.update_body(0, verts)
        c.set_iblank_body_fast()
        ib, gh, dd = c.gcm_set_internal_boundary()
        oc, _ = _oracle(grid, [body])
        assert np.array_equal(ib, oc.field(0)), ang
        assert np.array_equal(gh, oc.field(1)), ang
        assert np.array_equal(dd, oc.field(2)), ang
        _compare_rows(f"move{ang}/ghost", c.ghost_rows(), oc.ghosts(), GHOST_KEYS)
        _compare_rows(f"move{ang}/dead", c.dead_rows(), oc.deads(), DEAD_KEYS)
    c.close()


def test_config0_tagging_bit_exact():
    """The 128x64x64 sphere case (icosphere of 20480 triangles)."""
    grid, body = synth.config0_grid(), synth.config0_body()
    oc, _ = _oracle(grid, [body])
    c, _ = _device(grid, [body])
    ib, gh, dd = c.gcm_set_internal_boundary()
    assert np.array_equal(ib, oc.field(0))
    assert np.array_equal(gh, oc.field(1))
    assert np.array_equal(dd, oc.field(2))
    _compare_rows("c0/ghost", c.ghost_rows(), oc.ghosts(), GHOST_KEYS)
    _compare_rows("c0/dead", c.dead_rows(), oc.deads(), DEAD_KEYS)
    c.close()
