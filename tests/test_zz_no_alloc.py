"""fg_rows_relax_noalloc: the ghost/dead row relaxation for callers that
cannot allocate device memory (they only get memory from a pool or
framework they do not own, or may not stall the device with an
allocation).  It must give the same field as the handle-based entry
point fg_ghostcell_pressure, with its scratch in the library's fixed
static array; two calls in a row check that the shared array carries
nothing over between calls.  Collected last so that a run stopping at the
first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from feicar_b200 import fg, synth

pytestmark = pytest.mark.gpu

INC = np.array([[0, 0, 0], [0, 1, 0], [1, 1, 0], [1, 0, 0], [0, 0, 1], [0, 1, 1], [1, 1, 1], [1, 0, 1]])


def _lib():
    L = fg.lib()
    L.fg_rows_relax_noalloc.restype = C.c_int
    L.fg_rows_relax_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    return L


def _rows(grid, c):
    """Dead rows then ghost rows as element indices of the reference layout,
    with the target's own corner weighted 0 (homogeneous Neumann data)."""
    NX, NY = grid.nx + 2, grid.ny + 2
    tgt, cell, w = [], [], []
    for R in (c.dead_rows(), c.ghost_rows()):
        ijk, hc, coef = R["ijk"].astype(np.int64), R["cell"].astype(np.int64), R["coefN"].copy()
        corners = hc[:, None, :] + INC[None, :, :]
        own = np.all(corners == ijk[:, None, :], axis=2)
        coef[own] = 0.0
        tgt.append(ijk[:, 0] + NX * (ijk[:, 1] + NY * ijk[:, 2]))
        cell.append(hc[:, 0] + NX * (hc[:, 1] + NY * hc[:, 2]))
        w.append(coef)
    return np.concatenate(tgt), np.concatenate(cell), np.ascontiguousarray(np.concatenate(w))


def test_noalloc_matches_ghostcell_pressure_twice():
    grid = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0))
    c = fg.Case(grid, fg.default_config())
    c.add_body(synth.sphere_body((1.0, 1.0, 1.0), 1.0, 3))
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    c.mg_prepare()
    tgt, cell, w = _rows(grid, c)
    n = len(tgt)
    assert n > 0
    d_tgt = torch.from_numpy(tgt).cuda()
    d_cell = torch.from_numpy(cell).cuda()
    d_w = torch.from_numpy(w.ravel()).cuda()
    d_c0 = torch.zeros(n, dtype=torch.float64, device="cuda")
    L = _lib()
    rng = np.random.default_rng(11)
    p = np.asfortranarray(rng.standard_normal(grid.shape))
    for iters in (1, 3):  # two calls in a row on the shared scratch array
        want = p.copy(order="F")
        c.ghostcell_pressure(want, iterations=iters)
        d_p = torch.from_numpy(np.ascontiguousarray(p.transpose(2, 1, 0))).cuda()
        rc = L.fg_rows_relax_noalloc(grid.nx, grid.ny, grid.nz, d_p.data_ptr(), n, d_tgt.data_ptr(),
                                     d_cell.data_ptr(), d_w.data_ptr(), d_c0.data_ptr(), iters, None)
        assert rc == fg.FG_OK
        torch.cuda.synchronize()
        got = d_p.cpu().numpy().transpose(2, 1, 0)
        scale = max(1.0, float(np.abs(want).max()))
        assert np.abs(got - want).max() <= 1e-12 * scale
        assert not np.array_equal(got, p)  # the rows did move
        p = np.asfortranarray(got + rng.standard_normal(grid.shape) * 0.1)
    c.close()


def test_noalloc_rejects_more_rows_than_its_scratch():
    L = _lib()
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = L.fg_rows_relax_noalloc(4, 4, 4, d.data_ptr(), 262144 + 1, d.data_ptr(), d.data_ptr(),
                                 d.data_ptr(), None, 1, None)
    assert rc == 5  # FG_BAD_INPUT


def _relax_numpy(p_flat, tgt, cell, w, c0, nx, ny, iters):
    """The row update restated in numpy: every row gathers from the field
    as it was at the start of the pass, then all targets are written."""
    sy, sz = nx + 2, (nx + 2) * (ny + 2)
    off = np.array([0, sy, sy + 1, 1, sz, sz + sy, sz + sy + 1, sz + 1])
    ok = (cell >= 0) & (cell + off[6] < p_flat.size) & (tgt >= 0) & (tgt < p_flat.size)
    p = p_flat.copy()
    for _ in range(iters):
        vals = (w[ok] * p[cell[ok, None] + off[None, :]]).sum(axis=1) + c0[ok]
        p[tgt[ok]] = vals
    return p


def test_noalloc_constant_term_and_skipped_row():
    """Rows with a non-zero constant (the previous-step pressure of the
    dead-cell fallback, or dp/dn data) against the numpy restatement, and
    a row whose host cell lies outside the field: that row is skipped (its
    target keeps its value) while every other row is relaxed."""
    grid = synth.small_grid(32, 16, 16, (4.0, 2.0, 2.0))
    c = fg.Case(grid, fg.default_config())
    c.add_body(synth.sphere_body((1.0, 1.0, 1.0), 1.0, 3))
    c.set_iblank_body_fast()
    c.gcm_set_internal_boundary()
    tgt, cell, w = _rows(grid, c)
    c.close()
    n = len(tgt)
    assert len(np.unique(tgt)) == n
    rng = np.random.default_rng(5)
    c0 = rng.standard_normal(n)
    bad = n // 2
    cell = cell.copy()
    cell[bad] = int(np.prod(grid.shape))  # past the last element
    p = np.asfortranarray(rng.standard_normal(grid.shape))
    p_flat = p.ravel(order="F")
    want = _relax_numpy(p_flat, tgt, cell, w, c0, grid.nx, grid.ny, 2)
    d_p = torch.from_numpy(p_flat.copy()).cuda()
    d_tgt, d_cell = torch.from_numpy(tgt).cuda(), torch.from_numpy(cell).cuda()
    d_w, d_c0 = torch.from_numpy(w.ravel()).cuda(), torch.from_numpy(c0).cuda()
    L = _lib()
    for _ in range(2):  # two calls in a row, each from the same start
        d_p.copy_(torch.from_numpy(p_flat))
        rc = L.fg_rows_relax_noalloc(grid.nx, grid.ny, grid.nz, d_p.data_ptr(), n, d_tgt.data_ptr(),
                                     d_cell.data_ptr(), d_w.data_ptr(), d_c0.data_ptr(), 2, None)
        assert rc == fg.FG_OK
        torch.cuda.synchronize()
        got = d_p.cpu().numpy()
        assert np.abs(got - want).max() <= 1e-12 * max(1.0, float(np.abs(want).max()))
        assert got[tgt[bad]] == p_flat[tgt[bad]]  # targets are distinct cells
        assert np.count_nonzero(got != p_flat) > n // 2
