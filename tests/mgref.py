"""numpy model of the multigrid the CUDA library runs (NOT the reference's
multigrid: that one is restated in oracle/).  It is the same-operation
reference for the GPU kernel tests: zebra line relaxation, residual,
restriction, prolongation, ghost-row relaxation and the coarsest solve,
written with whole-array numpy operations in float64 or float32.

Discrete system (identical to the reference's fixed point, CORE_POISSON.F90
:494-521 and GCM_GHOSTCELL_UPDATE.F90:563-641):
  ACTIVE cell (fluid, not ghost):  sum_faces a (p_n - p_c) = f_c
  FIXED cell (ghost / dead / pure solid): value from its interpolation row
  boundary faces: homogeneous Neumann drops the face, Dirichlet p_n = -p_c
Coarse levels mark cells with >= 50 % solid volume OFF and drop their
faces (zero flux), so the coarse operator sees the body as a Neumann wall.
"""
from __future__ import annotations

import numpy as np

ACTIVE, FIXED, OFF = 0, 1, 2


class Level:
    def __init__(self, xn, yn, zn, types, bc=("N",) * 6, dtype=np.float64):
        """xn/yn/zn: node coordinates of this level (x(1..I)); types:
        int8 array (I-1, J-1, K-1) over interior cells."""
        self.dtype = dtype
        self.types = types
        self.I, self.J, self.K = len(xn), len(yn), len(zn)
        self.bc = bc
        self.ax = [self._axis(v) for v in (xn, yn, zn)]

    @staticmethod
    def _axis(xn):
        n = len(xn)
        x = np.zeros(n + 2); x[1:n + 1] = xn
        x[0] = 2 * x[1] - x[2]; x[n + 1] = 2 * x[n] - x[n - 1]
        xc = np.zeros(n + 2); xc[0:n + 1] = 0.5 * (x[1:n + 2] + x[0:n + 1])
        dxinv = 1.0 / (x[1:n + 1] - x[0:n])  # index 0..n-1 -> cells 0..n-1
        dxcinv = np.zeros(n + 2); dxcinv[1:n + 1] = 1.0 / (xc[1:n + 1] - xc[0:n])
        i = np.arange(1, n)  # interior cells 1..n-1
        am = dxcinv[i] * dxinv[i]
        ap = dxcinv[i + 1] * dxinv[i]
        vol = x[2:n + 1] - x[1:n]
        return dict(am=am, ap=ap, xc=xc[1:n], width=vol, x=x)


def coarse_axis_nodes(xf):
    """CORE_MG.F90:234-243: coarse nodes are every other fine node, the last
    node stays on the boundary; returns coarse node array."""
    nF = len(xf)
    nC = nF // 2 + 1 if nF % 2 == 0 else (nF + 1) // 2
    xc = np.empty(nC)
    xc[:nC - 1] = xf[0:2 * (nC - 1):2]
    xc[nC - 1] = xf[-1]
    return xc


def face_coeffs(L: Level):
    """Per-cell face coefficients (6, I-1, J-1, K-1) after dropping faces
    toward OFF cells and the domain boundary (Neumann) or doubling them on
    Dirichlet faces (diag only); also returns the diagonal and the
    coupling masks used in line solves."""
    t = L.types
    nx, ny, nz = t.shape
    ax, ay, az = L.ax
    A = np.zeros((6,) + t.shape)
    A[0] = ax["am"][:, None, None]; A[1] = ax["ap"][:, None, None]
    A[2] = ay["am"][None, :, None]; A[3] = ay["ap"][None, :, None]
    A[4] = az["am"][None, None, :]; A[5] = az["ap"][None, None, :]
    # neighbour types, boundary encoded as -1
    nb = np.full((6,) + t.shape, -1, dtype=np.int8)
    nb[0, 1:] = t[:-1]; nb[1, :-1] = t[1:]
    nb[2, :, 1:] = t[:, :-1]; nb[3, :, :-1] = t[:, 1:]
    nb[4, :, :, 1:] = t[:, :, :-1]; nb[5, :, :, :-1] = t[:, :, 1:]
    coup = (nb == ACTIVE) | (nb == FIXED)
    diag = np.zeros(t.shape)
    for f in range(6):
        dirich = (nb[f] == -1) & (L.bc[f] == "D")
        diag -= A[f] * (coup[f] + 2.0 * dirich)
    Acoup = A * coup
    return Acoup, diag


class Problem:
    """One grid + masks + interpolation rows; builds the level hierarchy."""

    def __init__(self, grid, iblank, ghost, dead, rows_g, rows_d, levels_xyz, ibk_levels,
                 dtype=np.float64, omega=1.0, nu1=2, nu2=2):
        self.grid = grid
        nx, ny, nz = grid.nx, grid.ny, grid.nz
        ib = iblank[1:nx, 1:ny, 1:nz]
        gh = ghost[1:nx, 1:ny, 1:nz]
        t0 = np.where((ib == 1) | (gh == 1), FIXED, ACTIVE).astype(np.int8)
        self.levels = [Level(grid.xn, grid.yn, grid.zn, t0, dtype=dtype)]
        for (xn, yn, zn), ibk in zip(levels_xyz[1:], ibk_levels[1:]):
            t = np.where(ibk == 1, OFF, ACTIVE).astype(np.int8)
            self.levels.append(Level(xn, yn, zn, t, dtype=dtype))
        self.solid0 = (ib == 1) & (dead[1:nx, 1:ny, 1:nz] != -1)
        self.dtype = dtype
        self.omega = omega
        self.nu1, self.nu2 = nu1, nu2
        self.coef = [face_coeffs(L) for L in self.levels]
        # interpolation rows in interior-cell coordinates (0-based cells)
        self.rows = []
        for R in (rows_d, rows_g):  # dead first, then ghost (reference order)
            if R is None or len(R["ijk"]) == 0:
                continue
            t = R["ijk"] - 1
            src = R["cell"][:, None, :] + np.array(
                [[0, 0, 0], [0, 1, 0], [1, 1, 0], [1, 0, 0], [0, 0, 1], [0, 1, 1], [1, 1, 1], [1, 0, 1]])[None] - 1
            w = R["coef"].copy()
            own = np.all(src == t[:, None, :], axis=2)
            w[own] = 0.0
            self.rows.append((t, src, w, R.get("fixed", np.zeros(len(t), bool))))
        self._coarsest_inverse()

    # ------------------------------------------------------------ operator
    def apply(self, lev, p):
        """(A p) on interior cells of level lev; p is (I-1,J-1,K-1)."""
        A, diag = self.coef[lev]
        out = diag * p
        pp = np.pad(p, 1)
        out += A[0] * pp[:-2, 1:-1, 1:-1] + A[1] * pp[2:, 1:-1, 1:-1]
        out += A[2] * pp[1:-1, :-2, 1:-1] + A[3] * pp[1:-1, 2:, 1:-1]
        out += A[4] * pp[1:-1, 1:-1, :-2] + A[5] * pp[1:-1, 1:-1, 2:]
        return out

    def residual(self, lev, p, f):
        r = f - self.apply(lev, p)
        r[self.levels[lev].types != ACTIVE] = 0.0
        return r

    # ---------------------------------------------------------- line relax
    def line_relax(self, lev, p, f, axis, color):
        """Zebra line relaxation along ``axis`` of the lines of ``color``.
        x-lines (j,k) colour (j+k)%2; y-lines (i,k) colour k%2 with the
        i-neighbours taken from the state before this direction (Jacobi in
        i); z-lines (i,j) colour j%2, Jacobi in i.  ``p_start`` snapshots
        are handled by the caller passing the pre-direction state."""
        raise NotImplementedError

    def smooth(self, lev, p, f):
        L = self.levels[lev]
        A, diag = self.coef[lev]
        t = L.types
        om = self.omega
        for axis in range(3):
            snap = p.copy()  # state before this direction (for Jacobi in i)
            for color in (0, 1):
                p[...] = _relax_dir(p, snap, f, A, diag, t, axis, color, om)
            if lev == 0:
                self.relax_rows(p, None)

    def relax_rows(self, p, g0):
        """One Jacobi pass over dead rows then ghost rows."""
        for (t, src, w, fixed) in self.rows:
            vals = np.sum(w * p[src[..., 0], src[..., 1], src[..., 2]], axis=1)
            p[t[:, 0], t[:, 1], t[:, 2]] = np.where(fixed, p[t[:, 0], t[:, 1], t[:, 2]], vals)

    # --------------------------------------------------------- transfers
    def restrict(self, lev, r):
        F, C = self.levels[lev], self.levels[lev + 1]
        out = np.zeros(C.types.shape)
        vol = np.zeros(C.types.shape)
        fx = [a["width"] for a in F.ax]
        w = fx[0][:, None, None] * fx[1][None, :, None] * fx[2][None, None, :]
        maps = [_child_map(F, C, a) for a in range(3)]
        np.add.at(out, np.ix_(maps[0], maps[1], maps[2]), w * r)
        np.add.at(vol, np.ix_(maps[0], maps[1], maps[2]), w)
        out = out / vol
        out[C.types != ACTIVE] = 0.0
        return out

    def prolong(self, lev, e_c):
        """Trilinear interpolation of the coarse correction (level lev+1) to
        the fine cell centres of level lev, skipping OFF coarse corners and
        renormalising; fine OFF cells receive nothing."""
        F, C = self.levels[lev], self.levels[lev + 1]
        act = (C.types == ACTIVE).astype(float)
        ix = [_interp_map(F, C, a) for a in range(3)]
        out = np.zeros(F.types.shape)
        wsum = np.zeros(F.types.shape)
        for cx in (0, 1):
            for cy in (0, 1):
                for cz in (0, 1):
                    i0, wx = ix[0][cx]; j0, wy = ix[1][cy]; k0, wz = ix[2][cz]
                    w = wx[:, None, None] * wy[None, :, None] * wz[None, None, :]
                    a = act[np.ix_(i0, j0, k0)]
                    out += w * a * e_c[np.ix_(i0, j0, k0)]
                    wsum += w * a
        out = np.where(wsum > 1e-12, out / np.maximum(wsum, 1e-300), 0.0)
        out[F.types == OFF] = 0.0
        if lev == 0:
            out[self.solid0] = 0.0
        return out

    def _coarsest_inverse(self):
        L = self.levels[-1]
        n = L.types.size
        eye = np.eye(n).reshape((n,) + L.types.shape)
        M = np.stack([self.apply(len(self.levels) - 1, eye[q]).ravel() for q in range(n)], axis=1)
        act = (L.types.ravel() == ACTIVE)
        Ma = M[np.ix_(act, act)]
        self.coarse_act = act
        self.coarse_pinv = np.linalg.pinv(Ma)

    def coarse_solve(self, r):
        L = self.levels[-1]
        e = np.zeros(r.size)
        e[self.coarse_act] = self.coarse_pinv @ r.ravel()[self.coarse_act]
        return e.reshape(r.shape)

    # ------------------------------------------------------------- V-cycle
    def vcycle(self, lev, x, f):
        if lev == len(self.levels) - 1:
            return self.coarse_solve(f)
        for _ in range(self.nu1):
            self.smooth(lev, x, f)
        r = self.residual(lev, x, f)
        rc = self.restrict(lev, r)
        ec = self.vcycle(lev + 1, np.zeros_like(rc), rc)
        x += self.prolong(lev, ec)
        if lev == 0:
            self.relax_rows(x, None)
        for _ in range(self.nu2):
            self.smooth(lev, x, f)
        return x


def _child_map(F, C, axis):
    nF = F.types.shape[axis]
    nC = C.types.shape[axis]
    if nF == nC:
        return np.arange(nF)
    return np.minimum(np.arange(nF) // 2, nC - 1)


def _interp_map(F, C, axis):
    xf = F.ax[axis]["xc"]
    xcg = C.ax[axis]["xc"]
    nC = len(xcg)
    lo = np.clip(np.searchsorted(xcg, xf, side="right") - 1, 0, nC - 1)
    hi = np.minimum(lo + 1, nC - 1)
    den = np.where(hi > lo, xcg[hi] - xcg[lo], 1.0)
    w = np.clip((xf - xcg[lo]) / den, 0.0, 1.0)
    w = np.where(hi > lo, w, 0.0)
    return [(lo, 1.0 - w), (hi, w)]


COLORING = "jacobi_i"   # y/z-lines: colour by k / j parity, Jacobi in i


def _relax_dir(p, snap, f, A, diag, t, axis, color, om):
    """Zebra line relaxation in direction ``axis`` for lines of ``color``."""
    n0, n1, n2 = t.shape
    pp = np.pad(p, 1)
    sp = np.pad(snap, 1)
    # move the line axis last
    perm = {0: (1, 2, 0), 1: (0, 2, 1), 2: (0, 1, 2)}[axis]
    inv = np.argsort(perm)
    # transverse contributions
    rhs = f.copy()
    nbs = [(0, pp[:-2, 1:-1, 1:-1], sp[:-2, 1:-1, 1:-1]), (1, pp[2:, 1:-1, 1:-1], sp[2:, 1:-1, 1:-1]),
           (2, pp[1:-1, :-2, 1:-1], sp[1:-1, :-2, 1:-1]), (3, pp[1:-1, 2:, 1:-1], sp[1:-1, 2:, 1:-1]),
           (4, pp[1:-1, 1:-1, :-2], sp[1:-1, 1:-1, :-2]), (5, pp[1:-1, 1:-1, 2:], sp[1:-1, 1:-1, 2:])]
    for f_, cur, old in nbs:
        if f_ // 2 == axis:
            continue
        # x-lines: all transverse neighbours are the other colour (use cur);
        # y/z-lines: i-neighbours use the pre-direction snapshot
        src = old if (axis != 0 and f_ // 2 == 0 and COLORING == "jacobi_i") else cur
        rhs = rhs - A[f_] * src
    a = A[2 * axis].copy(); c = A[2 * axis + 1].copy(); b = diag.copy()
    fixed = t != ACTIVE
    a[fixed] = 0.0; c[fixed] = 0.0; b[fixed] = 1.0; rhs[fixed] = p[fixed]
    # line colour
    I, J, K = np.meshgrid(np.arange(n0), np.arange(n1), np.arange(n2), indexing="ij")
    if axis == 0:
        col = (J + K) % 2
    elif axis == 1:
        col = K % 2 if COLORING == "jacobi_i" else (I + K) % 2
    else:
        col = J % 2 if COLORING == "jacobi_i" else (I + J) % 2
    sel = col == color
    a, b, c, rhs, pt, selt = (np.transpose(v, perm) for v in (a, b, c, rhs, p, sel))
    x = _thomas(a, b, c, rhs)
    new = np.where(selt, pt + om * (x - pt), pt)
    new = np.where(np.transpose(fixed, perm), pt, new)
    return np.transpose(new, inv)


def _thomas(a, b, c, d):
    n = a.shape[-1]
    cp = np.zeros_like(d); dp = np.zeros_like(d)
    cp[..., 0] = c[..., 0] / b[..., 0]
    dp[..., 0] = d[..., 0] / b[..., 0]
    for i in range(1, n):
        den = b[..., i] - a[..., i] * cp[..., i - 1]
        cp[..., i] = c[..., i] / den
        dp[..., i] = (d[..., i] - a[..., i] * dp[..., i - 1]) / den
    x = np.zeros_like(d)
    x[..., -1] = dp[..., -1]
    for i in range(n - 2, -1, -1):
        x[..., i] = dp[..., i] - cp[..., i] * x[..., i + 1]
    return x
