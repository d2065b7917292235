"""Synthetic inputs for the pressure-Poisson path: grids, triangulated bodies
and right-hand sides of the shapes the benchmark configurations name.

The reference reads its grid from ``xgrid.dat``-style node lists
(CORE_GRID.F90:40-89) and its body from a Gmsh file
(BOUNDARY_MARKER_INIT.F90:247-296); neither ships with the reference, so the
inputs here are generated, seeded and reproducible.

Conventions kept from the reference:

* node counts ``nx, ny, nz`` (cells = n - 1), node coordinates x(1..nx);
* triangle normals ``(v2-v1) x (v3-v2)`` point INTO the body
  (BOUNDARY_SET_ARCLENGTH_NORM.F90:74-79, :196-200);
* fields are Fortran-ordered ``(0:nx+1, 0:ny+1, 0:nz+1)`` arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# --------------------------------------------------------------------- grids


def uniform_nodes(ncells: int, lo: float, hi: float) -> np.ndarray:
    """x(1..n) of a uniform grid, CORE_GRID.F90:38-42."""
    n = ncells + 1
    delta = (hi - lo) / float(n - 1)
    return lo + np.arange(n, dtype=np.float64) * delta


def tanh_nodes(ncells: int, lo: float, hi: float, beta: float = 2.0) -> np.ndarray:
    """Nodes clustered toward the middle of [lo, hi]:
    y(eta) = c + (L/2) atanh(xi tanh(beta)) / beta, xi = 2 eta - 1.
    The end points are exactly lo and hi."""
    n = ncells + 1
    eta = np.arange(n, dtype=np.float64) / float(n - 1)
    xi = 2.0 * eta - 1.0
    c = 0.5 * (lo + hi)
    half = 0.5 * (hi - lo)
    y = c + half * np.arctanh(xi * math.tanh(beta)) / beta
    y[0] = lo
    y[-1] = hi
    return y


@dataclass
class Grid:
    """Node coordinates plus the derived metrics of CORE_GRID.F90:109-205."""

    xn: np.ndarray
    yn: np.ndarray
    zn: np.ndarray
    x: np.ndarray = field(init=False)
    y: np.ndarray = field(init=False)
    z: np.ndarray = field(init=False)
    xc: np.ndarray = field(init=False)
    yc: np.ndarray = field(init=False)
    zc: np.ndarray = field(init=False)

    def __post_init__(self):
        self.x, self.xc = _axis(self.xn)
        self.y, self.yc = _axis(self.yn)
        self.z, self.zc = _axis(self.zn)

    @property
    def nx(self) -> int:
        return len(self.xn)

    @property
    def ny(self) -> int:
        return len(self.yn)

    @property
    def nz(self) -> int:
        return len(self.zn)

    @property
    def shape(self):
        return (self.nx + 2, self.ny + 2, self.nz + 2)

    @property
    def cells(self) -> int:
        return (self.nx - 1) * (self.ny - 1) * (self.nz - 1)


def _axis(xn):
    n = len(xn)
    x = np.zeros(n + 2)
    x[1 : n + 1] = xn
    x[0] = x[1] * 2.0 - x[2]
    x[n + 1] = x[n] + x[n] - x[n - 1]
    xc = np.zeros(n + 2)
    xc[0 : n + 1] = 0.5 * (x[1 : n + 2] + x[0 : n + 1])
    xc[n + 1] = x[n + 1]
    return x, xc


# -------------------------------------------------------------------- bodies


@dataclass
class Body:
    """One triangulated surface; ``tri`` is 0-based (ntri, 3) int32."""

    verts: np.ndarray
    tri: np.ndarray
    surface: int = 1  # 1 solid, 2 membrane
    membrane_tkns: float = 0.0
    body_dim: int = 3

    @property
    def nvert(self):
        return self.verts.shape[0]

    @property
    def ntri(self):
        return self.tri.shape[0]


def _icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array(
        [
            [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
            [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
            [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1],
        ],
        dtype=np.float64,
    )
    f = np.array(
        [
            [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
            [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
            [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
            [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
        ],
        dtype=np.int64,
    )
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, f


def icosphere(subdiv: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere with 20*4**subdiv triangles, vertices on the sphere.

    Returns (verts, tri) with the reference's inward-normal winding."""
    v, f = _icosahedron()
    verts = [tuple(p) for p in v]
    for _ in range(subdiv):
        cache: dict[tuple[int, int], int] = {}
        nf = []

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key in cache:
                return cache[key]
            pa, pb = np.array(verts[a]), np.array(verts[b])
            m = 0.5 * (pa + pb)
            m /= np.linalg.norm(m)
            verts.append(tuple(m))
            cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = np.array(nf, dtype=np.int64)
    verts = np.array(verts, dtype=np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    # the icosahedron faces above are counter-clockwise seen from outside
    # (outward normals); swap two vertices to make (v2-v1)x(v3-v2) point in
    tri = f[:, [0, 2, 1]].astype(np.int32)
    return verts, tri


def sphere_body(center, diameter: float, subdiv: int) -> Body:
    v, t = icosphere(subdiv)
    verts = np.asarray(center, dtype=np.float64)[None, :] + 0.5 * diameter * v
    return Body(verts=verts, tri=t)


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform random rotation from a uniform unit quaternion."""
    u1, u2, u3 = rng.random(3)
    q = np.array(
        [
            math.sqrt(1 - u1) * math.sin(2 * math.pi * u2),
            math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
            math.sqrt(u1) * math.sin(2 * math.pi * u3),
            math.sqrt(u1) * math.cos(2 * math.pi * u3),
        ]
    )
    x, y, z, w = q
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
            [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
            [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
        ]
    )


def ellipsoid_body(center, semi_axes, rotation: np.ndarray, subdiv: int = 4) -> Body:
    """Icosphere scaled by the semi-axes and rotated; a positive-determinant
    linear map keeps the inward winding."""
    v, t = icosphere(subdiv)
    m = rotation @ np.diag(np.asarray(semi_axes, dtype=np.float64))
    verts = np.asarray(center, dtype=np.float64)[None, :] + v @ m.T
    return Body(verts=verts, tri=t)


def plate_body(n: int = 64, size: float = 1.0, tkns_factor: float = 1.0,
               grid_h: float = 1.0 / 32.0) -> Body:
    """Flat square membrane sheet of 2*n*n triangles in the x-z plane with its
    leading edge on x = 0 (pivot for pitching), thickness handled by the
    membrane band ``membrane_tkns = factor * sqrt(dx^2+dy^2+dz^2)``
    (BOUNDARY_MARKER_INIT.F90:425-428)."""
    xs = np.linspace(0.0, size, n + 1)
    zs = np.linspace(-0.5 * size, 0.5 * size, n + 1)
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    verts = np.stack([X.ravel(), np.zeros(X.size), Z.ravel()], axis=1)
    idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    a = idx[:-1, :-1].ravel()
    b = idx[1:, :-1].ravel()
    c = idx[1:, 1:].ravel()
    d = idx[:-1, 1:].ravel()
    tri = np.empty((2 * n * n, 3), dtype=np.int32)
    tri[0::2] = np.stack([a, b, c], axis=1)
    tri[1::2] = np.stack([a, c, d], axis=1)
    tk = tkns_factor * math.sqrt(3.0) * grid_h
    return Body(verts=verts, tri=tri, surface=2, membrane_tkns=tk)


def pitch_plate(body: Body, pivot, angle_rad: float) -> np.ndarray:
    """Vertices of the plate rotated about the z-axis through ``pivot``."""
    c, s = math.cos(angle_rad), math.sin(angle_rad)
    r = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    p = np.asarray(pivot, dtype=np.float64)
    return p[None, :] + (body.verts @ r.T)


# ------------------------------------------------------------ right-hand side


def box_smooth(a: np.ndarray, passes: int = 3) -> np.ndarray:
    """Three-point [1,2,1]/4 box filter applied ``passes`` times per axis,
    with edge replication."""
    out = a.copy()
    for ax in range(out.ndim):
        for _ in range(passes):
            p = np.concatenate(
                [np.take(out, [0], axis=ax), out, np.take(out, [-1], axis=ax)], axis=ax
            )
            n = out.shape[ax]
            out = 0.25 * np.take(p, range(0, n), axis=ax) + 0.5 * np.take(
                p, range(1, n + 1), axis=ax
            ) + 0.25 * np.take(p, range(2, n + 2), axis=ax)
    return out


def fortran_zeros(grid: Grid, dtype=np.float64) -> np.ndarray:
    return np.zeros(grid.shape, dtype=dtype, order="F")


def neumann_fill(grid: Grid, f: np.ndarray) -> None:
    """Boundary layers copy their neighbour: homogeneous Neumann
    (CORE_SET_OUTER_BC.F90:910, :1093 with pgrad = 0)."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    f[0, :, :] = f[1, :, :]
    f[nx, :, :] = f[nx - 1, :, :]
    f[:, 0, :] = f[:, 1, :]
    f[:, ny, :] = f[:, ny - 1, :]
    f[:, :, 0] = f[:, :, 1]
    f[:, :, nz] = f[:, :, nz - 1]


def laplacian(grid: Grid, p: np.ndarray) -> np.ndarray:
    """7-point operator of CORE_POISSON.F90:494-521 on interior cells."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    x, y, z, xc, yc, zc = grid.x, grid.y, grid.z, grid.xc, grid.yc, grid.zc
    dxinv = 1.0 / (x[1 : nx + 1] - x[0:nx])
    dyinv = 1.0 / (y[1 : ny + 1] - y[0:ny])
    dzinv = 1.0 / (z[1 : nz + 1] - z[0:nz])
    dxcinv = np.zeros(nx + 2); dxcinv[1 : nx + 1] = 1.0 / (xc[1 : nx + 1] - xc[0:nx])
    dycinv = np.zeros(ny + 2); dycinv[1 : ny + 1] = 1.0 / (yc[1 : ny + 1] - yc[0:ny])
    dzcinv = np.zeros(nz + 2); dzcinv[1 : nz + 1] = 1.0 / (zc[1 : nz + 1] - zc[0:nz])
    i = np.arange(1, nx)
    j = np.arange(1, ny)
    k = np.arange(1, nz)
    bmx = (dxcinv[i] * dxinv[i])[:, None, None]
    bpx = (dxcinv[i + 1] * dxinv[i])[:, None, None]
    bmy = (dycinv[j] * dyinv[j])[None, :, None]
    bpy = (dycinv[j + 1] * dyinv[j])[None, :, None]
    bmz = (dzcinv[k] * dzinv[k])[None, None, :]
    bpz = (dzcinv[k + 1] * dzinv[k])[None, None, :]
    c = p[1:nx, 1:ny, 1:nz]
    out = np.zeros_like(p)
    out[1:nx, 1:ny, 1:nz] = (
        bmx * (p[0 : nx - 1, 1:ny, 1:nz] - c) + bpx * (p[2 : nx + 1, 1:ny, 1:nz] - c)
        + bmy * (p[1:nx, 0 : ny - 1, 1:nz] - c) + bpy * (p[1:nx, 2 : ny + 1, 1:nz] - c)
        + bmz * (p[1:nx, 1:ny, 0 : nz - 1] - c) + bpz * (p[1:nx, 1:ny, 2 : nz + 1] - c)
    )
    return out


INC = np.array(
    [[0, 0, 0], [0, 1, 0], [1, 1, 0], [1, 0, 0], [0, 0, 1], [0, 1, 1], [1, 1, 1], [1, 0, 1]],
    dtype=np.int64,
)  # GCM_MEMORY_ALLOCATE.F90:593-623


@dataclass
class Interp:
    """Ghost/dead interpolation rows: target cell, host cell, 8 weights."""

    ijk: np.ndarray  # (n,3) target cell
    cell: np.ndarray  # (n,3) lower corner of the host cell
    coef: np.ndarray  # (n,8) Neumann weights (coeffGCMN / coeffGCMDeadN)


def _flat(grid: Grid, ijk: np.ndarray) -> np.ndarray:
    NX, NY = grid.nx + 2, grid.ny + 2
    return ijk[..., 0] + NX * (ijk[..., 1] + NY * ijk[..., 2])


def solve_interp_rows(grid: Grid, phi: np.ndarray, rows: list[Interp], fixed: np.ndarray,
                      iters: int = 500, tol: float = 1e-15) -> None:
    """Overwrite the targets of the interpolation rows with the fixed point
    phi_t = sum_q w_q phi_{cell+inc_q} (own slot excluded: homogeneous
    Neumann data), iterating Jacobi sweeps.  ``fixed`` marks rows whose
    value is held (dead cells using the inverse-distance fallback)."""
    flat = phi.reshape(-1, order="F")
    tgt, src, w = [], [], []
    for r in rows:
        if r.ijk.shape[0] == 0:
            continue
        t = _flat(grid, r.ijk)
        s = _flat(grid, r.cell[:, None, :] + INC[None, :, :])
        ww = r.coef.copy()
        ww[s == t[:, None]] = 0.0  # own slot multiplies dpdn = 0
        tgt.append(t); src.append(s); w.append(ww)
    if not tgt:
        return
    tgt = np.concatenate(tgt); src = np.concatenate(src); w = np.concatenate(w)
    keep = ~fixed.reshape(-1, order="F")[tgt]
    tgt, src, w = tgt[keep], src[keep], w[keep]
    scale = max(1.0, float(np.max(np.abs(flat))))
    for _ in range(iters):
        new = np.sum(w * flat[src], axis=1)
        d = float(np.max(np.abs(new - flat[tgt]))) if new.size else 0.0
        flat[tgt] = new
        if d <= tol * scale:
            break


def manufactured_rhs(grid: Grid, iblank: np.ndarray, ghost: np.ndarray, dead: np.ndarray,
                     rows: list[Interp], seed: int, sigma: float = 0.01,
                     dead_fixed: np.ndarray | None = None):
    """Seeded compatible right-hand side with a known discrete solution.

    The flow of the benchmark is u = (1,0,0) + grad(phi): phi is Gaussian
    noise smoothed by three [1,2,1]/4 passes per axis, scaled so the face
    velocities of grad(phi) have standard deviation ``sigma``.  The RHS is
    div(u) = L phi on fluid non-ghost cells (the 7-point operator), zero on
    ghost and solid cells, so the all-Neumann ghost-cell system is exactly
    compatible and its solution is phi up to a constant.  Ghost and dead
    values of phi satisfy their interpolation rows; pure-solid cells hold 0.

    Returns (rhs, phi) as Fortran-ordered arrays."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    phi = fortran_zeros(grid)
    noise = rng.standard_normal((nx - 1, ny - 1, nz - 1))
    noise = box_smooth(noise, 3)
    phi[1:nx, 1:ny, 1:nz] = noise
    neumann_fill(grid, phi)
    # scale: std of the x-face velocities (phi_i - phi_{i-1}) / dxc
    dxc = grid.xc[1:nx] - grid.xc[0 : nx - 1]
    ux = (phi[1:nx, 1:ny, 1:nz] - phi[0 : nx - 1, 1:ny, 1:nz]) / dxc[:, None, None]
    s = float(np.std(ux))
    phi *= sigma / s if s > 0 else 1.0
    solid = (iblank == 1) & (dead != -1)
    phi[solid] = 0.0
    fixed = solid.copy()
    if dead_fixed is not None:
        fixed |= dead_fixed
        phi[dead_fixed] = 0.0
    solve_interp_rows(grid, phi, rows, fixed)
    lap = laplacian(grid, phi)
    fluid = (iblank == 0) & (ghost == 0)
    rhs = fortran_zeros(grid)
    rhs[fluid] = lap[fluid]
    rhs[0, :, :] = 0.0; rhs[nx:, :, :] = 0.0
    rhs[:, 0, :] = 0.0; rhs[:, ny:, :] = 0.0
    rhs[:, :, 0] = 0.0; rhs[:, :, nz:] = 0.0
    return rhs, phi


def test_mg_rhs(grid: Grid) -> np.ndarray:
    """CORE_POISSON.F90:589-607: sum_{K=1..4} 10 cos(KX) cos(KY) cos(KZ) with
    X, Y, Z the cell-centre coordinates scaled to [0, 2 pi]."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    pi2 = 8.0 * math.atan(1.0)
    xx = (grid.xc[1:nx] - grid.xn[0]) / (grid.xn[-1] - grid.xn[0]) * pi2
    yy = (grid.yc[1:ny] - grid.yn[0]) / (grid.yn[-1] - grid.yn[0]) * pi2
    zz = (grid.zc[1:nz] - grid.zn[0]) / (grid.zn[-1] - grid.zn[0]) * pi2
    r = fortran_zeros(grid)
    acc = np.zeros((nx - 1, ny - 1, nz - 1))
    for K in range(1, 5):
        acc += 10 * np.cos(xx * K)[:, None, None] * np.cos(yy * K)[None, :, None] * np.cos(
            zz * K
        )[None, None, :]
    r[1:nx, 1:ny, 1:nz] = acc
    return r


def test_mg_exact(grid: Grid) -> np.ndarray:
    """Closed-form solution of the continuous all-Neumann problem for
    test_mg_rhs: p = -sum 10 cos cos cos / ((2 pi K)^2 (Lx^-2+Ly^-2+Lz^-2))."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    pi2 = 8.0 * math.atan(1.0)
    Lx = grid.xn[-1] - grid.xn[0]
    Ly = grid.yn[-1] - grid.yn[0]
    Lz = grid.zn[-1] - grid.zn[0]
    xx = (grid.xc[1:nx] - grid.xn[0]) / Lx * pi2
    yy = (grid.yc[1:ny] - grid.yn[0]) / Ly * pi2
    zz = (grid.zc[1:nz] - grid.zn[0]) / Lz * pi2
    acc = np.zeros((nx - 1, ny - 1, nz - 1))
    for K in range(1, 5):
        lam = (pi2 * K) ** 2 * (Lx ** -2 + Ly ** -2 + Lz ** -2)
        acc -= 10 * np.cos(xx * K)[:, None, None] * np.cos(yy * K)[None, :, None] * np.cos(
            zz * K
        )[None, None, :] / lam
    p = fortran_zeros(grid)
    p[1:nx, 1:ny, 1:nz] = acc
    return p


# --------------------------------------------------------------- configurations


def config0_grid() -> Grid:
    """128x64x64 uniform cells on [0,8]x[0,4]x[0,4]."""
    return Grid(uniform_nodes(128, 0, 8), uniform_nodes(64, 0, 4), uniform_nodes(64, 0, 4))


def config0_body() -> Body:
    return sphere_body((2.0, 2.0, 2.0), 1.0, 5)


def config1_grid() -> Grid:
    """512x256x256 cells on [0,16]x[0,8]x[0,8], tanh-stretched (beta = 2) in
    y and z toward the sphere centre."""
    return Grid(uniform_nodes(512, 0, 16), tanh_nodes(256, 0, 8, 2.0), tanh_nodes(256, 0, 8, 2.0))


def config1_body() -> Body:
    return sphere_body((4.0, 4.0, 4.0), 1.0, 6)


def config2_grid() -> Grid:
    """256x128x128 uniform cells on [0,8]x[0,4]x[0,4] (h = 1/32)."""
    return Grid(uniform_nodes(256, 0, 8), uniform_nodes(128, 0, 4), uniform_nodes(128, 0, 4))


def config2_plate() -> Body:
    """Flat 1x1 plate of 2*64*64 triangles on the membrane path, thickness
    factor * sqrt(dx^2+dy^2+dz^2) with factor 1 and h = 1/32, in its
    reference position (leading edge on x = 0, the x-z plane)."""
    return plate_body(n=64, size=1.0, tkns_factor=1.0, grid_h=1.0 / 32.0)


CONFIG2_PIVOT = (2.0, 2.0, 2.0)


def config2_verts(base: Body, step: int, period: int = 100, amp_deg: float = 30.0) -> np.ndarray:
    """Plate vertices at time step ``step``: pitch amp*sin(2 pi step/period)
    about the z-axis through the leading edge placed at (2, 2, 2)."""
    ang = math.radians(amp_deg) * math.sin(2.0 * math.pi * step / period)
    return pitch_plate(base, CONFIG2_PIVOT, ang)


def config2_body(step: int) -> Body:
    base = config2_plate()
    return Body(verts=config2_verts(base, step), tri=base.tri, surface=2,
                membrane_tkns=base.membrane_tkns)


def small_grid(ncx=32, ncy=16, ncz=16, L=(4.0, 2.0, 2.0), stretch=None) -> Grid:
    ax = [uniform_nodes(ncx, 0, L[0])]
    if stretch:
        ax += [tanh_nodes(ncy, 0, L[1], stretch), tanh_nodes(ncz, 0, L[2], stretch)]
    else:
        ax += [uniform_nodes(ncy, 0, L[1]), uniform_nodes(ncz, 0, L[2])]
    return Grid(*ax)


def serving_template(seed: int):
    """One problem shape of the serving workload: edge n log-uniform in
    [32, 256] cells, aspect 1:1:1 or 2:1:1 (x doubled) with p = 1/2, on
    [0, a] x [0,1]^2; a sphere (diameter U(0.3, 0.6)) or a randomly rotated
    ellipsoid (semi-axes U(0.15, 0.35)) with p = 1/2, 5120 triangles, at the
    centre of the unit cube that starts at the inflow side.  Returns
    (grid, body)."""
    rng = np.random.default_rng(7000 + seed)
    edge = int(round(math.exp(rng.uniform(math.log(32), math.log(256)))))
    a = 2 if rng.random() < 0.5 else 1
    g = Grid(uniform_nodes(a * edge, 0, float(a)), uniform_nodes(edge, 0, 1.0), uniform_nodes(edge, 0, 1.0))
    centre = (0.5, 0.5, 0.5)
    if rng.random() < 0.5:
        b = sphere_body(centre, rng.uniform(0.3, 0.6), 4)
    else:
        b = ellipsoid_body(centre, rng.uniform(0.15, 0.35, size=3), random_rotation(rng), 4)
    return g, b


def serving_trace(rate: float, seconds: float, ntemplates: int, seed: int = 7):
    """Poisson arrivals at `rate` per second over `seconds`: (arrival time,
    template index, time steps 1..10), seeded."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            return out
        out.append((t, int(rng.integers(ntemplates)), int(rng.integers(1, 11))))


def batch_problems(n: int = 64, seed0: int = 0, lo: int = 32, hi: int = 192):
    """Configuration of the batched workload: cubic grids with edge length
    log-uniform in [lo, hi] cells on [0,1]^3 scaled, each with a seeded
    ellipsoid (semi-axes U(0.15,0.35) of the edge, random orientation, 5120
    triangles) at the box centre.  Returns a list of (grid, body, seed)."""
    out = []
    for s in range(seed0, seed0 + n):
        rng = np.random.default_rng(1000 + s)
        edge = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        L = 1.0
        g = Grid(uniform_nodes(edge, 0, L), uniform_nodes(edge, 0, L), uniform_nodes(edge, 0, L))
        axes = rng.uniform(0.15, 0.35, size=3) * L
        rot = random_rotation(rng)
        b = ellipsoid_body((0.5 * L, 0.5 * L, 0.5 * L), axes, rot, 4)
        out.append((g, b, s))
    return out
