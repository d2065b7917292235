"""ctypes wrapper of the CPU FP64 restatement (``libfeicar_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline leg, always as the checker, never as the
product path.  Parity status: pinned by known answers only; the Fortran
reference cannot be compiled in this image, so parity against reference
outputs is unpinned.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libfeicar_oracle.so")

OR_PBC_DIRICHLET, OR_PBC_NEUMANN = 1, 2
OR_SOLVER_LSOR, OR_SOLVER_MG = 1, 3


class Params(C.Structure):
    _fields_ = [
        ("it_solver_type", C.c_int),
        ("itermax_pson", C.c_int),
        ("restol_pson", C.c_double),
        ("restol_gcp", C.c_double),
        ("itermax_gc", C.c_int),
        ("omega_pson", C.c_double),
        ("iterInter", C.c_int),
        ("pbc", C.c_int * 6),
        ("ppp", C.c_double * 6),
        ("vel_zero_gradient", C.c_int * 6),
        ("mix_GC_form", C.c_int),
        ("is_PBC_homogeneous", C.c_int),
        ("freeze_solid", C.c_int),
    ]


class RigidMotion(C.Structure):
    """PRESCRIBED_RIGID parameters and state (or_rigid_motion / fg_rigid_motion)."""
    _fields_ = [(n, C.c_double * 3) for n in ("vcent_trans", "amp", "freq", "angv_init", "ampang", "freqang",
                                              "angphase", "cent", "angv_old")]


class VelocityBC(C.Structure):
    """Outer velocity boundary data (or_velocity_bc / fg_velocity_bc): type
    per face x1, x2, y1, y2, z1, z2 (1 Dirichlet, 2 zero gradient, 3
    pulsatile inflow, 4 symmetry, 5 periodic, 6 user specified), (u, v, w)
    values and frequencies per face, the time and the channel-profile
    bounds (input.dat keys of MAIN.F90:196-207)."""
    _fields_ = [("type", C.c_int * 6), ("val", (C.c_double * 3) * 6), ("freq", (C.c_double * 3) * 6),
                ("time", C.c_double), ("yOrigin", C.c_double), ("yout", C.c_double), ("zOrigin", C.c_double),
                ("zout", C.c_double)]


class Stats(C.Structure):
    _fields_ = [
        ("outer_iterations", C.c_int),
        ("vcycles", C.c_int),
        ("maxres", C.c_double),
        ("maxres2", C.c_double),
        ("relres", C.c_double),
        ("seconds", C.c_double),
    ]


def build() -> str:
    """Compile the restatement with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
            os.path.join(_HERE, "feicar_oracle.c")
        ):
            build()
        L = C.CDLL(_LIB)
        P = C.c_void_p
        dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.or_case_create.restype = P
        L.or_case_create.argtypes = [C.c_int] * 3 + [dp] * 3 + [C.c_int] * 3
        L.or_case_destroy.argtypes = [P]
        L.or_case_dims.argtypes = [P, C.POINTER(C.c_int)]
        L.or_case_level_dims.argtypes = [P, C.c_int, C.POINTER(C.c_int)]
        L.or_case_add_body.argtypes = [P, C.c_int, C.c_int, dp,
                                       np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS"),
                                       C.c_int, C.c_double, C.c_int]
        L.or_case_update_body.argtypes = [P, C.c_int, dp]
        L.or_set_iblank_body_fast.argtypes = [P, C.c_int, C.c_int]
        L.or_gcm_set_internal_boundary.argtypes = [P, C.c_double, C.c_double]
        L.or_mg_prepare.argtypes = [P]
        L.or_get_field_i8.argtypes = [P, C.c_int, C.c_void_p]
        L.or_get_counts.argtypes = [P, C.POINTER(C.c_int)]
        L.or_get_ghosts.argtypes = [P] + [C.c_void_p] * 9
        L.or_get_deads.argtypes = [P] + [C.c_void_p] * 8
        L.or_get_mg_mask.argtypes = [P, C.c_int, C.c_int, C.c_void_p]
        L.or_solve_poisson.argtypes = [P] + [C.c_void_p] * 5 + [C.POINTER(Params), C.POINTER(Stats)]
        L.or_ghostcell_pressure.argtypes = [P] + [C.c_void_p] * 5 + [C.POINTER(Params), C.POINTER(C.c_int)]
        L.or_calc_residual.restype = C.c_double
        L.or_calc_residual.argtypes = [P, C.c_void_p, C.c_void_p]
        L.or_relres.restype = C.c_double
        L.or_relres.argtypes = [P, C.c_void_p, C.c_void_p]
        L.or_tdma.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_int]
        L.or_invert8.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_enforce_p_compatibility.argtypes = [P, C.c_void_p, C.POINTER(Params)]
        L.or_get_pgrad.argtypes = [P, C.c_int, C.c_void_p]
        L.or_set_pgrad.argtypes = [P, C.c_int, C.c_void_p]
        L.or_face_vel.argtypes = [P] + [C.c_void_p] * 9
        L.or_move_body.argtypes = [P, C.c_int, C.POINTER(RigidMotion), C.c_int, C.c_double, C.c_double,
                                   C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.or_get_body_markers.argtypes = [P, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_rhs_poisson.argtypes = [P] + [C.c_void_p] * 7 + [C.c_double, C.c_void_p, C.POINTER(C.c_double),
                                                             C.POINTER(C.c_double)]
        L.or_correct_vel.argtypes = [P, C.c_void_p, C.c_double] + [C.c_void_p] * 6
        L.or_update_pressure.argtypes = [P, C.c_void_p, C.c_void_p]
        L.or_set_solve_ad.argtypes = [P, C.c_double, C.c_double, C.c_void_p]
        L.or_body_intercept_values.argtypes = [P, C.c_int, C.c_double] + [C.c_void_p] * 4
        L.or_ghostcell_velocity.argtypes = [P] + [C.c_void_p] * 5 + [C.c_double, C.c_int, C.c_double,
                                                                     C.POINTER(C.c_int)]
        L.or_itsolv_ad.argtypes = [P] + [C.c_void_p] * 6 + [C.c_double, C.c_double]
        L.or_enforce_global_mass_consv.argtypes = [P] + [C.c_void_p] * 7
        L.or_set_outer_velocity_bc.argtypes = [P] + [C.c_void_p] * 4 + [C.POINTER(VelocityBC)]
        L.or_set_outer_ghost_velocity.argtypes = [P] + [C.c_void_p] * 4
        L.or_solve_ad.argtypes = ([P] + [C.c_void_p] * 13 + [C.c_double, C.c_double, C.POINTER(VelocityBC),
                                                            C.c_double, C.c_int, C.c_double, C.c_int, C.c_double,
                                                            C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_void_p])
        L.or_calc_residual_ad.argtypes = [P] + [C.c_void_p] * 6 + [C.c_double, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def default_params(**kw) -> Params:
    """Reference-mode parameters (input.dat keys of MAIN.F90:214-254)."""
    p = Params()
    p.it_solver_type = OR_SOLVER_MG
    p.itermax_pson = kw.get("itermax_pson", 200)
    p.restol_pson = kw.get("restol_pson", 1e-10)
    p.restol_gcp = kw.get("restol_gcp", 1e-10)
    p.itermax_gc = kw.get("itermax_gc", 50)
    p.omega_pson = kw.get("omega_pson", 1.2)
    p.iterInter = kw.get("iterInter", 4)
    for f in range(6):
        p.pbc[f] = kw.get("pbc", [OR_PBC_NEUMANN] * 6)[f]
        p.ppp[f] = kw.get("ppp", [0.0] * 6)[f]
        p.vel_zero_gradient[f] = kw.get("vzg", [0] * 6)[f]
    p.mix_GC_form = kw.get("mix_GC_form", 0)
    p.is_PBC_homogeneous = kw.get("is_PBC_homogeneous", 1)
    p.freeze_solid = kw.get("freeze_solid", 1)
    if kw.get("lsor"):
        p.it_solver_type = OR_SOLVER_LSOR
    return p


class OracleCase:
    """One grid + bodies + GCM state + MG hierarchy of the restatement."""

    def __init__(self, grid, mgrids=(0, 0, 0)):
        self.grid = grid
        L = lib()
        self.h = L.or_case_create(
            grid.nx, grid.ny, grid.nz,
            np.ascontiguousarray(grid.xn, dtype=np.float64),
            np.ascontiguousarray(grid.yn, dtype=np.float64),
            np.ascontiguousarray(grid.zn, dtype=np.float64), *mgrids)
        if not self.h:
            raise ValueError("or_case_create failed")
        d = (C.c_int * 4)()
        L.or_case_dims(self.h, d)
        self.mLevel = d[3]

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_case_destroy(self.h)
            self.h = None

    @property
    def shape(self):
        return self.grid.shape

    def level_dims(self, lev):
        d = (C.c_int * 3)()
        lib().or_case_level_dims(self.h, lev, d)
        return tuple(d)

    def add_body(self, body):
        xyz = np.ascontiguousarray(body.verts, dtype=np.float64).ravel()
        tri = np.ascontiguousarray(body.tri, dtype=np.int32).ravel()
        rc = lib().or_case_add_body(self.h, body.nvert, body.ntri, xyz, tri, body.surface,
                                    body.membrane_tkns, body.body_dim)
        if rc:
            raise ValueError(f"or_case_add_body -> {rc}")

    def update_body(self, ibody, verts):
        rc = lib().or_case_update_body(self.h, ibody, np.ascontiguousarray(verts, np.float64).ravel())
        if rc:
            raise ValueError(f"or_case_update_body -> {rc}")

    def set_iblank(self, ntime=1, ntime_start=0):
        return lib().or_set_iblank_body_fast(self.h, ntime, ntime_start)

    def gcm(self, pln=2.0, plnD=2.0):
        return lib().or_gcm_set_internal_boundary(self.h, pln, plnD)

    def mg_prepare(self):
        return lib().or_mg_prepare(self.h)

    def field(self, which):
        out = np.zeros(self.shape, dtype=np.int8, order="F")
        lib().or_get_field_i8(self.h, which, _ptr(out))
        return out

    def mg_mask(self, lev, which):
        I, J, K = self.level_dims(lev)
        out = np.zeros((I + 2, J + 2, K + 2), dtype=np.int8, order="F")
        lib().or_get_mg_mask(self.h, lev, which, _ptr(out))
        return out

    def counts(self):
        d = (C.c_int * 6)()
        lib().or_get_counts(self.h, d)
        keys = ["nGhost", "nDead", "nWarnSide", "nHostFail", "nStencilSolid", "nFallbackDead"]
        return dict(zip(keys, list(d)))

    def ghosts(self):
        n = self.counts()["nGhost"]
        r = dict(ijk=np.zeros((n, 3), np.int32), cell=np.zeros((n, 3), np.int32),
                 coefN=np.zeros((n, 8)), coefD=np.zeros((n, 8)), bi=np.zeros((n, 3)),
                 ip=np.zeros((n, 3)), probe=np.zeros(n), closest=np.zeros(n, np.int32),
                 alpha=np.zeros(n))
        lib().or_get_ghosts(self.h, *[_ptr(r[k]) for k in
                                      ["ijk", "cell", "coefN", "coefD", "bi", "ip", "probe", "closest", "alpha"]])
        return r

    def deads(self):
        n = self.counts()["nDead"]
        r = dict(ijk=np.zeros((n, 3), np.int32), cell=np.zeros((n, 3), np.int32),
                 coefN=np.zeros((n, 8)), coefD=np.zeros((n, 8)), bi=np.zeros((n, 3)),
                 ip=np.zeros((n, 3)), probe=np.zeros(n), closest=np.zeros(n, np.int32))
        lib().or_get_deads(self.h, *[_ptr(r[k]) for k in
                                     ["ijk", "cell", "coefN", "coefD", "bi", "ip", "probe", "closest"]])
        return r

    def solve_poisson(self, p, div, p_old=None, params=None, dpdn_g=None, dpdn_d=None):
        """CORE_POISSON.F90:83-200 on Fortran-ordered float64 arrays (p is
        updated in place).  Returns (status, stats dict)."""
        assert p.flags.f_contiguous and div.flags.f_contiguous
        prm = params or default_params()
        st = Stats()
        rc = lib().or_solve_poisson(self.h, _ptr(p), _ptr(div), _ptr(p_old), _ptr(dpdn_g),
                                    _ptr(dpdn_d), C.byref(prm), C.byref(st))
        return rc, {k: getattr(st, k) for k, _ in Stats._fields_}

    def ghostcell_pressure(self, p, div, p_old=None, params=None):
        prm = params or default_params()
        it = C.c_int()
        rc = lib().or_ghostcell_pressure(self.h, _ptr(p), _ptr(div), _ptr(p_old), None, None,
                                         C.byref(prm), C.byref(it))
        return rc, it.value

    def pgrad_shape(self, face):
        NX, NY, NZ = self.grid.nx + 2, self.grid.ny + 2, self.grid.nz + 2
        return [(NY, NZ), (NY, NZ), (NX, NZ), (NX, NZ), (NX, NY), (NX, NY)][face]

    def get_pgrad(self, face):
        out = np.zeros(self.pgrad_shape(face), order="F")
        lib().or_get_pgrad(self.h, face, _ptr(out))
        return out

    def set_pgrad(self, face, values):
        a = np.asfortranarray(values, dtype=np.float64)
        assert a.shape == self.pgrad_shape(face)
        lib().or_set_pgrad(self.h, face, _ptr(a))

    def enforce_p_compatibility(self, p, params=None):
        """GCM_GHOSTCELL_UPDATE.F90:865-1003 on p: updates the face gradients."""
        prm = params or default_params()
        lib().or_enforce_p_compatibility(self.h, _ptr(np.asfortranarray(p)), C.byref(prm))

    # the projection steps either side of the solve (Fortran-ordered arrays)
    def face_vel(self, u, v, w, bcxu, bcyv, bczw):
        out = [np.zeros(self.shape, order="F") for _ in range(3)]
        lib().or_face_vel(self.h, *[_ptr(np.asfortranarray(a)) for a in (u, v, w, bcxu, bcyv, bczw)],
                          *[_ptr(a) for a in out])
        return out

    def rhs_poisson(self, fu, fv, fw, bcxu, bcyv, bczw, vzg, dt):
        """Arrays are updated in place (mass conservation); returns (div, sumd, resdiv)."""
        div = np.zeros(self.shape, order="F")
        sd, rd = C.c_double(0.0), C.c_double(0.0)
        vz = np.ascontiguousarray(vzg, dtype=np.int32)
        lib().or_rhs_poisson(self.h, *[_ptr(a) for a in (fu, fv, fw, bcxu, bcyv, bczw, vz)], dt, _ptr(div),
                             C.byref(sd), C.byref(rd))
        return div, sd.value, rd.value

    def correct_vel(self, pp, dt, u, v, w):
        """u, v, w updated in place; returns (dpdx, dpdy, dpdz)."""
        g = [np.zeros(self.shape, order="F") for _ in range(3)]
        lib().or_correct_vel(self.h, _ptr(np.asfortranarray(pp)), dt, _ptr(u), _ptr(v), _ptr(w), *[_ptr(a) for a in g])
        return g

    def update_pressure(self, pp):
        """pp updated in place; returns p (= pp after the update)."""
        p = np.zeros(self.shape, order="F")
        lib().or_update_pressure(self.h, _ptr(pp), _ptr(p))
        return p

    def body_intercept_values(self, ntime, dt):
        """(ubi_ghost (ng,3), ubi_dead (nd,3), dpdn_ghost, dpdn_dead):
        GCM_SetBodyInterceptValues on the current rows."""
        cnt = self.counts()
        ng, nd = cnt["nGhost"], cnt["nDead"]
        ug, ud, pg, pd = np.zeros((ng, 3)), np.zeros((nd, 3)), np.zeros(ng), np.zeros(nd)
        lib().or_body_intercept_values(self.h, ntime, dt, _ptr(ug), _ptr(ud), _ptr(pg), _ptr(pd))
        return ug, ud, pg, pd

    def ghostcell_velocity(self, u, v, w, ubi_g, ubi_d, pld, itermax_gc, restol_gcv):
        """u, v, w (Fortran-ordered) updated in place; returns (status, sweeps)."""
        it = C.c_int(0)
        rc = lib().or_ghostcell_velocity(self.h, _ptr(u), _ptr(v), _ptr(w), _ptr(np.ascontiguousarray(ubi_g)),
                                         _ptr(np.ascontiguousarray(ubi_d)), pld, itermax_gc, restol_gcv,
                                         C.byref(it))
        return rc, it.value

    # momentum line SOR (CORE_SET_SOLVERS.F90 set_solve_ad, CORE_SOLVE_AD.F90)
    def set_solve_ad(self, dt, reinv):
        g = self.grid
        ad = np.zeros(2 * (g.nx + 2) + 2 * (g.ny + 2) + 2 * (g.nz + 2))
        lib().or_set_solve_ad(self.h, dt, reinv, _ptr(ad))
        return ad

    def itsolv_ad(self, ad, var, r, fu, fv, fw, half_dt, omega_ad):
        """One x/y/z line-sweep pass; var (Fortran-ordered) updated in place."""
        assert var.flags.f_contiguous
        lib().or_itsolv_ad(self.h, _ptr(ad), _ptr(var), *[_ptr(np.asfortranarray(a)) for a in (r, fu, fv, fw)],
                           half_dt, omega_ad)

    def calc_residual_ad(self, ad, var, r, fu, fv, fw, half_dt):
        m = C.c_double(0.0)
        loc = np.zeros(3, np.int32)
        lib().or_calc_residual_ad(self.h, _ptr(ad), *[_ptr(np.asfortranarray(a)) for a in (var, r, fu, fv, fw)],
                                  half_dt, C.byref(m), _ptr(loc))
        return m.value, tuple(int(x) for x in loc)

    # the outer velocity boundaries and the momentum iteration around them
    # (CORE_SET_OUTER_BC.F90, CORE_SOLVE_AD.F90:11-127); bc is the list of
    # the nine Fortran-ordered arrays bcxu, bcxv, bcxw (2, ny+2, nz+2),
    # bcyu, bcyv, bcyw (nx+2, 2, nz+2), bczu, bczv, bczw (nx+2, ny+2, 2)
    def bc_arrays(self):
        NX, NY, NZ = self.shape
        return ([np.zeros((2, NY, NZ), order="F") for _ in range(3)] +
                [np.zeros((NX, 2, NZ), order="F") for _ in range(3)] +
                [np.zeros((NX, NY, 2), order="F") for _ in range(3)])

    @staticmethod
    def _bcp(bc):
        assert len(bc) == 9 and all(a.flags.f_contiguous and a.dtype == np.float64 for a in bc)
        return (C.c_void_p * 9)(*[a.ctypes.data for a in bc])

    def enforce_global_mass_consv(self, fu, fv, fw, bcxu, bcyv, bczw, vzg):
        vz = np.ascontiguousarray(vzg, dtype=np.int32)
        lib().or_enforce_global_mass_consv(self.h, *[_ptr(a) for a in (fu, fv, fw, bcxu, bcyv, bczw, vz)])

    def set_outer_velocity_bc(self, u, v, w, bc, vb):
        """Fills the nine arrays of bc in place; returns the status."""
        bp = self._bcp(bc)
        return lib().or_set_outer_velocity_bc(self.h, *[_ptr(np.asfortranarray(a)) for a in (u, v, w)],
                                              C.cast(bp, C.c_void_p), C.byref(vb))

    def set_outer_ghost_velocity(self, u, v, w, bc):
        assert u.flags.f_contiguous and v.flags.f_contiguous and w.flags.f_contiguous
        bp = self._bcp(bc)
        lib().or_set_outer_ghost_velocity(self.h, _ptr(u), _ptr(v), _ptr(w), C.cast(bp, C.c_void_p))

    def solve_ad(self, ad, u, v, w, nlu, nlv, nlw, fu, fv, fw, bc, ubi_g, ubi_d, half_dt, omega_ad, vb, pld,
                 itermax_gc, restol_gcv, itermax_ad, restol_ad):
        """u, v, w, fu, fv, fw and bc updated in place; returns (status,
        iterations, residual, location)."""
        for a in (u, v, w, fu, fv, fw):
            assert a.flags.f_contiguous
        bp = self._bcp(bc)
        it, rm = C.c_int(0), C.c_double(0.0)
        loc = np.zeros(3, np.int32)
        rc = lib().or_solve_ad(self.h, _ptr(ad), _ptr(u), _ptr(v), _ptr(w),
                               *[_ptr(np.asfortranarray(a)) for a in (nlu, nlv, nlw)], _ptr(fu), _ptr(fv), _ptr(fw),
                               C.cast(bp, C.c_void_p), _ptr(np.ascontiguousarray(ubi_g)),
                               _ptr(np.ascontiguousarray(ubi_d)), half_dt, omega_ad, C.byref(vb), pld, itermax_gc,
                               restol_gcv, itermax_ad, restol_ad, C.byref(it), C.byref(rm), _ptr(loc))
        return rc, it.value, rm.value, tuple(int(x) for x in loc)

    def move_body(self, ibody, motion, ntime, time, dt):
        """One prescribed-motion step; motion (RigidMotion) is updated.
        Returns (ds_max, iblank_reset)."""
        ds, rs = C.c_double(0.0), C.c_int(0)
        lib().or_move_body(self.h, ibody, C.byref(motion), ntime, time, dt, C.byref(ds), C.byref(rs))
        return ds.value, rs.value

    def body_markers(self, ibody, nvert):
        xyz, uvw, dpdn = np.zeros((nvert, 3)), np.zeros((nvert, 3)), np.zeros(nvert)
        lib().or_get_body_markers(self.h, ibody, _ptr(xyz), _ptr(uvw), _ptr(dpdn))
        return xyz, uvw, dpdn

    def relres(self, p, div):
        return lib().or_relres(self.h, _ptr(p), _ptr(div))

    def calc_residual(self, p, div):
        return lib().or_calc_residual(self.h, _ptr(p), _ptr(div))


def tdma(a, b, c, r, n1, n2):
    u = np.zeros_like(r)
    lib().or_tdma(_ptr(a), _ptr(b), _ptr(c), _ptr(r), _ptr(u), n1, n2)
    return u


def invert8(a):
    """8x8 inverse with LAPACK getrf/getri semantics (column-major in/out)."""
    a = np.asfortranarray(a, dtype=np.float64)
    out = np.zeros((8, 8), order="F")
    info = C.c_int()
    lib().or_invert8(_ptr(a), _ptr(out), C.byref(info))
    return out, info.value


def set_threads(n):
    lib().or_set_threads(n)
