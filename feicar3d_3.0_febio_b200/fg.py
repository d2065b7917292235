"""Python binding of the C ABI in include/feicar_b200.h (libfeicar_b200.so).

The class :class:`Case` mirrors the Fortran subroutines of the reference's
pressure path that a time step calls, with the same names and argument
meaning (host arrays are Fortran-ordered ``(0:nx+1, 0:ny+1, 0:nz+1)``
fields, nx/ny/nz node counts):

* ``set_iblank_body_fast``        BOUNDARY_IBLANK_FAST.F90:2
* ``gcm_set_internal_boundary``   GCM_SET_BOUNDARY.F90:2
* ``mg_prepare``                  CORE_MG.F90:1365
* ``solve_poisson``               CORE_POISSON.F90:83
* ``ghostcell_pressure``          GCM_GHOSTCELL_UPDATE.F90:361

There is no fallback: without the compiled library every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# FEICAR_B200_LIB selects another build of the library (e.g. the bounds-checked
# diagnostic build of csrc/Makefile's "checked" target)
LIB_PATH = os.environ.get("FEICAR_B200_LIB") or os.path.join(_HERE, "libfeicar_b200.so")

FG_OK, FG_NOT_CONVERGED = 0, 1
FG_PBC_DIRICHLET, FG_PBC_NEUMANN = 1, 2
FG_PREC_FP64, FG_PREC_MIXED = 0, 1
FG_OUTER_RICHARDSON, FG_OUTER_FGMRES, FG_OUTER_LSOR = 0, 1, 2
STATUS = {0: "ok", 1: "not converged", 2: "image point has no host cell", 3: "allocation failed",
          4: "timeout", 5: "bad input", 6: "dead cell without body", 7: "CUDA error",
          8: "no CUDA device", 9: "rejected by admission"}


class FGError(RuntimeError):
    def __init__(self, status, what):
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")
        self.status = status


class SolverConfig(C.Structure):
    _fields_ = [
        ("precision", C.c_int),
        ("outer", C.c_int),
        ("nu1", C.c_int),
        ("nu2", C.c_int),
        ("omega", C.c_double),
        ("rtol", C.c_double),
        ("max_cycles", C.c_int),
        ("pbc", C.c_int * 6),
        ("ppp", C.c_double * 6),
        ("mgrids", C.c_int * 3),
        ("probe_length", C.c_double),
        ("probe_length_dead", C.c_double),
        ("membrane_tkns_factor", C.c_double),
        ("gauge_corner", C.c_int),
        ("restart", C.c_int),
    ]


class SolveStats(C.Structure):
    _fields_ = [
        ("cycles", C.c_int),
        ("relres", C.c_double),
        ("ghost_res", C.c_double),
        ("seconds", C.c_double),
        ("vcycle_ms", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


PROF_CLASSES = ["line_x0", "line_y0", "line_z0", "line_coarse", "residual0", "transfer", "rows",
                "coarsest"]


class Profile(C.Structure):
    _fields_ = [
        ("class_launches", C.c_longlong * 8),
        ("class_ms", C.c_double * 8),
        ("class_bytes", C.c_double * 8),
    ]

    def as_dict(self):
        return {name: {"launches": self.class_launches[i], "ms": self.class_ms[i],
                       "bytes": self.class_bytes[i]} for i, name in enumerate(PROF_CLASSES)}


_lib = None


def lib():
    """Load the CUDA library; raises when it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is not built; run __graft_entry__.build() or make -C csrc")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.c_int, C.c_double
        L.fg_version.restype = C.c_char_p
        L.fg_status_string.restype = C.c_char_p
        L.fg_status_string.argtypes = [ip]
        L.fg_device_count.argtypes = [C.POINTER(C.c_int)]
        L.fg_default_config.argtypes = [C.POINTER(SolverConfig)]
        L.fg_case_create.argtypes = [ip, ip, ip, vp, vp, vp, C.POINTER(SolverConfig), ip, C.POINTER(vp)]
        L.fg_case_destroy.argtypes = [vp]
        L.fg_case_levels.argtypes = [vp, C.POINTER(C.c_int), vp]
        L.fg_case_add_body.argtypes = [vp, ip, ip, vp, vp, ip, dp, ip]
        L.fg_case_update_body.argtypes = [vp, ip, vp]
        L.fg_set_iblank_body_fast.argtypes = [vp, vp]
        L.fg_gcm_set_internal_boundary.argtypes = [vp, vp, vp, vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.fg_get_ghost_rows.argtypes = [vp] + [vp] * 9
        L.fg_get_dead_rows.argtypes = [vp] + [vp] * 8
        L.fg_get_band.argtypes = [vp, vp]
        L.fg_case_set_geometry.argtypes = [vp, vp, vp, vp, ip, vp, vp, vp, ip, vp, vp, vp, vp, vp]
        L.fg_mg_prepare.argtypes = [vp]
        L.fg_solve_poisson.argtypes = [vp, vp, vp, vp, vp, vp, C.POINTER(SolveStats)]
        L.fg_solve_poisson_device.argtypes = [vp, vp, vp, vp, C.POINTER(SolveStats)]
        L.fg_ghostcell_pressure.argtypes = [vp, vp, vp, ip]
        L.fg_batch_create.argtypes = [ip, C.POINTER(SolverConfig), C.POINTER(vp)]
        L.fg_batch_add.argtypes = [vp, vp]
        L.fg_batch_solve_device.argtypes = [vp, vp, vp, C.POINTER(SolveStats)]
        L.fg_batch_destroy.argtypes = [vp]
        L.fg_case_set_stream.argtypes = [vp, vp]
        L.fg_launch_count.argtypes = [C.POINTER(C.c_longlong)]
        L.fg_case_profile.argtypes = [vp, ip]
        L.fg_case_solve_mode.argtypes = [vp, C.POINTER(C.c_int)]
        L.fg_calc_residual.argtypes = [vp, vp, vp, C.POINTER(C.c_double)]
        L.fg_set_pressure_gradient.argtypes = [vp, ip, vp]
        L.fg_get_pressure_gradient.argtypes = [vp, ip, vp]
        L.fg_enforce_p_compatibility.argtypes = [vp, vp, vp]
        L.fg_case_set_zero_gradient_faces.argtypes = [vp, vp]
        L.fg_calc_residual2.argtypes = [vp, vp, vp, C.POINTER(C.c_double)]
        L.fg_case_history.argtypes = [vp, vp, ip, C.POINTER(C.c_int)]
        L.fg_case_profile_read.argtypes = [vp, C.POINTER(Profile)]
        for name in ["fg_device_count", "fg_case_create", "fg_case_destroy", "fg_case_levels",
                     "fg_case_add_body", "fg_case_update_body", "fg_set_iblank_body_fast",
                     "fg_gcm_set_internal_boundary", "fg_get_ghost_rows", "fg_get_dead_rows",
                     "fg_get_band", "fg_case_set_geometry", "fg_mg_prepare", "fg_solve_poisson",
                     "fg_solve_poisson_device", "fg_ghostcell_pressure", "fg_batch_create",
                     "fg_batch_add", "fg_batch_solve_device", "fg_batch_destroy", "fg_case_set_stream",
                     "fg_launch_count", "fg_case_profile", "fg_case_profile_read",
                     "fg_case_history", "fg_case_solve_mode", "fg_calc_residual", "fg_calc_residual2",
                     "fg_set_pressure_gradient", "fg_get_pressure_gradient", "fg_enforce_p_compatibility",
                     "fg_case_set_zero_gradient_faces"]:
            getattr(L, name).restype = ip
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc, what, ok=(FG_OK,)):
    if rc not in ok:
        msg = lib().fg_status_string(rc).decode()
        raise FGError(rc, f"{what} [{msg}]")
    return rc


def default_config(**kw) -> SolverConfig:
    cfg = SolverConfig()
    lib().fg_default_config(C.byref(cfg))
    for k, v in kw.items():
        if k in ("pbc", "ppp", "mgrids"):
            arr = getattr(cfg, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(cfg, k, v)
    return cfg


def launch_count() -> int:
    """Kernels the library has launched in this process."""
    n = C.c_longlong(0)
    _check(lib().fg_launch_count(C.byref(n)), "fg_launch_count")
    return n.value


def device_count() -> int:
    n = C.c_int(0)
    lib().fg_device_count(C.byref(n))
    return n.value


class Case:
    """One grid + bodies + device-resident GCM state and MG hierarchy."""

    def __init__(self, grid, config: SolverConfig | None = None, device: int = 0):
        self.grid = grid
        self.cfg = config or default_config()
        h = C.c_void_p()
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (grid.xn, grid.yn, grid.zn)]
        self._keep = xs
        _check(lib().fg_case_create(grid.nx, grid.ny, grid.nz, _p(xs[0]), _p(xs[1]), _p(xs[2]),
                                    C.byref(self.cfg), device, C.byref(h)), "fg_case_create")
        self.h = h
        self.nGhost = 0
        self.nDead = 0

    def close(self):
        if getattr(self, "h", None):
            lib().fg_case_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return self.grid.shape

    def levels(self):
        n = C.c_int()
        dims = np.zeros(3 * 16, np.int32)
        _check(lib().fg_case_levels(self.h, C.byref(n), _p(dims)), "fg_case_levels")
        return [tuple(dims[3 * i:3 * i + 3]) for i in range(n.value)]

    # -------------------------------------------------------- geometry
    def add_body(self, body):
        xyz = np.ascontiguousarray(body.verts, dtype=np.float64).ravel()
        tri = np.ascontiguousarray(body.tri, dtype=np.int32).ravel()
        _check(lib().fg_case_add_body(self.h, body.nvert, body.ntri, _p(xyz), _p(tri), body.surface,
                                      body.membrane_tkns, body.body_dim), "fg_case_add_body")

    def update_body(self, ibody, verts):
        xyz = np.ascontiguousarray(verts, dtype=np.float64).ravel()
        _check(lib().fg_case_update_body(self.h, ibody, _p(xyz)), "fg_case_update_body")

    def set_iblank_body_fast(self):
        ib = np.zeros(self.shape, np.int8, order="F")
        _check(lib().fg_set_iblank_body_fast(self.h, _p(ib)), "fg_set_iblank_body_fast")
        return ib

    def gcm_set_internal_boundary(self):
        ib = np.zeros(self.shape, np.int8, order="F")
        gh = np.zeros(self.shape, np.int8, order="F")
        dd = np.zeros(self.shape, np.int8, order="F")
        ng, nd = C.c_int(), C.c_int()
        rc = lib().fg_gcm_set_internal_boundary(self.h, _p(ib), _p(gh), _p(dd), C.byref(ng), C.byref(nd))
        _check(rc, "fg_gcm_set_internal_boundary")
        self.nGhost, self.nDead = ng.value, nd.value
        return ib, gh, dd

    def band(self):
        b = np.zeros(self.shape, np.int8, order="F")
        _check(lib().fg_get_band(self.h, _p(b)), "fg_get_band")
        return b

    def ghost_rows(self):
        n = self.nGhost
        r = dict(ijk=np.zeros((n, 3), np.int32), cell=np.zeros((n, 3), np.int32),
                 coefN=np.zeros((n, 8)), coefD=np.zeros((n, 8)), bi=np.zeros((n, 3)),
                 ip=np.zeros((n, 3)), probe=np.zeros(n), closest=np.zeros(n, np.int32),
                 alpha=np.zeros(n))
        _check(lib().fg_get_ghost_rows(self.h, *[_p(r[k]) for k in
                                                 ["ijk", "cell", "coefN", "coefD", "bi", "ip", "probe",
                                                  "closest", "alpha"]]), "fg_get_ghost_rows")
        return r

    def dead_rows(self):
        n = self.nDead
        r = dict(ijk=np.zeros((n, 3), np.int32), cell=np.zeros((n, 3), np.int32),
                 coefN=np.zeros((n, 8)), coefD=np.zeros((n, 8)), bi=np.zeros((n, 3)),
                 ip=np.zeros((n, 3)), probe=np.zeros(n), closest=np.zeros(n, np.int32))
        _check(lib().fg_get_dead_rows(self.h, *[_p(r[k]) for k in
                                                ["ijk", "cell", "coefN", "coefD", "bi", "ip", "probe",
                                                 "closest"]]), "fg_get_dead_rows")
        return r

    def set_geometry(self, iblank, ghost, dead, ghosts: dict, deads: dict):
        """Masks and interpolation rows computed elsewhere (e.g. a host that
        keeps its own GCM setup)."""
        arrs = [np.asfortranarray(a, dtype=np.int8) for a in (iblank, ghost, dead)]
        g = {k: np.ascontiguousarray(ghosts[k]) for k in ("ijk", "cell", "coefN")}
        d = {k: np.ascontiguousarray(deads[k]) for k in ("ijk", "cell", "coefN", "probe", "ip")}
        g["ijk"] = g["ijk"].astype(np.int32); g["cell"] = g["cell"].astype(np.int32)
        d["ijk"] = d["ijk"].astype(np.int32); d["cell"] = d["cell"].astype(np.int32)
        self._geo_keep = (arrs, g, d)
        _check(lib().fg_case_set_geometry(
            self.h, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]), len(g["ijk"]), _p(g["ijk"]), _p(g["cell"]),
            _p(g["coefN"]), len(d["ijk"]), _p(d["ijk"]), _p(d["cell"]), _p(d["coefN"]), _p(d["probe"]),
            _p(d["ip"])), "fg_case_set_geometry")
        self.nGhost, self.nDead = len(g["ijk"]), len(d["ijk"])

    def mg_prepare(self):
        _check(lib().fg_mg_prepare(self.h), "fg_mg_prepare")

    # ----------------------------------------------------------- solve
    def solve_poisson(self, p, div, p_old=None, dpdn_ghost=None, dpdn_dead=None,
                      allow_not_converged=False):
        """p is updated in place (Fortran-ordered float64 field)."""
        assert p.dtype == np.float64 and p.flags.f_contiguous and p.shape == self.shape
        div = np.asfortranarray(div, dtype=np.float64)
        st = SolveStats()
        rc = lib().fg_solve_poisson(self.h, _p(p), _p(div), _p(p_old), _p(dpdn_ghost), _p(dpdn_dead),
                                    C.byref(st))
        ok = (FG_OK, FG_NOT_CONVERGED) if allow_not_converged else (FG_OK,)
        _check(rc, "fg_solve_poisson", ok)
        return st.as_dict()

    def solve_poisson_device(self, d_p: int, d_div: int, allow_not_converged=False, d_p_old=None,
                             d_dpdn_ghost=None, d_dpdn_dead=None):
        """Device pointers (ints) of Fortran-layout float64 fields (and of
        the previous pressure and dp/dn data, when given)."""
        st = SolveStats()
        L = lib()
        if d_p_old is None and d_dpdn_ghost is None and d_dpdn_dead is None:
            rc = L.fg_solve_poisson_device(self.h, C.c_void_p(d_p), C.c_void_p(d_div), None, C.byref(st))
        else:
            if not getattr(L, "_bc_ready", False):
                L.fg_solve_poisson_device_bc.argtypes = [C.c_void_p] * 6 + [C.POINTER(SolveStats)]
                L.fg_solve_poisson_device_bc.restype = C.c_int
                L._bc_ready = True
            vp = lambda x: C.c_void_p(x) if x else None
            rc = L.fg_solve_poisson_device_bc(self.h, C.c_void_p(d_p), C.c_void_p(d_div), vp(d_p_old),
                                              vp(d_dpdn_ghost), vp(d_dpdn_dead), C.byref(st))
        ok = (FG_OK, FG_NOT_CONVERGED) if allow_not_converged else (FG_OK,)
        _check(rc, "fg_solve_poisson_device", ok)
        return st.as_dict()

    def set_stream(self, stream_handle: int | None):
        """Order the case's work on a caller's cudaStream_t (an int handle,
        e.g. ``torch.cuda.current_stream().cuda_stream``); None: own stream."""
        _check(lib().fg_case_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None),
               "fg_case_set_stream")

    def history(self) -> np.ndarray:
        """Relative residual after each cycle of the last solve."""
        n = C.c_int(0)
        _check(lib().fg_case_history(self.h, None, 0, C.byref(n)), "fg_case_history")
        out = np.zeros(n.value)
        _check(lib().fg_case_history(self.h, _p(out), n.value, C.byref(n)), "fg_case_history")
        return out

    def solve_mode(self) -> int:
        """1 when the last solve was one CUDA graph launch, 0 when the host
        drove its kernels step by step."""
        m = C.c_int(0)
        _check(lib().fg_case_solve_mode(self.h, C.byref(m)), "fg_case_solve_mode")
        return m.value

    def profile(self, enable=True):
        _check(lib().fg_case_profile(self.h, 1 if enable else 0), "fg_case_profile")

    def profile_read(self) -> dict:
        pr = Profile()
        _check(lib().fg_case_profile_read(self.h, C.byref(pr)), "fg_case_profile_read")
        return pr.as_dict()

    def calc_residual(self, p, div) -> float:
        """The reference's residual measure (CORE_POISSON.F90:460-551)."""
        v = C.c_double(0.0)
        _check(lib().fg_calc_residual(self.h, _p(np.asfortranarray(p)), _p(np.asfortranarray(div)), C.byref(v)),
               "fg_calc_residual")
        return v.value

    def calc_residual2(self, p, p_temp) -> float:
        """The reference's iterate change (CORE_POISSON.F90:679-724)."""
        v = C.c_double(0.0)
        _check(lib().fg_calc_residual2(self.h, _p(np.asfortranarray(p)), _p(np.asfortranarray(p_temp)),
                                       C.byref(v)), "fg_calc_residual2")
        return v.value

    def pgrad_shape(self, face):
        NX, NY, NZ = self.grid.nx + 2, self.grid.ny + 2, self.grid.nz + 2
        return [(NY, NZ), (NY, NZ), (NX, NZ), (NX, NZ), (NX, NY), (NX, NY)][face]

    def set_pressure_gradient(self, face, values):
        a = np.asfortranarray(values, dtype=np.float64)
        assert a.shape == self.pgrad_shape(face)
        _check(lib().fg_set_pressure_gradient(self.h, face, _p(a)), "fg_set_pressure_gradient")

    def get_pressure_gradient(self, face):
        out = np.zeros(self.pgrad_shape(face), order="F")
        _check(lib().fg_get_pressure_gradient(self.h, face, _p(out)), "fg_get_pressure_gradient")
        return out

    def enforce_p_compatibility(self, p, vel_zero_gradient):
        v = np.ascontiguousarray(vel_zero_gradient, dtype=np.int32)
        _check(lib().fg_enforce_p_compatibility(self.h, _p(np.asfortranarray(p)), _p(v)),
               "fg_enforce_p_compatibility")

    def set_zero_gradient_faces(self, vel_zero_gradient=None):
        v = None if vel_zero_gradient is None else np.ascontiguousarray(vel_zero_gradient, dtype=np.int32)
        self._vzg = v
        _check(lib().fg_case_set_zero_gradient_faces(self.h, _p(v)), "fg_case_set_zero_gradient_faces")

    def ghostcell_pressure(self, p, p_old=None, iterations=1):
        _check(lib().fg_ghostcell_pressure(self.h, _p(p), _p(p_old), iterations), "fg_ghostcell_pressure")


class Batch:
    """Many cases solved together: one launch per multigrid stage."""

    def __init__(self, config: SolverConfig | None = None, device: int = 0):
        self.cfg = config or default_config()
        h = C.c_void_p()
        _check(lib().fg_batch_create(device, C.byref(self.cfg), C.byref(h)), "fg_batch_create")
        self.h = h
        self.cases = []

    def add(self, case: Case):
        _check(lib().fg_batch_add(self.h, case.h), "fg_batch_add")
        self.cases.append(case)

    def solve_device(self, d_ps, d_divs, allow_not_converged=False):
        n = len(self.cases)
        P = (C.c_void_p * n)(*[C.c_void_p(x) for x in d_ps])
        D = (C.c_void_p * n)(*[C.c_void_p(x) for x in d_divs])
        st = SolveStats()
        rc = lib().fg_batch_solve_device(self.h, P, D, C.byref(st))
        ok = (FG_OK, FG_NOT_CONVERGED) if allow_not_converged else (FG_OK,)
        _check(rc, "fg_batch_solve_device", ok)
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            lib().fg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ serving
class ServeRequest(C.Structure):
    _fields_ = [
        ("id", C.c_longlong),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xn", C.c_void_p), ("yn", C.c_void_p), ("zn", C.c_void_p),
        ("nvert", C.c_int), ("ntri", C.c_int),
        ("xyz", C.c_void_p), ("tri", C.c_void_p),
        ("surface_type", C.c_int),
        ("membrane_tkns", C.c_double),
        ("nsteps", C.c_int),
        ("div", C.c_void_p),
        ("p", C.c_void_p),
        ("p0", C.c_void_p),
    ]


class ServeResult(C.Structure):
    _fields_ = [
        ("id", C.c_longlong),
        ("status", C.c_int),
        ("steps_done", C.c_int),
        ("cycles_max", C.c_int),
        ("relres_max", C.c_double),
        ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_longlong), ("finished", C.c_longlong), ("pending", C.c_longlong),
        ("active", C.c_int), ("active_peak", C.c_int),
        ("bytes_in_use", C.c_size_t),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _serve_lib():
    L = lib()
    if not getattr(L, "_serve_ready", False):
        vp, ip = C.c_void_p, C.c_int
        L.fg_case_estimate_bytes.argtypes = [ip, ip, ip, C.POINTER(SolverConfig), C.POINTER(C.c_size_t)]
        L.fg_server_create.argtypes = [ip, C.POINTER(SolverConfig), C.c_size_t, ip, C.POINTER(vp)]
        L.fg_server_submit.argtypes = [vp, C.POINTER(ServeRequest)]
        L.fg_server_poll.argtypes = [vp, vp, ip, C.POINTER(C.c_int)]
        L.fg_server_wait_idle.argtypes = [vp, C.c_double]
        L.fg_server_info.argtypes = [vp, C.POINTER(ServerStats)]
        L.fg_server_clock.argtypes = [vp]
        L.fg_server_clock.restype = C.c_double
        L.fg_server_destroy.argtypes = [vp]
        for name in ["fg_case_estimate_bytes", "fg_server_create", "fg_server_submit", "fg_server_poll",
                     "fg_server_wait_idle", "fg_server_info", "fg_server_destroy"]:
            getattr(L, name).restype = ip
        L._serve_ready = True
    return L


def estimate_bytes(grid, config: SolverConfig | None = None) -> int:
    n = C.c_size_t(0)
    cfg = config or default_config()
    _check(_serve_lib().fg_case_estimate_bytes(grid.nx, grid.ny, grid.nz, C.byref(cfg), C.byref(n)),
           "fg_case_estimate_bytes")
    return n.value


class Server:
    """A request stream over many cases (fg_server_*): requests are admitted
    as slots and device memory free up and their steps overlap on the
    device.  The host arrays handed to :meth:`submit` are kept alive here
    until the request's result has been polled."""

    def __init__(self, config: SolverConfig | None = None, budget_bytes: int = 150 * 10**9,
                 max_active: int = 8, device: int = 0):
        self.cfg = config or default_config()
        h = C.c_void_p()
        _check(_serve_lib().fg_server_create(device, C.byref(self.cfg), int(budget_bytes), max_active,
                                             C.byref(h)), "fg_server_create")
        self.h = h
        self._keep = {}

    def clock(self) -> float:
        return _serve_lib().fg_server_clock(self.h)

    def submit(self, rid, grid, body, divs, outs=None, p0=None):
        """divs / outs: lists of Fortran-ordered float64 fields (outs may be
        None: nothing is copied back)."""
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (grid.xn, grid.yn, grid.zn)]
        xyz = np.ascontiguousarray(body.verts, dtype=np.float64).ravel()
        tri = np.ascontiguousarray(body.tri, dtype=np.int32).ravel()
        n = len(divs)
        for d in divs:
            assert d.dtype == np.float64 and d.flags.f_contiguous and d.shape == grid.shape
        dptrs = (C.c_void_p * n)(*[d.ctypes.data for d in divs])
        pptrs = None
        if outs is not None:
            assert len(outs) == n
            for o in outs:
                assert o.dtype == np.float64 and o.flags.f_contiguous and o.shape == grid.shape
            pptrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        r = ServeRequest()
        r.id = rid
        r.nx, r.ny, r.nz = grid.nx, grid.ny, grid.nz
        r.xn, r.yn, r.zn = (a.ctypes.data for a in xs)
        r.nvert, r.ntri = body.nvert, body.ntri
        r.xyz, r.tri = xyz.ctypes.data, tri.ctypes.data
        r.surface_type, r.membrane_tkns = body.surface, body.membrane_tkns
        r.nsteps = n
        r.div = C.cast(dptrs, C.c_void_p)
        r.p = C.cast(pptrs, C.c_void_p) if pptrs is not None else None
        r.p0 = p0.ctypes.data if p0 is not None else None
        rc = _serve_lib().fg_server_submit(self.h, C.byref(r))
        _check(rc, "fg_server_submit")
        self._keep[rid] = (xs, xyz, tri, divs, outs, dptrs, pptrs, p0)

    def poll(self, capacity=1024):
        out = (ServeResult * capacity)()
        n = C.c_int(0)
        _check(_serve_lib().fg_server_poll(self.h, out, capacity, C.byref(n)), "fg_server_poll")
        res = [out[i].as_dict() for i in range(n.value)]
        for r in res:
            self._keep.pop(r["id"], None)
        return res

    def wait_idle(self, timeout_s=600.0):
        _check(_serve_lib().fg_server_wait_idle(self.h, timeout_s), "fg_server_wait_idle")

    def info(self) -> dict:
        st = ServerStats()
        _check(_serve_lib().fg_server_info(self.h, C.byref(st)), "fg_server_info")
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            _serve_lib().fg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- autotuner
LINE_FAMILIES = {0: {1: "x_registers", 2: "x_registers_32_lanes", 3: "x_shared_memory"},
                 1: {1: "yz_registers_thomas", 2: "yz_block_pcr", 3: "yz_warp_per_line",
                     4: "yz_block_pcr_loads_first", 5: "yz_block_pcr_4_rows",
                     6: "yz_block_pcr_both_colours_one_launch"}}


class RigidMotion(C.Structure):
    """fg_rigid_motion: PRESCRIBED_RIGID parameters and state."""
    _fields_ = [(n, C.c_double * 3) for n in ("vcent_trans", "amp", "freq", "angv_init", "ampang", "freqang",
                                              "angphase", "cent", "angv_old")]


def move_body(case, ibody, motion, ntime, time, dt):
    """One prescribed-motion step on the device; returns (ds_max, iblank_reset)."""
    L = lib()
    if not getattr(L, "_move_ready", False):
        L.fg_move_body.argtypes = [C.c_void_p, C.c_int, C.POINTER(RigidMotion), C.c_int, C.c_double, C.c_double,
                                   C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.fg_get_body_markers.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.fg_move_body.restype = C.c_int
        L.fg_get_body_markers.restype = C.c_int
        L._move_ready = True
    ds, rs = C.c_double(0.0), C.c_int(0)
    _check(L.fg_move_body(case.h, ibody, C.byref(motion), ntime, time, dt, C.byref(ds), C.byref(rs)), "fg_move_body")
    return ds.value, rs.value


def body_markers(case, ibody, nvert):
    L = lib()
    xyz, uvw, dpdn = np.zeros((nvert, 3)), np.zeros((nvert, 3)), np.zeros(nvert)
    L.fg_get_body_markers.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.fg_get_body_markers.restype = C.c_int
    _check(L.fg_get_body_markers(case.h, ibody, _p(xyz), _p(uvw), _p(dpdn)), "fg_get_body_markers")
    return xyz, uvw, dpdn


class Tuning(C.Structure):
    _fields_ = [
        ("nlevels", C.c_int),
        ("line_variant", (C.c_int * 3) * 12),
        ("line_us", (C.c_double * 3) * 12),
        ("nu1", C.c_int), ("nu2", C.c_int),
        ("solve_ms", C.c_double * 4),
        ("tuned", C.c_int),
        ("nu1_coarse", C.c_int), ("nu2_coarse", C.c_int),
        ("solve_ms_coarse", C.c_double * 2),
        ("coarse_from", C.c_int),
    ]

    def as_dict(self):
        levels = []
        for L in range(self.nlevels):
            row = {}
            for a, name in enumerate("xyz"):
                v = self.line_variant[L][a]
                if v:
                    row[name] = {"family": LINE_FAMILIES[0 if a == 0 else 1][v],
                                 "us": round(self.line_us[L][a], 2)}
            levels.append(row)
        return {"levels": levels, "nu1": self.nu1, "nu2": self.nu2,
                "solve_ms_nu11_21_22_33": [round(x, 3) for x in self.solve_ms], "tuned": bool(self.tuned),
                "nu_coarse": [self.nu1_coarse, self.nu2_coarse], "coarse_from": self.coarse_from}


def _tune_lib():
    L = lib()
    if not getattr(L, "_tune_ready", False):
        vp = C.c_void_p
        L.fg_batch_autotune.argtypes = [vp, vp, vp, C.POINTER(Tuning)]
        L.fg_batch_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.fg_case_autotune.argtypes = [vp, vp, vp, C.POINTER(Tuning)]
        L.fg_batch_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.fg_case_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        for n in ("fg_batch_autotune", "fg_batch_get_tuning", "fg_case_autotune", "fg_batch_set_tuning",
                  "fg_case_set_tuning"):
            getattr(L, n).restype = C.c_int
        L._tune_ready = True
    return L


def batch_autotune(batch, d_ps, d_divs) -> dict:
    n = len(batch.cases)
    P = (C.c_void_p * n)(*[C.c_void_p(x) for x in d_ps])
    D = (C.c_void_p * n)(*[C.c_void_p(x) for x in d_divs])
    t = Tuning()
    _check(_tune_lib().fg_batch_autotune(batch.h, P, D, C.byref(t)), "fg_batch_autotune")
    return t.as_dict()


def _tuning_struct(families, nu=(0, 0), nu_coarse=(0, 0), coarse_from=2):
    """families: {level: {"x": v, "y": v, "z": v}} or one family per axis
    {"x": v, ...} for every level (LINE_FAMILIES numbers); nu_coarse: the
    smoothing steps from level coarse_from down ((0, 0): nu)."""
    t = Tuning()
    t.nu1_coarse, t.nu2_coarse = int(nu_coarse[0]), int(nu_coarse[1])
    t.coarse_from = int(coarse_from)
    t.nlevels = 12
    for L in range(12):
        row = families.get(L, {}) if any(isinstance(k, int) for k in families) else families
        for a, name in enumerate("xyz"):
            t.line_variant[L][a] = int(row.get(name, 0))
    t.nu1, t.nu2 = int(nu[0]), int(nu[1])
    return t


def case_set_tuning(case, families, nu=(0, 0), nu_coarse=(0, 0), coarse_from=2):
    t = _tuning_struct(families, nu, nu_coarse, coarse_from)
    _check(_tune_lib().fg_case_set_tuning(case.h, C.byref(t)), "fg_case_set_tuning")


def batch_set_tuning(batch, families, nu=(0, 0), nu_coarse=(0, 0), coarse_from=2):
    t = _tuning_struct(families, nu, nu_coarse, coarse_from)
    _check(_tune_lib().fg_batch_set_tuning(batch.h, C.byref(t)), "fg_batch_set_tuning")


def batch_get_tuning(batch) -> dict:
    t = Tuning()
    _check(_tune_lib().fg_batch_get_tuning(batch.h, C.byref(t)), "fg_batch_get_tuning")
    return t.as_dict()


def case_autotune(case, d_p: int, d_div: int) -> dict:
    t = Tuning()
    _check(_tune_lib().fg_case_autotune(case.h, C.c_void_p(d_p), C.c_void_p(d_div), C.byref(t)),
           "fg_case_autotune")
    return t.as_dict()


# ------------------------------------------------------------ projection steps
def _proj_lib():
    L = lib()
    if not getattr(L, "_proj_ready", False):
        vp = C.c_void_p
        L.fg_face_vel_device.argtypes = [vp] + [vp] * 9
        L.fg_rhs_poisson_device.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, C.c_double, vp,
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.fg_correct_vel_device.argtypes = [vp, vp, C.c_double, vp, vp, vp, vp, vp, vp]
        L.fg_update_pressure_device.argtypes = [vp, vp, vp]
        for n in ("fg_face_vel_device", "fg_rhs_poisson_device", "fg_correct_vel_device",
                  "fg_update_pressure_device"):
            getattr(L, n).restype = C.c_int
        L._proj_ready = True
    return L


def _dp(x):
    return None if x is None else C.c_void_p(x)


def face_vel_device(case, u, v, w, bcxu, bcyv, bczw, fu, fv, fw):
    """Device pointers (ints) of reference-layout fields and boundary arrays."""
    _check(_proj_lib().fg_face_vel_device(case.h, *[_dp(x) for x in (u, v, w, bcxu, bcyv, bczw, fu, fv, fw)]),
           "fg_face_vel_device")


def rhs_poisson_device(case, fu, fv, fw, bcxu, bcyv, bczw, vel_zero_gradient, dt, div):
    vz = None if vel_zero_gradient is None else np.ascontiguousarray(vel_zero_gradient, dtype=np.int32)
    sd, rd = C.c_double(0.0), C.c_double(0.0)
    _check(_proj_lib().fg_rhs_poisson_device(case.h, _dp(fu), _dp(fv), _dp(fw), _dp(bcxu), _dp(bcyv), _dp(bczw),
                                             _p(vz), dt, _dp(div), C.byref(sd), C.byref(rd)),
           "fg_rhs_poisson_device")
    return sd.value, rd.value


def update_pressure_device(case, d_pprime: int, d_p: int | None = None):
    """update_pressure on device fields: p' zeroed on non-dead solid cells
    and the domain edge lines, then copied to p."""
    _check(_proj_lib().fg_update_pressure_device(case.h, C.c_void_p(d_pprime), C.c_void_p(d_p) if d_p else None),
           "fg_update_pressure_device")


def _bi_lib():
    L = lib()
    if not getattr(L, "_bi_ready", False):
        vp = C.c_void_p
        L.fg_body_intercept_values_device.argtypes = [vp, C.c_int, C.c_double] + [vp] * 4
        L.fg_ghostcell_velocity_device.argtypes = [vp] * 6 + [C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.fg_body_intercept_values_device.restype = C.c_int
        L.fg_ghostcell_velocity_device.restype = C.c_int
        L._bi_ready = True
    return L


def body_intercept_values_device(case, ntime, dt, d_ubi_ghost=None, d_ubi_dead=None, d_dpdn_ghost=None,
                                 d_dpdn_dead=None):
    """Intercept velocities and dp/dn of the ghost and dead rows into device
    arrays (pointers; None skips an output)."""
    vp = lambda x: C.c_void_p(x) if x else None
    _check(_bi_lib().fg_body_intercept_values_device(case.h, ntime, dt, vp(d_ubi_ghost), vp(d_ubi_dead),
                                                     vp(d_dpdn_ghost), vp(d_dpdn_dead)),
           "fg_body_intercept_values_device")


def ghostcell_velocity_device(case, d_u, d_v, d_w, d_ubi_ghost, d_ubi_dead, itermax_gc=200, restol_gcv=1e-10,
                              allow_not_converged=False):
    """The velocity ghost and dead cells on device fields; returns the sweeps run."""
    vp = lambda x: C.c_void_p(x) if x else None
    it = C.c_int(0)
    rc = _bi_lib().fg_ghostcell_velocity_device(case.h, C.c_void_p(d_u), C.c_void_p(d_v), C.c_void_p(d_w),
                                                 vp(d_ubi_ghost), vp(d_ubi_dead), itermax_gc, restol_gcv,
                                                 C.byref(it))
    _check(rc, "fg_ghostcell_velocity_device", (FG_OK, FG_NOT_CONVERGED) if allow_not_converged else (FG_OK,))
    return it.value


class AdParams(C.Structure):
    """fg_ad_params: the momentum sweeps' time step, viscosity (1/Re),
    relaxation and whether convection is implicit (Crank-Nicolson)."""
    _fields_ = [("dt", C.c_double), ("reinv", C.c_double), ("omega_ad", C.c_double), ("crank_nicolson", C.c_int)]


def _ad_lib():
    L = lib()
    if not getattr(L, "_ad_ready", False):
        vp = C.c_void_p
        L.fg_itsolv_ad_device.argtypes = [vp] * 6 + [C.POINTER(AdParams)]
        L.fg_calc_residual_ad_device.argtypes = [vp] * 6 + [C.POINTER(AdParams), C.POINTER(C.c_double), vp]
        L.fg_itsolv_ad_device.restype = C.c_int
        L.fg_calc_residual_ad_device.restype = C.c_int
        L._ad_ready = True
    return L


def itsolv_ad_device(case, var, r, fu, fv, fw, prm: AdParams):
    """One pass of the momentum line SOR on device fields (pointers)."""
    _check(_ad_lib().fg_itsolv_ad_device(case.h, *[C.c_void_p(x) for x in (var, r, fu, fv, fw)], C.byref(prm)),
           "fg_itsolv_ad_device")


def calc_residual_ad_device(case, var, r, fu, fv, fw, prm: AdParams):
    m = C.c_double(0.0)
    loc = np.zeros(3, np.int32)
    _check(_ad_lib().fg_calc_residual_ad_device(case.h, *[C.c_void_p(x) for x in (var, r, fu, fv, fw)],
                                                C.byref(prm), C.byref(m), _p(loc)), "fg_calc_residual_ad_device")
    return m.value, tuple(int(x) for x in loc)


class VelocityBC(C.Structure):
    """fg_velocity_bc: outer velocity boundary type per face x1, x2, y1, y2,
    z1, z2 (1 Dirichlet, 2 zero gradient, 3 pulsatile inflow, 4 symmetry, 5
    periodic, 6 user specified), (u, v, w) values and frequencies per face,
    the flow time and the bounds of the user-specified channel profiles."""
    _fields_ = [("type", C.c_int * 6), ("val", (C.c_double * 3) * 6), ("freq", (C.c_double * 3) * 6),
                ("time", C.c_double), ("yOrigin", C.c_double), ("yout", C.c_double), ("zOrigin", C.c_double),
                ("zout", C.c_double)]


BC_ARRAY_NAMES = ("bcxu", "bcxv", "bcxw", "bcyu", "bcyv", "bcyw", "bczu", "bczv", "bczw")


class VelocityBCArrays(C.Structure):
    """fg_velocity_bc_arrays: device pointers of the nine outer boundary
    arrays in the reference layout."""
    _fields_ = [(n, C.c_void_p) for n in BC_ARRAY_NAMES]

    @classmethod
    def of(cls, ptrs):
        assert len(ptrs) == 9
        return cls(*[C.c_void_p(int(x)) for x in ptrs])


class SolveAdStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("residual", C.c_double), ("loc", C.c_int * 3)]


def _vbc_lib():
    L = lib()
    if not getattr(L, "_vbc_ready", False):
        vp = C.c_void_p
        A, V = C.POINTER(VelocityBCArrays), C.POINTER(VelocityBC)
        L.fg_set_outer_velocity_bc_device.argtypes = [vp] * 4 + [A, V]
        L.fg_set_outer_ghost_velocity_device.argtypes = [vp] * 4 + [A]
        L.fg_enforce_global_mass_consv_device.argtypes = [vp] * 8
        L.fg_solve_ad_device.argtypes = ([vp] * 10 + [A, vp, vp, C.POINTER(AdParams), V, C.c_int, C.c_double,
                                                      C.c_int, C.c_double, C.POINTER(SolveAdStats)])
        for n in ("fg_set_outer_velocity_bc_device", "fg_set_outer_ghost_velocity_device",
                  "fg_enforce_global_mass_consv_device", "fg_solve_ad_device"):
            getattr(L, n).restype = C.c_int
        L._vbc_ready = True
    return L


def set_outer_velocity_bc_device(case, d_u, d_v, d_w, bc_ptrs, vb: VelocityBC):
    """set_outer_velocity_bc into the nine device boundary arrays (pointers)."""
    a = VelocityBCArrays.of(bc_ptrs)
    _check(_vbc_lib().fg_set_outer_velocity_bc_device(case.h, *[C.c_void_p(x) for x in (d_u, d_v, d_w)],
                                                      C.byref(a), C.byref(vb)), "fg_set_outer_velocity_bc_device")


def set_outer_ghost_velocity_device(case, d_u, d_v, d_w, bc_ptrs):
    a = VelocityBCArrays.of(bc_ptrs)
    _check(_vbc_lib().fg_set_outer_ghost_velocity_device(case.h, *[C.c_void_p(x) for x in (d_u, d_v, d_w)],
                                                         C.byref(a)), "fg_set_outer_ghost_velocity_device")


def enforce_global_mass_consv_device(case, fu, fv, fw, bcxu, bcyv, bczw, vel_zero_gradient):
    vz = np.ascontiguousarray(vel_zero_gradient, dtype=np.int32)
    _check(_vbc_lib().fg_enforce_global_mass_consv_device(case.h, *[_dp(x) for x in (fu, fv, fw, bcxu, bcyv, bczw)],
                                                          _p(vz)), "fg_enforce_global_mass_consv_device")


def solve_ad_device(case, d_u, d_v, d_w, d_nlu, d_nlv, d_nlw, d_fu, d_fv, d_fw, bc_ptrs, d_ubi_ghost, d_ubi_dead,
                    prm: AdParams, vb: VelocityBC, itermax_gc=200, restol_gcv=1e-10, itermax_ad=100,
                    restol_ad=1e-8):
    """solve_ad on device fields (pointers); returns (iterations, residual,
    location)."""
    a = VelocityBCArrays.of(bc_ptrs)
    st = SolveAdStats()
    vp = lambda x: C.c_void_p(x) if x else None
    _check(_vbc_lib().fg_solve_ad_device(case.h, *[C.c_void_p(x) for x in (d_u, d_v, d_w, d_nlu, d_nlv, d_nlw,
                                                                            d_fu, d_fv, d_fw)],
                                         C.byref(a), vp(d_ubi_ghost), vp(d_ubi_dead), C.byref(prm), C.byref(vb),
                                         itermax_gc, restol_gcv, itermax_ad, restol_ad, C.byref(st)),
           "fg_solve_ad_device")
    return st.iterations, st.residual, tuple(st.loc)


def correct_vel_device(case, pp, dt, u=None, v=None, w=None, dpdx=None, dpdy=None, dpdz=None):
    _check(_proj_lib().fg_correct_vel_device(case.h, _dp(pp), dt, *[_dp(x) for x in (u, v, w, dpdx, dpdy, dpdz)]),
           "fg_correct_vel_device")
