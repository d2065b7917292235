"""Host-side formats around the pressure path, through the C ABI
(``fg_read_msh22``, ``fg_write_restart``/``fg_read_restart``,
``fg_write_tecplot`` in ``csrc/fg_io.cpp``):

* the Gmsh MSH 2.2 body surface of the marker initialisation
  (BOUNDARY_MARKER_INIT.F90:247-296), returned as a ``synth.Body``-like
  triple (vertices, 0-based triangles, skipped element count);
* the restart file of write_restart / read_restart (MAIN.F90:983-1122);
* the Tecplot POINT dump of write_flowfield (UTIL_GENERAL.F90:167-247).

Arrays are Fortran-ordered numpy arrays with the reference's shapes
(``(nx+2, ny+2, nz+2)`` for a field of node counts nx, ny, nz).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import fg

FG_IO_ERROR = 10

_D = C.POINTER(C.c_double)


class RestartFlow(C.Structure):
    _fields_ = ([("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("time", C.c_double), ("ntime", C.c_int)]
                + [(n, _D) for n in ("u", "v", "w", "p", "face_u", "face_v", "face_w", "pPrime",
                                      "bcxu", "bcxv", "bcxw", "bcxp", "bcyu", "bcyv", "bcyw", "bcyp",
                                      "bczu", "bczv", "bczw", "bczp")]
                + [("pgrad", _D * 6), ("iblank", C.c_void_p), ("ghostcellmark", C.c_void_p)])


class RestartBody(C.Structure):
    _fields_ = ([("npts", C.c_int), ("nelm", C.c_int)]
                + [(n, _D) for n in ("x", "y", "z", "u", "v", "w", "fx", "fy", "fz")]
                + [("tri", C.POINTER(C.c_int))]
                + [(n, C.c_double * 3) for n in ("cent", "ang", "vcent", "angv")])


class TecplotFields(C.Structure):
    _fields_ = ([(n, _D) for n in ("u", "v", "w", "p", "ox", "oy", "oz", "lmd")]
                + [(n, C.c_void_p) for n in ("iblank", "ghost", "dead", "bodynum", "goa")])


FIELD3 = ("u", "v", "w", "p", "face_u", "face_v", "face_w", "pPrime")
BC = ("bcxu", "bcxv", "bcxw", "bcxp", "bcyu", "bcyv", "bcyw", "bcyp", "bczu", "bczv", "bczw", "bczp")
BODY_ARRAYS = ("x", "y", "z", "u", "v", "w", "fx", "fy", "fz")


def _lib():
    L = fg.lib()
    if not getattr(L, "_io_ready", False):
        vp, ip = C.c_void_p, C.c_int
        L.fg_read_msh22.argtypes = [C.c_char_p, C.POINTER(ip), C.POINTER(ip), vp, ip, vp, ip, C.POINTER(ip)]
        L.fg_write_restart.argtypes = [C.c_char_p, C.POINTER(RestartFlow), ip, vp]
        L.fg_read_restart.argtypes = [C.c_char_p, C.POINTER(RestartFlow), ip, vp]
        L.fg_write_tecplot.argtypes = [C.c_char_p, ip, ip, ip, vp, vp, vp, C.POINTER(TecplotFields)]
        L.fg_set_max_subrecord.argtypes = [C.c_longlong]
        L.fg_set_max_subrecord.restype = None
        for n in ("fg_read_msh22", "fg_write_restart", "fg_read_restart", "fg_write_tecplot"):
            getattr(L, n).restype = ip
        L._io_ready = True
    return L


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def shapes(nx, ny, nz):
    """The reference's array shapes for node counts nx, ny, nz."""
    NX, NY, NZ = nx + 2, ny + 2, nz + 2
    s = {k: (NX, NY, NZ) for k in FIELD3 + ("iblank", "ghostcellmark")}
    s.update({k: (2, NY, NZ) for k in BC[0:4]})
    s.update({k: (NX, 2, NZ) for k in BC[4:8]})
    s.update({k: (NX, NY, 2) for k in BC[8:12]})
    s["pgrad"] = [(NY, NZ), (NY, NZ), (NX, NZ), (NX, NZ), (NX, NY), (NX, NY)]
    return s


def read_msh22(path):
    """(xyz (nvert, 3), tri (ntri, 3) 0-based, n_skipped_elements)."""
    L = _lib()
    nv, nt, ns = C.c_int(), C.c_int(), C.c_int()
    fg._check(L.fg_read_msh22(path.encode(), C.byref(nv), C.byref(nt), None, 0, None, 0, C.byref(ns)),
              "fg_read_msh22")
    xyz = np.zeros((nv.value, 3))
    tri = np.zeros((nt.value, 3), np.int32)
    fg._check(L.fg_read_msh22(path.encode(), C.byref(nv), C.byref(nt), _vp(xyz), nv.value, _vp(tri), nt.value,
                              C.byref(ns)), "fg_read_msh22")
    return xyz, tri, ns.value


def _flow_struct(nx, ny, nz, arrays, time=0.0, ntime=0):
    sh = shapes(nx, ny, nz)
    f = RestartFlow(nx=nx, ny=ny, nz=nz, time=time, ntime=ntime)
    keep = []
    for k in FIELD3 + BC:
        a = arrays.get(k)
        if a is not None:
            assert a.shape == sh[k] and a.dtype == np.float64 and a.flags.f_contiguous, k
            setattr(f, k, _dp(a))
            keep.append(a)
    pg = arrays.get("pgrad")
    if pg is not None:
        for q in range(6):
            if pg[q] is not None:
                assert pg[q].shape == sh["pgrad"][q] and pg[q].flags.f_contiguous
                f.pgrad[q] = _dp(pg[q])
                keep.append(pg[q])
    for k in ("iblank", "ghostcellmark"):
        a = arrays.get(k)
        if a is not None:
            assert a.shape == sh[k] and a.dtype == np.int8 and a.flags.f_contiguous, k
            setattr(f, k, _vp(a))
            keep.append(a)
    return f, keep


def _body_structs(bodies):
    arr = (RestartBody * max(1, len(bodies)))()
    keep = []
    for n, b in enumerate(bodies):
        B = arr[n]
        B.npts, B.nelm = int(b["npts"]), int(b["nelm"])
        for k in BODY_ARRAYS:
            a = b.get(k)
            if a is not None:
                assert a.shape == (B.npts,) and a.dtype == np.float64, k
                setattr(B, k, _dp(a))
                keep.append(a)
        if b.get("tri") is not None:
            t = b["tri"]
            assert t.shape == (B.nelm, 3) and t.dtype == np.int32 and t.flags.c_contiguous
            B.tri = t.ctypes.data_as(C.POINTER(C.c_int))
            keep.append(t)
        for k in ("cent", "ang", "vcent", "angv"):
            if k in b:
                getattr(B, k)[:] = [float(x) for x in b[k]]
    return arr, keep


def write_restart(path, nx, ny, nz, arrays, bodies=(), time=0.0, ntime=0):
    """arrays: dict of the flow arrays (missing ones are written as zeros);
    bodies: list of dicts with npts, nelm, x..fz, tri (nelm, 3) 0-based,
    cent, ang, vcent, angv."""
    f, keep = _flow_struct(nx, ny, nz, arrays, time, ntime)
    barr, keep2 = _body_structs(list(bodies))
    fg._check(_lib().fg_write_restart(path.encode(), C.byref(f), len(bodies), C.cast(barr, C.c_void_p)),
              "fg_write_restart")


def read_restart(path, nx, ny, nz, bodies=()):
    """Reads every array; bodies: list of (npts, nelm).  Returns
    (time, ntime, arrays dict, list of body dicts)."""
    sh = shapes(nx, ny, nz)
    arrays = {k: np.zeros(sh[k], order="F") for k in FIELD3 + BC}
    arrays["pgrad"] = [np.zeros(s, order="F") for s in sh["pgrad"]]
    for k in ("iblank", "ghostcellmark"):
        arrays[k] = np.zeros(sh[k], np.int8, order="F")
    f, keep = _flow_struct(nx, ny, nz, arrays)
    bl = []
    for npts, nelm in bodies:
        d = {"npts": npts, "nelm": nelm, **{k: np.zeros(npts) for k in BODY_ARRAYS},
             "tri": np.zeros((nelm, 3), np.int32)}
        bl.append(d)
    barr, keep2 = _body_structs(bl)
    fg._check(_lib().fg_read_restart(path.encode(), C.byref(f), len(bl), C.cast(barr, C.c_void_p)),
              "fg_read_restart")
    for d, B in zip(bl, barr):
        for k in ("cent", "ang", "vcent", "angv"):
            d[k] = np.array(getattr(B, k)[:])
    return f.time, f.ntime, arrays, bl


def set_max_subrecord(nbytes):
    _lib().fg_set_max_subrecord(int(nbytes))


def write_tecplot(path, xc, yc, zc, fields=None):
    """xc, yc, zc: cell centres with ghost layers (lengths nx+1.., the
    reference's xc(0:nx)...); fields: dict of (nx+2, ny+2, nz+2) arrays
    u, v, w, p, ox, oy, oz, lmd (float64) and iblank, ghost, dead, bodynum,
    goa (int8); missing ones are written as zeros."""
    nx, ny, nz = len(xc) - 1, len(yc) - 1, len(zc) - 1
    xc, yc, zc = (np.ascontiguousarray(a, np.float64) for a in (xc, yc, zc))
    t = TecplotFields()
    keep = []
    for k, a in (fields or {}).items():
        real = k in ("u", "v", "w", "p", "ox", "oy", "oz", "lmd")
        a = np.asfortranarray(a, dtype=np.float64 if real else np.int8)
        assert a.shape == (nx + 2, ny + 2, nz + 2), k
        keep.append(a)
        setattr(t, k, _dp(a) if real else _vp(a))
    fg._check(_lib().fg_write_tecplot(path.encode(), nx, ny, nz, _vp(xc), _vp(yc), _vp(zc), C.byref(t)),
              "fg_write_tecplot")
