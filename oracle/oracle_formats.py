"""Restatement of the reference's file formats around the pressure path.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the
library's readers and writers, never by the product.

* ``read_msh22_reference`` follows the reference's own reading sequence of
  the unstructured surface file line by line (BOUNDARY_MARKER_INIT.F90:
  247-296): four lines skipped, the physical-name count and lines, two
  lines skipped, the node count and ``i x y z`` lines, two lines skipped,
  the element count and ``i1 i1 i1 i1 i1 n1 n2 n3`` lines.
* ``read_records`` / ``write_records`` restate the unformatted sequential
  layout (4-byte length markers around each subrecord; negative leading
  markers on every subrecord but the last, negative trailing markers on
  every one but the first) in which write_restart (MAIN.F90:1049-1122)
  leaves its records.
* ``pe12_5`` / ``i2`` / ``tecplot_lines`` restate the edit descriptors and
  loop order of write_flowfield (UTIL_GENERAL.F90:200-219).
"""
from __future__ import annotations

import math
import struct

import numpy as np


# ------------------------------------------------------------------ MSH 2.2
def write_msh22(path, xyz, tri, phys=((2, 1, "body"),), extra_elements=(), tags=None):
    """A Gmsh MSH 2.2 ASCII surface in the layout the reference reads.
    tri is 0-based; node tags are ``tags`` (default 1..n).  extra_elements
    are raw element lines placed before the triangles."""
    n = len(xyz)
    tags = list(range(1, n + 1)) if tags is None else list(tags)
    out = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(phys))]
    out += [f'{d} {t} "{name}"' for d, t, name in phys]
    out += ["$EndPhysicalNames", "$Nodes", str(n)]
    out += [f"{tags[i]} {float(xyz[i][0])!r} {float(xyz[i][1])!r} {float(xyz[i][2])!r}" for i in range(n)]
    out += ["$EndNodes", "$Elements", str(len(tri) + len(extra_elements))]
    out += list(extra_elements)
    base = len(extra_elements)
    out += [f"{base + e + 1} 2 2 1 1 {tags[t[0]]} {tags[t[1]]} {tags[t[2]]}" for e, t in enumerate(tri)]
    out += ["$EndElements"]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_msh22_reference(path):
    """The reference's read sequence: (xyz, tri 1-based as triElemNeig)."""
    with open(path) as f:
        lines = f.read().split("\n")
    at = 4  # DO i=1,4: READ
    num_tags = int(lines[at].split()[0]); at += 1
    at += num_tags  # i1, ibElTagVal, cLine
    at += 2  # DO n=1,2: READ cLine
    npts = int(lines[at].split()[0]); at += 1
    xyz = np.zeros((npts, 3))
    for n in range(npts):
        w = lines[at].split(); at += 1
        xyz[n] = [float(w[1]), float(w[2]), float(w[3])]
    at += 2
    nelm = int(lines[at].split()[0]); at += 1
    tri = np.zeros((nelm, 3), np.int64)
    for n in range(nelm):
        w = lines[at].split(); at += 1
        tri[n] = [int(w[5]), int(w[6]), int(w[7])]
    return xyz, tri


# ------------------------------------------------- unformatted sequential
def write_records(path, records, max_sub=2147483639):
    with open(path, "wb") as f:
        for rec in records:
            off, first = 0, True
            while True:
                ln = min(len(rec) - off, max_sub)
                last = off + ln == len(rec)
                f.write(struct.pack("<i", ln if last else -ln))
                f.write(rec[off:off + ln])
                f.write(struct.pack("<i", ln if first else -ln))
                off += ln
                first = False
                if off >= len(rec):
                    break


def read_records(path):
    """Records (bytes) and, per record, its list of (lead, trail) markers."""
    recs, marks = [], []
    with open(path, "rb") as f:
        data = f.read()
    at = 0
    while at < len(data):
        body, mk = b"", []
        while True:
            lead = struct.unpack_from("<i", data, at)[0]; at += 4
            ln = abs(lead)
            body += data[at:at + ln]; at += ln
            trail = struct.unpack_from("<i", data, at)[0]; at += 4
            assert abs(trail) == ln
            mk.append((lead, trail))
            if lead >= 0:
                break
        recs.append(body)
        marks.append(mk)
    return recs, marks


def restart_flow_record(nx, ny, nz, arrays):
    """Record 2 of write_restart from a dict of Fortran-ordered arrays."""
    NX, NY, NZ = nx + 2, ny + 2, nz + 2
    parts = []
    for k in ("u", "v", "w", "p", "face_u", "face_v", "face_w", "pPrime"):
        parts.append(np.asfortranarray(arrays.get(k, np.zeros((NX, NY, NZ))), np.float64).tobytes(order="F"))
    for k, sh in (("bcxu", (2, NY, NZ)), ("bcxv", (2, NY, NZ)), ("bcxw", (2, NY, NZ)), ("bcxp", (2, NY, NZ)),
                  ("bcyu", (NX, 2, NZ)), ("bcyv", (NX, 2, NZ)), ("bcyw", (NX, 2, NZ)), ("bcyp", (NX, 2, NZ)),
                  ("bczu", (NX, NY, 2)), ("bczv", (NX, NY, 2)), ("bczw", (NX, NY, 2)), ("bczp", (NX, NY, 2))):
        parts.append(np.asfortranarray(arrays.get(k, np.zeros(sh)), np.float64).tobytes(order="F"))
    pg = arrays.get("pgrad", [None] * 6)
    for q, sh in enumerate([(NY, NZ), (NY, NZ), (NX, NZ), (NX, NZ), (NX, NY), (NX, NY)]):
        parts.append(np.asfortranarray(pg[q] if pg[q] is not None else np.zeros(sh), np.float64).tobytes(order="F"))
    for k in ("iblank", "ghostcellmark"):
        parts.append(np.asfortranarray(arrays.get(k, np.zeros((NX, NY, NZ), np.int8)), np.int8).tobytes(order="F"))
    return b"".join(parts)


def restart_body_record(b):
    parts = [np.asarray(b[k], np.float64).tobytes() for k in ("x", "y", "z", "u", "v", "w", "fx", "fy", "fz")]
    parts.append((np.asarray(b["tri"], np.int32) + 1).tobytes(order="C"))  # triElemNeig(1:3, 1:nelm)
    for k in ("cent", "ang", "vcent", "angv"):
        parts.append(np.asarray(b[k], np.float64).tobytes())
    return b"".join(parts)


# ----------------------------------------------------------------- Tecplot
def pe12_5(v):
    """Fortran 1PE12.5 (one digit before the point, 5 after, exponent
    E+dd, or +ddd without the letter for a three-digit exponent)."""
    v = float(v)
    if math.isnan(v):
        return "NaN".rjust(12)
    if math.isinf(v):
        return ("Infinity" if v > 0 else "-Infinity").rjust(12)
    m, e = f"{v:.5E}".split("E")
    ex = int(e)
    s = f"{m}E{'+' if ex >= 0 else '-'}{abs(ex):02d}" if abs(ex) < 100 else f"{m}{'+' if ex >= 0 else '-'}{abs(ex):03d}"
    return s.rjust(12) if len(s) <= 12 else "*" * 12


def i2(n):
    n = int(n)
    return f"{n:2d}" if -9 <= n <= 99 else "**"


def tecplot_lines(xc, yc, zc, fields):
    """The data lines of write_flowfield (3-D) as text, k then j then i
    from the ghost layer 0 to n (format 123: 11(2x,pe12.5),5(2x,i2))."""
    nx, ny, nz = len(xc) - 1, len(yc) - 1, len(zc) - 1
    shp = (nx + 2, ny + 2, nz + 2)
    real = [fields.get(k, np.zeros(shp)) for k in ("u", "v", "w", "p", "ox", "oy", "oz", "lmd")]
    ints = [fields.get(k, np.zeros(shp, np.int8)) for k in ("iblank", "ghost", "dead", "bodynum", "goa")]
    out = []
    for k in range(nz + 1):
        for j in range(ny + 1):
            for i in range(nx + 1):
                s = "".join("  " + pe12_5(v) for v in (xc[i], yc[j], zc[k]))
                s += "".join("  " + pe12_5(a[i, j, k]) for a in real)
                s += "".join("  " + i2(a[i, j, k]) for a in ints)
                out.append(s)
    return out
