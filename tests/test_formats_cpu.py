"""The formats around the path (``csrc/fg_io.cpp``) without a GPU, against
the oracle's restatement of the reference's layouts (oracle_formats.py):

* MSH 2.2 surface: the library's reader gives the vertices and triangles
  of the reference's fixed-line read sequence (BOUNDARY_MARKER_INIT.F90:
  247-296) on files in the layout that sequence expects, bit for bit; it
  also reads files that sequence cannot (line elements, non-consecutive
  node tags) and refuses broken ones;
* restart: every record of fg_write_restart is byte-identical to the
  write_restart layout (MAIN.F90:1049-1122) restated from the arrays,
  including records split into subrecords; fg_read_restart reads it back;
* Tecplot: every line of fg_write_tecplot equals write_flowfield's format
  123 (UTIL_GENERAL.F90:200-219), three-digit exponents included.
"""
import os
import struct

import numpy as np
import pytest

from feicar_b200 import fg, formats, synth
import oracle_formats as OF


def test_msh22_reads_like_the_reference(tmp_path):
    body = synth.sphere_body((1.0, 2.0, 3.0), 0.8, 3)
    p = str(tmp_path / "unstruc_surface_in.dat")
    OF.write_msh22(p, body.verts, body.tri, phys=((2, 1, "sphere"), (2, 7, "tip")))
    xyz, tri, skipped = formats.read_msh22(p)
    rx, rt = OF.read_msh22_reference(p)
    assert skipped == 0
    assert np.array_equal(xyz, rx) and np.array_equal(xyz, body.verts)
    assert np.array_equal(tri + 1, rt) and np.array_equal(tri, body.tri)


def test_msh22_tags_and_other_elements(tmp_path):
    body = synth.sphere_body((0.0, 0.0, 0.0), 1.0, 2)
    tags = 1000 + 3 * np.arange(body.nvert)[::-1]  # descending, gapped
    p = str(tmp_path / "s.msh")
    OF.write_msh22(p, body.verts, body.tri, tags=tags,
                   extra_elements=[f"1 15 2 0 1 {tags[0]}", f"2 1 2 0 1 {tags[0]} {tags[1]}"])
    xyz, tri, skipped = formats.read_msh22(p)
    assert skipped == 2
    assert np.array_equal(xyz, body.verts) and np.array_equal(tri, body.tri)


def test_msh22_refuses_broken_files(tmp_path):
    with pytest.raises(fg.FGError) as e:
        formats.read_msh22(str(tmp_path / "missing.msh"))
    assert e.value.status == formats.FG_IO_ERROR
    body = synth.sphere_body((0.0, 0.0, 0.0), 1.0, 1)
    p = str(tmp_path / "t.msh")
    OF.write_msh22(p, body.verts, body.tri)
    text = open(p).read()
    open(p, "w").write(text.replace("$EndElements\n", ""))  # truncated
    with pytest.raises(fg.FGError):
        formats.read_msh22(p)
    bad = text.replace(f"\n1 2 2 1 1 ", "\n1 2 2 1 1 99999 ", 1)  # unknown node tag in triangle 1
    lines = bad.split("\n")
    i = next(k for k, s in enumerate(lines) if s.startswith("1 2 2 1 1 "))
    w = lines[i].split()
    lines[i] = " ".join(w[:5] + ["99999"] + w[6:8])
    open(p, "w").write("\n".join(lines))
    with pytest.raises(fg.FGError) as e:
        formats.read_msh22(p)
    assert e.value.status == 5  # FG_BAD_INPUT
    open(p, "w").write(text.replace("2.2 0 8", "2.2 1 8"))  # binary files are not read
    with pytest.raises(fg.FGError):
        formats.read_msh22(p)


def _restart_case(rng, nx=7, ny=5, nz=4):
    sh = formats.shapes(nx, ny, nz)
    arrays = {k: np.asfortranarray(rng.standard_normal(sh[k])) for k in formats.FIELD3 + formats.BC}
    arrays["pgrad"] = [np.asfortranarray(rng.standard_normal(s)) for s in sh["pgrad"]]
    for k in ("iblank", "ghostcellmark"):
        arrays[k] = np.asfortranarray(rng.integers(0, 2, sh[k]).astype(np.int8))
    bodies = []
    for npts, nelm in ((12, 20), (5, 3)):
        b = {"npts": npts, "nelm": nelm, **{k: rng.standard_normal(npts) for k in formats.BODY_ARRAYS},
             "tri": rng.integers(0, npts, (nelm, 3)).astype(np.int32)}
        for k in ("cent", "ang", "vcent", "angv"):
            b[k] = rng.standard_normal(3)
        bodies.append(b)
    return nx, ny, nz, arrays, bodies


@pytest.mark.parametrize("max_sub", [None, 1000])
def test_restart_layout_and_round_trip(tmp_path, max_sub):
    rng = np.random.default_rng(3)
    nx, ny, nz, arrays, bodies = _restart_case(rng)
    p = str(tmp_path / "restart_0000.dat")
    try:
        if max_sub:
            formats.set_max_subrecord(max_sub)
        formats.write_restart(p, nx, ny, nz, arrays, bodies, time=12.5, ntime=345)
    finally:
        formats.set_max_subrecord(0)  # back to the default
    recs, marks = OF.read_records(p)
    assert len(recs) == 2 + len(bodies)
    assert recs[0] == struct.pack("<di", 12.5, 345)
    assert recs[1] == OF.restart_flow_record(nx, ny, nz, arrays)
    for r, b in zip(recs[2:], bodies):
        assert r == OF.restart_body_record(b)
    if max_sub:
        mk = marks[1]
        assert len(mk) == -(-len(recs[1]) // max_sub)
        assert all(l < 0 for l, _ in mk[:-1]) and mk[-1][0] > 0
        assert mk[0][1] > 0 and all(t < 0 for _, t in mk[1:])
        # the oracle's own writer gives the same bytes
        q = str(tmp_path / "oracle.dat")
        OF.write_records(q, recs, max_sub)
        assert open(q, "rb").read() == open(p, "rb").read()
    t, n, back, bb = formats.read_restart(p, nx, ny, nz, [(b["npts"], b["nelm"]) for b in bodies])
    assert (t, n) == (12.5, 345)
    for k in formats.FIELD3 + formats.BC + ("iblank", "ghostcellmark"):
        assert np.array_equal(back[k], arrays[k]), k
    for q in range(6):
        assert np.array_equal(back["pgrad"][q], arrays["pgrad"][q])
    for b0, b1 in zip(bodies, bb):
        for k in formats.BODY_ARRAYS + ("tri", "cent", "ang", "vcent", "angv"):
            assert np.array_equal(b0[k], b1[k]), k


def test_restart_refuses_a_wrong_grid(tmp_path):
    rng = np.random.default_rng(4)
    nx, ny, nz, arrays, bodies = _restart_case(rng)
    p = str(tmp_path / "r.dat")
    formats.write_restart(p, nx, ny, nz, arrays, bodies[:1])
    with pytest.raises(fg.FGError) as e:
        formats.read_restart(p, nx + 1, ny, nz, [(12, 20)])
    assert e.value.status == formats.FG_IO_ERROR
    with pytest.raises(fg.FGError):
        formats.read_restart(p, nx, ny, nz, [(11, 20)])


def test_tecplot_lines_match_format_123(tmp_path):
    rng = np.random.default_rng(5)
    grid = synth.small_grid(6, 5, 4, (1.2, 1.0, 0.8), stretch=1.5)
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    xc, yc, zc = grid.xc[:nx + 1], grid.yc[:ny + 1], grid.zc[:nz + 1]
    shp = (nx + 2, ny + 2, nz + 2)
    fields = {k: np.asfortranarray(rng.standard_normal(shp) * 10.0 ** rng.integers(-120, 120, shp))
              for k in ("u", "v", "w", "p", "ox", "oy", "oz")}
    fields["p"][1, 1, 1] = -0.0
    fields["u"][2, 1, 1] = 9.999995e-5  # rounds up into the next decade
    fields["v"][2, 1, 1] = 1e300
    for k in ("iblank", "ghost", "dead", "bodynum", "goa"):
        fields[k] = np.asfortranarray(rng.integers(0, 3, shp).astype(np.int8))
    fields["bodynum"][0, 0, 0] = 120  # does not fit I2
    p = str(tmp_path / "q_0000001.0000")
    formats.write_tecplot(p, xc, yc, zc, fields)
    lines = open(p).read().split("\n")
    assert lines[0] == ('VARIABLES="X","Y","Z","U","V","W","P","OX","OY","OZ","LMD","IBLANK","GHOST",'
                        '"DEAD","B#","goa"')
    assert lines[1].split() == ["ZONE", "F=POINT,", f"I={nx + 1},", f"J={ny + 1}", f"K={nz + 1}"]
    want = OF.tecplot_lines(xc, yc, zc, fields)
    assert lines[2:-1] == want
    assert lines[-1] == ""
    assert "**" in want[0] and "+300" in "".join(want)
