"""Mesh files (host side): OBJ / STL import as EmbeddedDeltaSet2D(fn) does it, and the JSON ACSet
tables.

* The reference's own import checks (test/MeshInterop.jl:16-22: the first triangle of
  assets/square.obj and of assets/square.stl has vertices [1, 2, 3]) run on copies of those two
  files in tests/golden/ (tests/golden/make_mesh_assets.py made them).
* The gluing equals the oracle's glue_sorted_triangle! on the same faces, array for array.
* OBJ, binary and ASCII STL and JSON ACSet files round-trip; STL points merge by location in
  first-occurrence order; non-triangular faces are refused.
"""
import json
import os
import struct

import numpy as np
import pytest

from conftest import uniform

ASSETS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def mio(dec):
    return dec.mesh_io


@pytest.mark.parametrize("name", ["square.obj", "square.stl"])
def test_reference_square_assets(mio, name):
    path = os.path.join(ASSETS, name)
    s = mio.load_mesh(path)
    np.testing.assert_array_equal(mio.triangle_vertices(s)[0], [0, 1, 2])
    assert (s.nv, s.nt) == (4, 2) and s.tri_orientation is None


def _oracle_glued(O, points, faces):
    m = O.Mesh()
    for p in points:
        m.add_vertex(*[float(x) for x in p])
    for f in faces:
        m.glue_sorted_triangle(*[int(x) for x in f])
    return m


def test_gluing_matches_oracle(O, mio):
    g = O.triangulated_grid(6, 5, 1.0, 0.8, False)
    pts = np.asarray(g.points)
    faces = np.asarray(g.tri_vertices())
    rng = np.random.default_rng(7)
    faces = faces[rng.permutation(len(faces))]
    faces = np.array([rng.permutation(f) for f in faces])  # any vertex order: sorted on gluing
    ours = mio.from_faces(pts, faces)
    ref = _oracle_glued(O, pts, faces)
    for k in ("ev0", "ev1", "te0", "te1", "te2"):
        np.testing.assert_array_equal(getattr(ours, k), getattr(ref, k))
    np.testing.assert_array_equal(ours.points, ref.points)


def test_obj_round_trip(mio, tmp_path):
    m = mio.from_faces(np.c_[uniform(1, 30).reshape(10, 3)], [[0, 1, 2], [1, 2, 3], [2, 3, 4], [5, 6, 7], [7, 8, 9]])
    p = tmp_path / "m.obj"
    mio.write_obj(p, m)
    m2 = mio.load_mesh(p)
    for k in ("points", "ev0", "ev1", "te0", "te1", "te2"):
        np.testing.assert_array_equal(getattr(m2, k), getattr(m, k))
    (tmp_path / "q.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    with pytest.raises(ValueError, match="triangular"):
        mio.load_mesh(tmp_path / "q.obj")
    (tmp_path / "n.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nf -3/1 -2/2 -1/3\n")
    np.testing.assert_array_equal(mio.triangle_vertices(mio.load_mesh(tmp_path / "n.obj")), [[0, 1, 2]])


def test_stl_merges_points(mio, tmp_path):
    corners = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    body = b"".join(struct.pack("<3f", 0, 0, 1) + corners[3 * t:3 * t + 3].tobytes() + b"\0\0" for t in range(2))
    (tmp_path / "b.stl").write_bytes(b"\0" * 80 + struct.pack("<I", 2) + body)
    text = "solid s\n" + "".join(
        "facet normal 0 0 1\nouter loop\n" + "".join(f"vertex {x} {y} {z}\n" for x, y, z in corners[3 * t:3 * t + 3])
        + "endloop\nendfacet\n" for t in range(2)) + "endsolid s\n"
    (tmp_path / "a.stl").write_text(text)
    for name in ("b.stl", "a.stl"):
        s = mio.load_mesh(tmp_path / name)
        assert (s.nv, s.ne, s.nt) == (4, 5, 2)
        np.testing.assert_array_equal(s.points, [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]])
        np.testing.assert_array_equal(mio.triangle_vertices(s), [[0, 1, 2], [0, 2, 3]])


def test_json_acset_round_trip(O, mio, tmp_path):
    g = O.triangulated_grid(4, 3, 1.0, 0.9, False)
    m = mio.from_faces(np.asarray(g.points), np.asarray(g.tri_vertices()))
    with pytest.raises(ValueError, match="orientation"):
        mio.write_acset_json(tmp_path / "x.json", m)
    to = np.arange(m.nt, dtype=np.int8) % 2
    p = tmp_path / "m.json"
    mio.write_acset_json(p, m, tri_orientation=to)
    doc = json.loads(p.read_text(encoding="utf-8"))
    assert set(doc) == {"V", "E", "Tri"}
    assert doc["E"][0] == {"_id": 1, "∂v0": int(m.ev0[0]) + 1, "∂v1": int(m.ev1[0]) + 1, "edge_orientation": False}
    assert doc["Tri"][1]["tri_orientation"] is True and doc["V"][2]["point"] == [float(x) for x in m.points[2]]
    m2 = mio.read_acset_json(p)
    for k in ("points", "ev0", "ev1", "te0", "te1", "te2", "edge_orientation"):
        np.testing.assert_array_equal(getattr(m2, k), getattr(m, k))
    np.testing.assert_array_equal(m2.tri_orientation, to)
    doc["E"] = doc["E"][::-1]  # rows in any order, numbered by _id
    doc["DualV"] = [{"_id": 1}]  # a dual complex's extra tables are ignored
    p.write_text(json.dumps(doc, ensure_ascii=False), encoding="utf-8")
    np.testing.assert_array_equal(mio.read_acset_json(p).ev0, m.ev0)
