"""Meshes on disk, host side: the reference's mesh import and its JSON format for this path.

* ``load_mesh(path)`` is ``EmbeddedDeltaSet2D(fn::String)`` (src/MeshInterop.jl:156-173) for
  Wavefront OBJ and STL (ASCII or binary): the file's points and triangles, points merged by
  location for STL (``force_unique``, whose first-occurrence numbering is
  ``unique_index_map``, :85-104), every face glued with ``glue_sorted_triangle!`` in file order,
  the triangle orientation left for ``orient!`` (run by the library when the mesh is created, as
  the reference runs it at the end of the import, :116-129).  Faces with more than three
  vertices are refused, as the reference refuses non-simplicial meshes.
* ``write_acset_json`` / ``read_acset_json`` store the primal tables of an ``EmbeddedDeltaSet2D``
  in Catlab's JSON layout for ACSets (the format ``parse_json_acset`` reads in
  src/CombMeshes.jl:43-53): one list per object (``V``, ``E``, ``Tri``) of rows with a 1-based
  ``_id``, the face maps by name (``∂v0``, ``∂v1``, ``∂e0``, ``∂e1``, ``∂e2``, 1-based) and the
  attributes (``point`` as [x, y, z], ``edge_orientation`` and ``tri_orientation`` as booleans).
  A dual-complex file's extra tables are ignored on reading: the library rebuilds the dual.
  Written files skip the regeneration of large hierarchies' base meshes.
"""
import json
import struct

import numpy as np

from .meshes import HostMesh, _Builder


def unique_index_map(coords, force_unique):
    """(ind_map, uniques): every point's new index, and the first occurrence of each distinct
    point (identity when force_unique is False)."""
    n = len(coords)
    if not force_unique:
        return np.arange(n), np.arange(n)
    seen, ind_map, uniques = {}, np.empty(n, np.int64), []
    for j, c in enumerate(map(tuple, coords)):
        i = seen.get(c)
        if i is None:
            i = seen[c] = len(uniques)
            uniques.append(j)
        ind_map[j] = i
    return ind_map, np.asarray(uniques, np.int64)


def from_faces(points, faces, force_unique=False):
    """A HostMesh from points (n, 3) and 0-based triangles, glued with glue_sorted_triangle!
    (each face's vertices sorted, then glue_triangle!), orientation unset."""
    points = np.asarray(points, np.float64)
    if points.ndim != 2 or points.shape[1] not in (2, 3):
        raise ValueError("points must be (n, 2) or (n, 3)")
    if points.shape[1] == 2:
        points = np.concatenate([points, np.zeros((points.shape[0], 1))], axis=1)
    ind_map, uniques = unique_index_map(points, force_unique)
    b = _Builder()
    for f in faces:
        if len(f) != 3:
            raise ValueError("only triangular faces are supported (the mesh is not simplicial)")
        v = sorted(int(ind_map[int(k)]) for k in f)
        b.glue(*v)
    return b.mesh(points[uniques], None)


def _obj_index(tok, nv):
    k = int(tok.split("/")[0])
    return k - 1 if k > 0 else nv + k  # negative indices count back from the last vertex


def read_obj(path):
    """Points (v lines) and triangles (f lines, 1-based, v/vt/vn forms accepted) of an OBJ file."""
    pts, faces = [], []
    with open(path, "r") as fh:
        for line in fh:
            t = line.split()
            if not t:
                continue
            if t[0] == "v":
                pts.append([float(x) for x in t[1:4]])
            elif t[0] == "f":
                faces.append([_obj_index(x, len(pts)) for x in t[1:]])
    return np.asarray(pts, np.float64), faces


def read_stl(path):
    """Triangle corners of an STL file (binary or ASCII) as separate points and faces."""
    with open(path, "rb") as fh:
        data = fh.read()
    ntri = struct.unpack_from("<I", data, 80)[0] if len(data) >= 84 else -1
    if ntri >= 0 and len(data) == 84 + 50 * ntri:
        rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]),
                            count=ntri, offset=84)
        pts = rec["v"].reshape(-1, 3).astype(np.float64)
    else:
        pts = [[float(x) for x in line.split()[1:4]] for line in data.decode("ascii", "replace").splitlines()
               if line.strip().startswith("vertex")]
        pts = np.asarray(pts, np.float64).reshape(-1, 3)
    faces = np.arange(len(pts)).reshape(-1, 3).tolist()
    return pts, faces


def load_mesh(path):
    """EmbeddedDeltaSet2D(fn::String): an OBJ or STL file as a HostMesh (STL points merged by
    location)."""
    p = str(path)
    if p.lower().endswith(".stl"):
        return from_faces(*read_stl(p), force_unique=True)
    if p.lower().endswith(".obj"):
        return from_faces(*read_obj(p))
    raise ValueError(f"unsupported mesh file {p!r} (OBJ and STL are read)")


def write_obj(path, mesh):
    """The mesh's points and triangles (vertices ∂v1∂e1, ∂v0∂e2, ∂v0∂e1) as an OBJ file."""
    tv = triangle_vertices(mesh)
    with open(path, "w") as fh:
        for p in np.asarray(mesh.points):
            fh.write("v %r %r %r\n" % (float(p[0]), float(p[1]), float(p[2])))
        for a, b, c in tv + 1:
            fh.write(f"f {a} {b} {c}\n")


def triangle_vertices(mesh):
    """(nt, 3) 0-based triangle vertices (src/SimplicialSets.jl:305-309)."""
    ev0, ev1 = np.asarray(mesh.ev0), np.asarray(mesh.ev1)
    te1, te2 = np.asarray(mesh.te1), np.asarray(mesh.te2)
    return np.stack([ev1[te1], ev0[te2], ev0[te1]], axis=1)


def write_acset_json(path, mesh, tri_orientation=None):
    """The primal tables of the mesh in Catlab's JSON ACSet layout.  The triangle orientation is
    the mesh's, or ``tri_orientation`` when given (for instance ``Mesh.orientation()[1]`` after
    the library ran orient!)."""
    to = mesh.tri_orientation if tri_orientation is None else tri_orientation
    if to is None:
        raise ValueError("the triangle orientation is unset: pass tri_orientation (Mesh.orientation())")
    pts = np.asarray(mesh.points, np.float64)
    doc = {
        "V": [{"_id": i + 1, "point": [float(x) for x in pts[i]]} for i in range(len(pts))],
        "E": [{"_id": e + 1, "∂v0": int(mesh.ev0[e]) + 1, "∂v1": int(mesh.ev1[e]) + 1,
               "edge_orientation": bool(mesh.edge_orientation[e])} for e in range(len(mesh.ev0))],
        "Tri": [{"_id": t + 1, "∂e0": int(mesh.te0[t]) + 1, "∂e1": int(mesh.te1[t]) + 1,
                 "∂e2": int(mesh.te2[t]) + 1, "tri_orientation": bool(to[t])} for t in range(len(mesh.te0))],
    }
    with open(path, "w", encoding="utf-8") as fh:
        json.dump(doc, fh, ensure_ascii=False)


def read_acset_json(path):
    """A HostMesh from the V / E / Tri tables of a JSON ACSet (rows in _id order)."""
    with open(path, "r", encoding="utf-8") as fh:
        doc = json.load(fh)
    rows = {k: sorted(doc.get(k, []), key=lambda r: r["_id"]) for k in ("V", "E", "Tri")}
    for k in ("V", "E", "Tri"):
        if [r["_id"] for r in rows[k]] != list(range(1, len(rows[k]) + 1)):
            raise ValueError(f"JSON ACSet: the {k} rows do not number 1..n")
    pts = np.asarray([r["point"] for r in rows["V"]], np.float64)
    if pts.size == 0:
        pts = pts.reshape(0, 3)
    if pts.shape[1] == 2:
        pts = np.concatenate([pts, np.zeros((pts.shape[0], 1))], axis=1)
    ev0 = np.asarray([r["∂v0"] - 1 for r in rows["E"]], np.int32)
    ev1 = np.asarray([r["∂v1"] - 1 for r in rows["E"]], np.int32)
    eo = np.asarray([1 if r.get("edge_orientation", False) else 0 for r in rows["E"]], np.int8)
    te = np.asarray([[r["∂e0"] - 1, r["∂e1"] - 1, r["∂e2"] - 1] for r in rows["Tri"]], np.int32).reshape(-1, 3)
    to = None
    if rows["Tri"] and all("tri_orientation" in r for r in rows["Tri"]):
        to = np.asarray([1 if r["tri_orientation"] else 0 for r in rows["Tri"]], np.int8)
    return HostMesh(pts, ev0, ev1, te[:, 0].copy(), te[:, 1].copy(), te[:, 2].copy(), eo, to)
