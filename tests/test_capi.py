"""The C-ABI library loads and exports every symbol include/dec_b200.h declares (no GPU needed),
and its argument checks reject bad input before any device work."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "dec_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dec_[a-z0-9_]+)\s*\(", text)))


def test_header_parses():
    names = declared_functions()
    assert "dec_mesh_create" in names and "dec_mg_solve" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol(dec):
    L = dec.lib()
    for name in declared_functions():
        assert hasattr(L, name), f"{name} declared in dec_b200.h but not exported"


def test_ctypes_signatures_cover_header(dec):
    from importlib import import_module
    capi = import_module("dec_b200._capi")
    assert set(declared_functions()) == set(capi.SIGNATURES), (
        set(declared_functions()) ^ set(capi.SIGNATURES))


def test_version_and_error_string(dec):
    L = dec.lib()
    assert L.dec_version() >= 1
    assert isinstance(L.dec_last_error(), bytes)


def _desc(capi, pts, ev0, ev1, te0, te1, te2, eo=None, to=None, base=0, keep=None):
    keep = keep if keep is not None else []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(C.c_void_p)

    d = capi.MeshDesc()
    d.nv, d.ne, d.nt = len(pts), len(ev0), len(te0)
    d.index_base = base
    d.points = arr(pts, np.float64)
    d.e_v0, d.e_v1 = arr(ev0, np.int32), arr(ev1, np.int32)
    d.t_e0, d.t_e1, d.t_e2 = arr(te0, np.int32), arr(te1, np.int32), arr(te2, np.int32)
    d.edge_orientation = None if eo is None else arr(eo, np.int8)
    d.tri_orientation = None if to is None else arr(to, np.int8)
    d.center = 0
    return d, keep


def test_mesh_rejects_out_of_range_indices(dec):
    from importlib import import_module
    capi = import_module("dec_b200._capi")
    L = dec.lib()
    pts = np.zeros((3, 3))
    d, keep = _desc(capi, pts, [1, 2, 2], [0, 1, 0], [1], [2], [7])  # edge 7 does not exist
    h = C.c_void_p()
    st = L.dec_mesh_create(C.byref(d), C.byref(h))
    assert st == 1
    assert b"out of range" in L.dec_last_error()


def test_mesh_rejects_bad_base(dec):
    from importlib import import_module
    capi = import_module("dec_b200._capi")
    L = dec.lib()
    d, keep = _desc(capi, np.zeros((3, 3)), [1, 2, 2], [0, 1, 0], [1], [2], [0], base=3)
    h = C.c_void_p()
    assert L.dec_mesh_create(C.byref(d), C.byref(h)) == 1


def test_non_orientable_mesh_is_reported(dec, O):
    """A Möbius strip: orient! fails, so the library returns DEC_ERR_NON_ORIENTABLE
    (make_dual_simplices_2d! raises in the reference, DiscreteExteriorCalculus.jl:577)."""
    from importlib import import_module
    capi = import_module("dec_b200._capi")
    L = dec.lib()
    m = O.Mesh()
    n = 6
    for i in range(2 * n):
        m.add_vertex(float(i), float(i % 3), 0.0)
    # strip of n squares whose last square is glued back with a half twist
    top = list(range(n))
    bot = list(range(n, 2 * n))
    for i in range(n):
        a, b = top[i], top[(i + 1) % n]
        c, d = bot[i], bot[(i + 1) % n]
        if i == n - 1:
            b, d = d, b
        m.glue_sorted_triangle(a, b, c)
        m.glue_sorted_triangle(b, c, d)
    assert not O.orient(m.copy())
    d_, keep = _desc(capi, m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2)
    h = C.c_void_p()
    assert L.dec_mesh_create(C.byref(d_), C.byref(h)) == 7


def test_null_arguments(dec):
    L = dec.lib()
    h = C.c_void_p()
    assert L.dec_mesh_create(None, C.byref(h)) == 1
    assert L.dec_wedge_apply(None, None, None, None, None) == 1
    assert L.dec_op_apply(None, None, None, 1.0, 0.0, None) == 1


def _csc(capi, m, n, colptr, rowval, nzval, base=0, keep=None):
    keep = keep if keep is not None else []
    cp = np.ascontiguousarray(colptr, np.int32)
    rv = np.ascontiguousarray(rowval, np.int32)
    nz = np.ascontiguousarray(nzval, np.float64)
    keep += [cp, rv, nz]
    c = capi.Csc()
    c.m, c.n, c.index_base = m, n, base
    c.colptr, c.rowval, c.nzval = (cp.ctypes.data_as(C.c_void_p), rv.ctypes.data_as(C.c_void_p),
                                   nz.ctypes.data_as(C.c_void_p))
    return c, keep


@pytest.mark.parametrize("case,msg", [
    (dict(colptr=[1, 2, 3], rowval=[0, 1], nzval=[1.0, 2.0]), b"colptr[0]"),          # base 0, colptr[0] = 1
    (dict(colptr=[0, 2, 1], rowval=[0, 1], nzval=[1.0, 2.0]), b"nondecreasing"),
    (dict(colptr=[0, 1, 2], rowval=[0, 5], nzval=[1.0, 2.0]), b"out of range"),
    (dict(colptr=[0, 2, 2], rowval=[1, 0], nzval=[1.0, 2.0]), b"strictly increasing"),
])
def test_csc_operator_rejects_malformed_matrices(dec, case, msg):
    """dec_op_create_csc checks the SparseMatrixCSC layout on the host before any device work."""
    from importlib import import_module
    capi = import_module("dec_b200._capi")
    L = dec.lib()
    c, keep = _csc(capi, 2, 2, **case)
    h = C.c_void_p()
    assert L.dec_op_create_csc(C.byref(c), 0, C.byref(h)) == 1
    assert msg in L.dec_last_error()


def test_mg_from_csc_rejects_mismatched_levels(dec):
    """dec_mg_create_from_csc checks the options and every matrix's dimensions before any device work."""
    from importlib import import_module
    capi = import_module("dec_b200._capi")
    L = dec.lib()
    keep = []
    a0, _ = _csc(capi, 3, 3, [0, 1, 2, 3], [0, 1, 2], [1.0, 1.0, 1.0], keep=keep)
    a1, _ = _csc(capi, 2, 2, [0, 1, 2], [0, 1], [1.0, 1.0], keep=keep)
    r_bad, _ = _csc(capi, 3, 2, [0, 1, 2], [0, 1], [1.0, 1.0], keep=keep)   # should be 2 x 3
    p0, _ = _csc(capi, 3, 2, [0, 1, 2], [0, 1], [1.0, 1.0], keep=keep)
    ops = (capi.Csc * 2)(a0, a1)
    rs = (capi.Csc * 1)(r_bad)
    ps = (capi.Csc * 1)(p0)
    o = capi.MGOptions()
    L.dec_mg_default_options(C.byref(o))
    h = C.c_void_p()
    assert L.dec_mg_create_from_csc(2, ops, rs, ps, None, C.byref(o), C.byref(h)) == 1
    assert b"restriction" in L.dec_last_error()
    o.smoother = 3
    assert L.dec_mg_create_from_csc(2, ops, rs, ps, None, C.byref(o), C.byref(h)) == 1
    L.dec_mg_default_options(C.byref(o))
    steps = (C.c_int32 * 2)(3, 17)
    assert L.dec_mg_create_from_csc(2, ops, rs, ps, steps, C.byref(o), C.byref(h)) == 1
    assert b"steps" in L.dec_last_error()


def _c_struct_fields(name):
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    body = re.search(r"typedef struct " + name + r" \{(.*?)\}", text, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = re.sub(r"\bconst\b", " ", decl).replace("*", " ").strip()
        if decl:
            fields += [f.strip() for f in decl.split(None, 1)[1].split(",")]
    return [f for f in fields if f]


def _julia_struct_fields(text, name):
    body = re.search(r"struct " + name + r"\n(.*?)\nend", text, flags=re.S).group(1)
    fields = []
    for line in body.splitlines():
        line = line.split("#")[0]
        if "()" in line:
            continue
        fields += re.findall(r"(\w+)::", line)
    return fields


def test_julia_extension_matches_the_header(dec):
    """ext/CombinatorialSpacesB200Ext.jl (the Val(:B200) backend a Julia caller loads) ccalls only
    symbols that the header declares and the library exports, and mirrors the C structs field for
    field (Julia is not installed here, so this is the check that runs)."""
    jl = (ROOT / "ext" / "CombinatorialSpacesB200Ext.jl").read_text()
    called = set(re.findall(r":(dec_[a-z0-9_]+)", jl))
    declared = set(declared_functions())
    assert called and called <= declared, called - declared
    L = dec.lib()
    for name in called:
        assert hasattr(L, name)
    for cname, jname in (("dec_mesh_desc", "DecMeshDesc"), ("dec_csc", "DecCsc"),
                         ("dec_mg_options", "DecMGOptions"), ("dec_solve_report", "DecSolveReport")):
        assert _julia_struct_fields(jl, jname) == _c_struct_fields(cname), cname
    # the reference CUDA extension's entry points all have Val(:B200) methods
    for fn in ("cache_wedge", "dec_boundary", "dec_dual_derivative", "dec_differential", "dec_hodge_star",
               "dec_inv_hodge_star", "dec_wedge_product", "multigrid_vcycles", "full_multigrid"):
        assert re.search(r"\n" + fn + r"\(.*Val\{:B200\}|function " + fn + r"\(.*Val\{:B200\}|\n" + fn +
                         r"\(u::CuVecOrMat|function " + fn + r"\(b::CuVecOrMat", jl), fn


def test_tuning_table_round_trip(dec, tmp_path):
    """The autotuner's table: set / get, saved as JSON and merged back after a clear; a file that is
    not a tuning table is refused (host only, no device work)."""
    import json
    dec.tune_clear()
    assert dec.tune_get("ell/f32/W7/n21") is None
    dec.tune_set("ell/f32/W7/n21", 2)
    dec.tune_set("sweep/f32/K32/W6/n19", 4)
    assert dec.tune_get("ell/f32/W7/n21") == 2
    path = tmp_path / "tune.json"
    dec.tune_save(path)
    d = json.loads(path.read_text())
    assert d["format"] == "dec_b200 tuning table" and d["version"] == 1
    assert d["entries"] == {"ell/f32/W7/n21": 2, "sweep/f32/K32/W6/n19": 4}
    dec.tune_clear()
    assert dec.tune_get("sweep/f32/K32/W6/n19") is None
    assert dec.tune_load(path) == 2
    assert dec.tune_get("sweep/f32/K32/W6/n19") == 4
    bad = tmp_path / "bad.json"
    bad.write_text('{"entries": {"x": 1}}')
    with pytest.raises(dec.DecError, match="tuning table"):
        dec.tune_load(bad)
    dec.tune_clear()
