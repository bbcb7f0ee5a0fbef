"""Pin the CPU oracle to the reference's own known-answer tests.

Each test restates a check from CombinatorialSpaces.jl's test suite (file:line cited) and runs it
against the oracle.  Indices are 0-based here (the reference is 1-based).
"""
import math

import numpy as np
import pytest

from conftest import csc

SQ5 = math.sqrt(5.0)


def gillette(O, center):
    # test/DiscreteExteriorCalculus.jl:288-296: unit right triangle, true orientations.
    m = O.Mesh()
    m.add_vertex(0, 0, 0)
    m.add_vertex(1, 0, 0)
    m.add_vertex(0, 1, 0)
    m.glue_triangle(0, 1, 2, 1)
    m.set_edge_orientation(1)
    return O.dualize(m, center)


def test_dual_layout_square(O):
    # test/DiscreteExteriorCalculus.jl:183-201
    m = O.Mesh()
    for _ in range(4):
        m.add_vertex(0, 0, 0)
    m.glue_triangle(0, 1, 2)
    m.glue_triangle(0, 2, 3)
    # coordinates are irrelevant for the layout; give them distinct positions
    m = O.mesh_from_arrays(np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], float),
                           m.ev0, m.ev1, m.te0, m.te1, m.te2,
                           np.full(m.ne, -1, np.int8), np.full(m.nt, -1, np.int8))
    d = O.dualize(m, O.BARYCENTER)
    nv, ne, nt = m.nv, m.ne, m.nt
    assert len(d.D_dv0) == 2 * ne + 6 * nt
    assert len(d.D_de0) == 6 * nt
    assert d.dual_point.shape[0] == nv + ne + nt
    # primal_vertex(subsimplices(Tri(1))) == [1,1,2,2,3,3]
    prim = [d.D_dv1[d.D_de2[i * nt + 0]] for i in range(6)]
    assert prim == [0, 0, 1, 1, 2, 2]
    # elementary_duals(1, s, 2) has one dual edge, (1, s, 3) has two, both ending at the edge center
    for e, count in ((1, 1), (2, 2)):
        des = np.nonzero(d.D_dv1 == nv + e)[0]
        assert len(des) == count
    # [length(elementary_duals(s, V(i))) for i in 1:4] == [4,2,4,2]
    counts = [int(np.sum(d.D_dv1[d.D_de1] == v)) for v in range(4)]
    assert counts == [4, 2, 4, 2]
    assert d.dual_triangle_vertices(0) == (0, 6, 9)           # [1,7,10]
    assert (int(d.D_dv0[0]), int(d.D_dv1[0])) == (4, 1)       # [5,2]


def test_gillette_barycentric(O):
    d = gillette(O, O.BARYCENTER)
    # :298-302
    np.testing.assert_allclose(d.dual_point[d.nv + d.ne + 0][:2], [1 / 3, 1 / 3], rtol=1e-14)
    np.testing.assert_allclose(d.area, [0.5], rtol=1e-14)
    np.testing.assert_allclose(O.hodge_diag(d, 0), [1 / 6] * 3, rtol=1e-14)
    # :305
    np.testing.assert_allclose(O.hodge_diag(d, 1), [SQ5 / 6, 1 / 6, SQ5 / 6], rtol=1e-14)
    # :306-308  δ1 = ⋆0⁻¹ · dual_d(1) · ⋆1
    delta1 = (np.diag(O.inv_hodge_diag(d, 0)) @ csc(O.dec_dual_derivative(d, 1)).toarray()
              @ np.diag(O.hodge_diag(d, 1)))
    np.testing.assert_allclose(delta1, [[2.236, 0, 2.236], [-2.236, 1, 0], [0, -1, -2.236]], atol=1e-3)
    # :331-333 inverse Hodge stars
    np.testing.assert_allclose(O.inv_hodge_diag(d, 2), [0.5], rtol=1e-14)
    np.testing.assert_allclose(O.inv_hodge_diag(d, 1), [-6 / SQ5, -6, -6 / SQ5], rtol=1e-14)


def test_gillette_circumcentric(O):
    d = gillette(O, O.CIRCUMCENTER)
    # test/DiscreteExteriorCalculus.jl:362-368
    np.testing.assert_allclose(d.dual_point[d.nv + d.ne + 0][:2], [0.5, 0.5], rtol=1e-14)
    np.testing.assert_allclose(O.hodge_diag(d, 0), [1 / 4, 1 / 8, 1 / 8], rtol=1e-14)
    np.testing.assert_allclose(O.hodge_diag(d, 1), [0.5, 0.0, 0.5], atol=1e-15)
    delta1 = (np.diag(O.inv_hodge_diag(d, 0)) @ csc(O.dec_dual_derivative(d, 1)).toarray()
              @ np.diag(O.hodge_diag(d, 1)))
    np.testing.assert_allclose(delta1, [[2, 0, 2], [-4, 0, 0], [0, 0, -4]], atol=1e-12)
    # Δ(0) = δ1 d0 = -fast_laplace_beltrami
    L = csc(O.laplace_beltrami0(d)).toarray()
    np.testing.assert_allclose(-L, delta1 @ csc(O.dec_differential(d, 0)).toarray(), atol=1e-12)


def test_gillette_exterior_derivative(O):
    d = gillette(O, O.BARYCENTER)
    d0 = csc(O.dec_differential(d, 0)).toarray()
    d1 = csc(O.dec_differential(d, 1)).toarray()
    np.testing.assert_array_equal(d0, [[-1, 1, 0], [0, -1, 1], [-1, 0, 1]])
    np.testing.assert_array_equal(d1, [[1, 1, -1]])
    np.testing.assert_array_equal(d1 @ d0, np.zeros((1, 3)))
    np.testing.assert_array_equal(csc(O.dec_boundary(d, 1)).toarray(), d0.T)
    np.testing.assert_array_equal(csc(O.dec_boundary(d, 2)).toarray(), d1.T)
    np.testing.assert_array_equal(csc(O.dec_dual_derivative(d, 0)).toarray(), d1.T)
    np.testing.assert_array_equal(csc(O.dec_dual_derivative(d, 1)).toarray(), -d0.T)


def const_form(mesh, X):
    # eval_constant_primal_form, DiscreteExteriorCalculus.jl:2172-2177
    p = mesh.points
    sg = np.where(mesh.edge_orientation == 1, 1.0, -1.0)
    return ((p[mesh.ev0] - p[mesh.ev1]) @ np.asarray(X, float)) * sg


def test_wedge_02_unit_area(O):
    # test/DiscreteExteriorCalculus.jl:535-547: ∧(3, 5 dx∧dy) = 15 on a unit-area 3-4-5 triangle.
    m = O.Mesh()
    m.add_vertex(0, 0, 0)
    m.add_vertex(6 / 8, 0, 0)
    m.add_vertex(6 / 8, 8 / 3, 0)
    m.glue_triangle(0, 1, 2, 1)
    m.set_edge_orientation(1)
    d = O.dualize(m, O.BARYCENTER)
    out = O.wedge(d, 2, np.array([3.0, 3, 3]), np.array([d.area[0] * 5]))
    np.testing.assert_allclose(out, [15.0], rtol=1e-14)


def test_wedge_identities_grid_345(O):
    # test/DiscreteExteriorCalculus.jl:549-570
    d = O.dualize(O.grid_345(), O.BARYCENTER)
    m = d.mesh
    one = np.ones(d.nv)
    np.testing.assert_allclose(O.wedge(d, 1, one, np.arange(1.0, d.ne + 1)), np.arange(1.0, d.ne + 1), rtol=1e-14)
    np.testing.assert_allclose(O.wedge(d, 2, one, np.arange(1.0, d.nt + 1)), np.arange(1.0, d.nt + 1), rtol=1e-14)
    dx = const_form(m, [1, 0, 0])
    dy = const_form(m, [0, 1, 0])
    np.testing.assert_allclose(O.wedge(d, 11, dx, dy), d.area, rtol=1e-14)
    np.testing.assert_array_equal(O.wedge(d, 11, dx, dy), -O.wedge(d, 11, dy, dx))
    np.testing.assert_array_equal(O.wedge(d, 11, 3 * dx, 2 * dy), O.wedge(d, 11, 2 * dx, 3 * dy))


def test_wedge_orientation_flip_invariance(O):
    # test/DiscreteExteriorCalculus.jl:560-565: flipping one edge's orientation (and the sign of
    # the forms on it) leaves dx∧dy unchanged.
    base = O.grid_345()
    for i in range(base.ne):
        eo = base.edge_orientation.copy()
        eo[i] = 1 - eo[i]
        m = O.mesh_from_arrays(base.points, base.ev0, base.ev1, base.te0, base.te1, base.te2,
                               eo, base.tri_orientation)
        d = O.dualize(m, O.BARYCENTER)
        dx, dy = const_form(m, [1, 0, 0]), const_form(m, [0, 1, 0])
        np.testing.assert_allclose(O.wedge(d, 11, dx, dy), d.area, rtol=1e-13)


def test_wedge_cw_triangle(O):
    # test/DiscreteExteriorCalculus.jl:567-570: tri_345_false gives -area.
    d = O.dualize(O.tri_345(False), O.BARYCENTER)
    dx, dy = const_form(d.mesh, [1, 0, 0]), const_form(d.mesh, [0, 1, 0])
    np.testing.assert_allclose(O.wedge(d, 11, dx, dy), -d.area, rtol=1e-14)


def test_subdivision_structure(O):
    # test/Multigrid.jl:14-19
    s = O.triangulated_grid(1, 1, 1, 1, False)
    S = csc(O.subdivision_matrix(s)).toarray()
    nv = s.nv
    np.testing.assert_array_equal(S[:nv, :nv], np.eye(nv))
    for e in range(s.ne):
        col = S[:, nv + e]
        rows = np.nonzero(col)[0]
        assert list(rows) == [s.ev1[e], s.ev0[e]]
        np.testing.assert_array_equal(col[rows], [0.5, 0.5])


def test_subdivision_counts_and_orientation(O):
    # test/Multigrid.jl:21-41 (binary): counts per round and orient! succeeds.
    s = O.triangulated_grid(1, 1, 1, 1, False)
    for _ in range(4):
        t = O.refine_binary(s, 0.0)
        assert (t.nv, t.ne, t.nt) == (s.nv + s.ne, 2 * s.ne + 3 * s.nt, 4 * s.nt)
        assert O.orient(t)
        s = t


def test_icosphere_counts(O):
    # Icosphere L_k = k binary subdivisions of the icosahedron: nv = 10·4^k + 2, nt = 20·4^k.
    s = O.icosahedron()
    assert (s.nv, s.ne, s.nt) == (12, 30, 20)
    for k in range(1, 5):
        s = O.refine_binary(s, 1.0)
        assert (s.nv, s.ne, s.nt) == (10 * 4 ** k + 2, 30 * 4 ** k, 20 * 4 ** k)
        np.testing.assert_allclose(np.linalg.norm(s.points, axis=1), 1.0, rtol=1e-15)
        assert O.orient(s)


def test_triangulated_grid_config(O):
    # CombMeshes.jl:79-133 with (127, 127, 1.0, 1.0, Point3d, false): 128 x 128 vertices.
    s = O.triangulated_grid(127, 127, 1.0, 1.0, False)
    assert (s.nv, s.ne, s.nt) == (16384, 48641, 32258)
    p = s.points
    assert p[0].tolist() == [0, 0, 0]
    assert p[128].tolist() == [0.5, 1.0, 0.0]     # even (1-based) rows are shifted by dx/2
    assert s.edge_orientation.max() == 0
    o = s.tri_orientation
    assert o[0] == 1 and o[1] == 0 and o[254] == 0 and o[255] == 1


def _mg_residual_setup(O, steps):
    # test/Multigrid.jl:54-90 and :94-111: 4 binary levels over triangulated_grid(1,1,1/4,√3/8).
    s = O.triangulated_grid(1, 1, 1 / 4, math.sqrt(3) / 2 * 1 / 4, False)
    md = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, steps)
    L = csc(md.op(0))
    rng = np.random.default_rng(0)
    b = L @ rng.random(L.shape[0])
    return md, L, b


def test_multigrid_residuals(O):
    md, L, b = _mg_residual_setup(O, 3)
    u0 = np.zeros_like(b)
    rel = lambda u: np.linalg.norm(L @ u - b) / np.linalg.norm(b)
    assert rel(O.mu_cycles(md, u0, b, 5, 1)) < 1e-7   # V
    assert rel(O.mu_cycles(md, u0, b, 5, 2)) < 1e-7   # W
    assert rel(O.full_multigrid(md, b, 5, 1)) < 1e-6  # FMG-V
    assert rel(O.full_multigrid(md, b, 5, 2)) < 1e-7  # FMG-W


def test_multigrid_zero_steps(O):
    # test/Multigrid.jl:151-170 (issue #178): steps = 0 runs no smoothing at all.
    md0, L, b = _mg_residual_setup(O, 0)
    md1, _, _ = _mg_residual_setup(O, 1)
    u0 = np.zeros_like(b)
    r0 = np.linalg.norm(L @ O.mu_cycles(md0, u0, b, 5, 1) - b)
    r1 = np.linalg.norm(L @ O.mu_cycles(md1, u0, b, 5, 1) - b)
    assert r1 < r0


def test_multigrid_hierarchy_shapes(O):
    md, L, _ = _mg_residual_setup(O, 3)
    assert md.nlevels == 5
    for k in range(4):
        A = csc(md.op(k))
        Ac = csc(md.op(k + 1))
        R = csc(md.restriction(k))
        P = csc(md.prolongation(k))
        assert R.shape == (Ac.shape[0], A.shape[0])
        assert P.shape == (A.shape[0], Ac.shape[0])
        np.testing.assert_allclose(np.asarray(R.sum(axis=1)).ravel(), 1.0, rtol=1e-15)


def _primal_const(m, alpha):
    """eval_constant_primal_form (src/DiscreteExteriorCalculus.jl:2172-2177):
    α · (p[tgt e] - p[src e]) · sign(e), tgt = ∂v0, src = ∂v1."""
    p = np.asarray(m.points).reshape(-1, 3)
    v = (p[np.asarray(m.ev0)] - p[np.asarray(m.ev1)]) @ np.asarray(alpha, float)
    return v * np.where(np.asarray(m.edge_orientation) > 0, 1.0, -1.0)


def _dual_const(O, d, alpha):
    """eval_constant_dual_form (:2189-2193): hodge_star(1, s) -- the geometric ⋆1, the default
    for 1-forms in 2D (:1650) -- applied to the primal form of (α₂, -α₁, α₃)."""
    return csc(O.hodge_geometric1(d)) @ _primal_const(d.mesh, [alpha[1], -alpha[0], alpha[2]])


@pytest.mark.parametrize("mesh", ["tri_345", "grid_345"])
def test_flat_sharp_and_pd_wedges(O, mesh):
    """test/DiscreteExteriorCalculus.jl:701-745 (flat counter-clockwise meshes, barycentric duals):
    ♭♯ maps a constant field's dual 1-form to its primal 1-form (up to the orientation sign),
    and the primal-dual (1,1) wedges are antisymmetric, exactly across pd and dp."""
    d = O.dualize(getattr(O, mesh)(), O.BARYCENTER)
    fs = csc(O.flat_sharp_mat(d))
    X = [3 / math.sqrt(2), 1 / math.sqrt(2), 0.0]
    Xf = _dual_const(O, d, X)
    got = fs @ Xf
    want = _primal_const(d.mesh, X)
    assert np.allclose(got, want, atol=1e-13) or np.allclose(got, -want, atol=1e-13)
    pd = lambda f, g: O.wedge(d, 11, f, fs @ g)
    dp = lambda f, g: O.wedge(d, 11, fs @ f, g)
    fd, gd = [2.0, 7.0, 0.0], [8.0, 1.0, 0.0]
    f1, g1 = _primal_const(d.mesh, fd), _primal_const(d.mesh, gd)
    f2, g2 = _dual_const(O, d, fd), _dual_const(O, d, gd)
    np.testing.assert_allclose(pd(f1, g2), -pd(g1, f2), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(dp(f2, g1), -dp(g2, f1), rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(pd(f1, g2), -dp(g2, f1))
    np.testing.assert_array_equal(dp(f2, g1), -pd(g1, f2))
    np.testing.assert_allclose(pd(f1, f2), 0, atol=1e-11)
    np.testing.assert_allclose(pd(g1, g2), 0, atol=1e-11)


@pytest.mark.parametrize("mesh,center", [("tri_345", "BARYCENTER"), ("grid_345", "BARYCENTER"),
                                         ("grid", "BARYCENTER"), ("grid", "CIRCUMCENTER"), ("ico", "CIRCUMCENTER")])
def test_geometric_hodge_fast_matches_dec(O, mesh, center):
    """test/Operators.jl:184-197: FastDEC's geometric ⋆1 equals the DEC one to 1e-12 (the
    reference compares them with rtol / atol 1e-12).  On planar circumcentric duals it is the
    diagonal ⋆1; on a curved surface its z-axis orientation trick (crossdot,
    DiscreteExteriorCalculus.jl:1667-1670) flips some entries, so that check is planar only."""
    if mesh == "grid":
        m = O.triangulated_grid(10, 7, 1.3, 0.9, True)
    elif mesh == "ico":
        m = O.refine_binary(O.refine_binary(O.icosahedron(), 1.0), 1.0)
    else:
        m = getattr(O, mesh)()
    d = O.dualize(m, getattr(O, center))
    fast = csc(O.hodge_geometric1_fast(d)).toarray()
    dec = csc(O.hodge_geometric1(d)).toarray()
    np.testing.assert_allclose(fast, dec, rtol=1e-12, atol=1e-12)
    if center == "CIRCUMCENTER" and mesh == "grid":
        np.testing.assert_allclose(fast, np.diag(O.hodge_diag(d, 1)), rtol=1e-12, atol=1e-12)


def _cache_meshes(O):
    return [O.dualize(O.grid_345(), O.BARYCENTER), O.dualize(O.triangulated_grid(6, 5, 1.0, 0.8, False), O.CIRCUMCENTER)]


def test_cached_wedge_kernels_match_mesh_wedges(O):
    """dec_c_wedge_product! on the reference's caches (FastDEC.jl:217-232) equals the mesh-bound
    wedges (which the reference's identities above pin) bit for bit: (0,1) with p = [∂v0 ∂v1]
    (an ne x 2 column-major matrix), (0,2) and (1,1) with the 6 x nt / 3 x nt caches."""
    rng = np.random.default_rng(11)
    for d in _cache_meshes(O):
        m = d.mesh
        f, a, b, t = rng.uniform(-1, 1, d.nv), rng.uniform(-1, 1, d.ne), rng.uniform(-1, 1, d.ne), rng.uniform(-1, 1, d.nt)
        p01 = np.concatenate([m.ev0, m.ev1]).astype(np.int32)
        np.testing.assert_array_equal(O.c_wedge(0, 1, d.ne, p01, np.zeros(0), f, a), O.wedge(d, 1, f, a))
        v, c = O.wedge02_cache(d)
        np.testing.assert_array_equal(O.c_wedge(0, 2, d.nt, v, c, f, t), O.wedge(d, 2, f, t))
        e, c = O.wedge11_cache(d)
        np.testing.assert_array_equal(O.c_wedge(1, 1, d.nt, e, c, a, b), O.wedge(d, 11, a, b))


def test_cached_3d_wedge_kernels(O):
    """The 3D kernels wedge_kernel_03! (FastDEC.jl:172-182) and wedge_kernel_21! (:193-205) against
    a vectorised numpy statement of the same sums, on random caches."""
    rng = np.random.default_rng(12)
    n, nv, ne, nt = 37, 50, 80, 60
    p3 = rng.integers(0, nv, (n, 24)).astype(np.int32)
    c3 = rng.uniform(-1, 1, (n, 24))
    f, beta = rng.uniform(-1, 1, nv), rng.uniform(-1, 1, n)
    ref3 = np.zeros(n)
    for j in range(24):
        ref3 = ref3 + beta * c3[:, j] * f[p3[:, j]]
    np.testing.assert_array_equal(O.c_wedge(0, 3, n, p3, c3, f, beta), ref3)
    p21 = np.concatenate([rng.integers(0, ne, (n, 6)), rng.integers(0, nt, (n, 4))], axis=1).astype(np.int32)
    c21 = rng.uniform(-1, 1, (n, 12))
    al, be = rng.uniform(-1, 1, nt), rng.uniform(-1, 1, ne)
    B = [be[p21[:, q]] for q in range(6)]
    A = [al[p21[:, 6 + q]] for q in range(4)]
    w = [c21[:, q] for q in range(12)]
    ref21 = (w[0] * B[3] * A[3] - w[1] * B[4] * A[2] + w[2] * B[5] * A[1] + w[3] * B[1] * A[3] - w[4] * B[2] * A[2]
             + w[5] * B[5] * A[0] + w[6] * B[0] * A[3] - w[7] * B[2] * A[1] + w[8] * B[4] * A[0] + w[9] * B[0] * A[2]
             - w[10] * B[1] * A[1] + w[11] * B[3] * A[0])
    np.testing.assert_array_equal(O.c_wedge(2, 1, n, p21, c21, al, be), ref21)
    # 1 ∧ β = β when every tetrahedron's coefficients sum to one
    c1 = rng.uniform(0, 1, (n, 24))
    c1 /= c1.sum(axis=1, keepdims=True)
    np.testing.assert_allclose(O.c_wedge(0, 3, n, p3, c1, np.ones(nv), beta), beta, rtol=1e-14, atol=1e-15)


def test_galerkin_mode_thresholds(O):
    """test_galerkin (test/Multigrid.jl:115-142) with BinarySubdivision: coarse operators R A P
    (GalerkinMode, Multigrid.jl:740-748), CG smoothing with 3 steps, the reference's residual
    thresholds after 5 cycles; each coarse operator is R A P of the level above (scipy, 1e-14)."""
    s = O.triangulated_grid(1, 1, 1 / 4, np.sqrt(3) / 8, False)
    md = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, 3, galerkin=True)
    direct = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, 3)
    L = csc(md.op(0))
    np.testing.assert_array_equal(L.toarray(), csc(direct.op(0)).toarray())
    for k in range(4):
        rap = csc(md.restriction(k)) @ csc(md.op(k)) @ csc(md.prolongation(k))
        Ac = csc(md.op(k + 1))
        assert abs(Ac - rap).max() <= 1e-14 * abs(rap).max()
    rng = np.random.default_rng(0)
    b = L @ rng.random(L.shape[0])
    u0 = np.zeros_like(b)
    rel = lambda u: np.linalg.norm(L @ u - b) / np.linalg.norm(b)
    assert rel(O.mu_cycles(md, u0, b, 5, 1)) < 2e-6   # V
    assert rel(O.mu_cycles(md, u0, b, 5, 2)) < 7e-7   # W
    assert rel(O.full_multigrid(md, b, 5, 1)) < 1e-3  # FMG-V
    assert rel(O.full_multigrid(md, b, 5, 2)) < 5e-6  # FMG-W
