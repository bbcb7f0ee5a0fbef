"""Caller matrices on the device: `dec_op_create_csc` (the reference's A * x on a SparseMatrixCSC)
and `dec_mg_create_from_csc`, the hierarchy of MultigridData(g, r, p, s) (src/Multigrid.jl:538-546)
with per-level steps (:542, :858-871).

* A caller operator applies bit for bit like the oracle's SparseArrays-order CSC product (FP64,
  square and rectangular, 0- and 1-based).
* The oracle's own binary-subdivision hierarchy passed as matrices runs the same V-cycle as the
  hierarchy the library builds from the mesh (Chebyshev, 1e-11 against the oracle's statement).
* Operators that are not L + cI -- the ⋆0-weighted Helmholtz operator d0ᵀ⋆1d0 + c⋆0 on every level,
  and GalerkinMode's R A P -- with per-level steps run the reference's cycle (Krylov CG smoother)
  as the oracle does, to 1e-9 (dot-product reduction orders differ), V and W; the mixed-precision
  Chebyshev solve on them reaches 1e-10 and the direct solution.
* dec_mg_set_level_steps on a mesh hierarchy gives the oracle's cycle with the same steps.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import csc, uniform

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _tuple(A):
    A = sp.csc_matrix(A)
    A.sort_indices()
    return (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64), A.shape)


def _random_sparse(seed, m, n, density):
    rng = np.random.default_rng(seed)
    A = sp.random(m, n, density=density, random_state=rng, format="csc")
    A.data = rng.uniform(-1, 1, A.nnz)
    return A


@pytest.mark.parametrize("shape", [(300, 300), (257, 411), (500, 120)])
@pytest.mark.parametrize("base", [0, 1])
def test_sparse_operator_matches_oracle_product(O, dec, shape, base):
    A = _random_sparse(sum(shape) + base, shape[0], shape[1], 0.03)
    op = dec.sparse_operator(A, index_base=base)
    assert op.shape == shape
    x = uniform(11, shape[1])
    y = op(torch.tensor(x, device="cuda")).cpu().numpy()
    np.testing.assert_array_equal(y, O.csc_matvec(_tuple(A), x))
    rp, ci, v, _ = op.csr()
    R = A.tocsr()
    R.sort_indices()
    np.testing.assert_array_equal(rp, R.indptr)
    np.testing.assert_array_equal(ci, R.indices)
    np.testing.assert_array_equal(v, R.data)
    op32 = dec.sparse_operator(A, dtype="float32")
    y32 = op32(torch.tensor(x, dtype=torch.float32, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(y32, A @ x, rtol=1e-5, atol=1e-5 * np.abs(A @ x).max())


def _oracle_matrices(md):
    nl = md.nlevels
    return ([md.op(k) for k in range(nl)], [md.restriction(k) for k in range(nl - 1)],
            [md.prolongation(k) for k in range(nl - 1)])


def test_binary_hierarchy_as_matrices_runs_the_mesh_cycle(O, dec):
    ico = O.icosahedron()
    md = O.build_mg(ico, 4, O.CIRCUMCENTER, 1.0, 1.0, 3)
    ops, rs, ps = _oracle_matrices(md)
    opts = dict(smoother=1, pre=2, post=2, cheb_ratio=4.0, precision=0)
    mgc = dec.MultigridData.from_matrices(ops, rs, ps, **opts)
    mgm = dec.MultigridData(ico, 4, shift=1.0, center="circumcenter", project_radius=1.0, **opts)
    assert [mgc.level_info(l)[0] for l in range(5)] == [10 * 4 ** (4 - l) + 2 for l in range(5)]
    n = mgc.n
    b = uniform(21, n)
    u0 = uniform(22, n) * 0.1
    lmax = [mgc.level_info(l)[3] for l in range(5)]
    ref = O.plain_vcycles(md, u0, b, 3, 1, 2, 2, 0.8, 4.0, lmax)
    uc = mgc.cycles(torch.tensor(u0, device="cuda"), torch.tensor(b, device="cuda"), 3).cpu().numpy()
    np.testing.assert_allclose(uc, ref, rtol=0, atol=1e-11 * np.abs(ref).max())
    # the mesh-built hierarchy (Morton-ordered levels, its own λ estimates) against the same statement
    lmax_m = [mgm.level_info(l)[3] for l in range(5)]
    ref_m = O.plain_vcycles(md, u0, b, 3, 1, 2, 2, 0.8, 4.0, lmax_m)
    um = mgm.cycles(torch.tensor(u0, device="cuda"), torch.tensor(b, device="cuda"), 3).cpu().numpy()
    np.testing.assert_allclose(um, ref_m, rtol=0, atol=1e-11 * np.abs(ref_m).max())
    for l in range(5):  # the level operators are the caller's, in the caller's numbering
        rp, ci, v, shape = mgc.level_op(l).csr()
        R = csc(ops[l]).tocsr()
        R.sort_indices()
        np.testing.assert_array_equal(v, R.data)
    with pytest.raises(dec.DecError, match="no level meshes"):
        mgc.level_mesh(0)


def _star_weighted(O, md, c):
    """d0ᵀ ⋆1 d0 + c ⋆0 on every level: ⋆0 (L + c I), symmetric, not of the form L + c I."""
    out = []
    for k in range(md.nlevels):
        d = O.dualize(md.mesh(k), O.CIRCUMCENTER)
        s0 = O.hodge_diag(d, 0)
        L = csc(md.op(k))
        out.append(_tuple(sp.diags(s0) @ (L + c * sp.identity(L.shape[0]))))
    return out


@pytest.mark.parametrize("mu", [1, 2])
def test_star_weighted_operator_cg_cycles_with_level_steps(O, dec, mu):
    s = O.triangulated_grid(1, 1, 1 / 4, np.sqrt(3) / 8, False)
    md0 = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, 3)
    ops = _star_weighted(O, md0, 0.5)
    _, rs, ps = _oracle_matrices(md0)
    steps = [3, 2, 2, 1, 4]
    md = O.mgdata_from_csc(ops, rs, ps, steps)
    mg = dec.MultigridData.from_matrices(ops, rs, ps, steps=steps, smoother=2, mu=mu)
    n = mg.n
    A = csc(ops[0])
    b = A @ ((uniform(30, n) + 1) / 2)
    for cycles in (1, 2, 4):
        ref = O.mu_cycles(md, np.zeros(n), b, cycles, mu)
        u = mg.cycles(torch.zeros(n, dtype=torch.float64, device="cuda"), torch.tensor(b, device="cuda"), cycles)
        np.testing.assert_allclose(u.cpu().numpy(), ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    # the reference's cycle converges on it (slowly: Krylov cg with few steps on a weighted operator)
    assert np.linalg.norm(A @ u.cpu().numpy() - b) / np.linalg.norm(b) < 1e-3


def test_galerkin_matrices_cg_cycles(O, dec):
    s = O.triangulated_grid(1, 1, 1 / 4, np.sqrt(3) / 8, False)
    md = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, 3, galerkin=True)
    ops, rs, ps = _oracle_matrices(md)
    mg = dec.MultigridData.from_matrices(ops, rs, ps, steps=3, smoother=2)
    n = mg.n
    L = csc(ops[0])
    b = L @ ((uniform(31, n) + 1) / 2)
    ref = O.mu_cycles(md, np.zeros(n), b, 5, 1)
    u = mg.cycles(torch.zeros(n, dtype=torch.float64, device="cuda"), torch.tensor(b, device="cuda"), 5).cpu().numpy()
    # the singular Laplacian: compare modulo constants, as the library's own Galerkin test does
    assert np.linalg.norm((u - u.mean()) - (ref - ref.mean())) <= 1e-8 * np.linalg.norm(ref - ref.mean())
    assert np.linalg.norm(L @ u - b) / np.linalg.norm(b) < 2e-6   # the reference's V threshold


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_star_weighted_mixed_precision_solve(O, dec, precision):
    """The ⋆0-weighted operator is symmetric, so its hierarchy restricts with R = Pᵀ = S (the
    reference's row-normalised R suits the pointwise L + cI form): the Chebyshev solve in FP64,
    FP32 and FP16 storage inside FP64 refinement reaches 1e-10 and the direct solution."""
    import scipy.sparse.linalg as spla
    ico = O.icosahedron()
    md0 = O.build_mg(ico, 4, O.CIRCUMCENTER, 0.0, 1.0, 3)
    ops = _star_weighted(O, md0, 1.0)
    _, _, ps = _oracle_matrices(md0)
    rs = [_tuple(csc(P).T) for P in ps]
    mg = dec.MultigridData.from_matrices(ops, rs, ps, smoother=1, pre=0, post=2, cheb_ratio=3.0,
                                         inner_cycles=2, precision=precision)
    n = mg.n
    A = csc(ops[0]).tocsc()
    B = np.stack([uniform(40 + j, n) for j in range(3)])
    U, rep = mg.solve(torch.zeros((3, n), dtype=torch.float64, device="cuda"), torch.tensor(B, device="cuda"),
                      rtol=1e-10, max_iters=60, use_initial_guess=False)
    assert rep.converged == 1
    U = U.cpu().numpy()
    for j in range(3):
        assert np.linalg.norm(B[j] - A @ U[j]) / np.linalg.norm(B[j]) <= 1e-10 * 1.0001
        exact = spla.spsolve(A, B[j])
        assert np.linalg.norm(U[j] - exact) / np.linalg.norm(exact) < 1e-8


def test_level_steps_on_mesh_hierarchy(O, dec):
    s = O.triangulated_grid(1, 1, 1 / 4, np.sqrt(3) / 8, False)
    md = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, 3)
    mg = dec.MultigridData(s, 4, shift=0.0, center="circumcenter", smoother=2, pre=3, post=3)
    steps = [2, 3, 0, 1, 2]
    md.set_level_steps(steps)
    mg.set_level_steps(steps)
    n = mg.n
    L = csc(md.op(0))
    b = L @ ((uniform(32, n) + 1) / 2)
    ref = O.mu_cycles(md, np.zeros(n), b, 3, 1)
    u = mg.cycles(torch.zeros(n, dtype=torch.float64, device="cuda"), torch.tensor(b, device="cuda"), 3)
    np.testing.assert_allclose(u.cpu().numpy(), ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    mg.set_level_steps(None)  # back to pre = post = 3 everywhere
    md.set_steps(3)
    ref3 = O.mu_cycles(md, np.zeros(n), b, 3, 1)
    u3 = mg.cycles(torch.zeros(n, dtype=torch.float64, device="cuda"), torch.tensor(b, device="cuda"), 3)
    np.testing.assert_allclose(u3.cpu().numpy(), ref3, rtol=1e-9, atol=1e-9 * np.abs(ref3).max())


def test_from_matrices_rejects_bad_input(O, dec):
    ico = O.icosahedron()
    md = O.build_mg(ico, 2, O.CIRCUMCENTER, 1.0, 1.0, 3)
    ops, rs, ps = _oracle_matrices(md)
    with pytest.raises(dec.DecError, match="restriction"):
        dec.MultigridData.from_matrices(ops, [ps[0], rs[1]], ps)
    with pytest.raises(dec.DecError, match="learned|CG, Jacobi or Chebyshev"):
        dec.MultigridData.from_matrices(ops, rs, ps, smoother=3)
    zero_diag = list(ops)
    Z = csc(ops[1]).tolil()
    Z[3, 3] = 0.0
    zero_diag[1] = _tuple(Z.tocsc())
    with pytest.raises(dec.DecError, match="nonzero diagonal"):
        dec.MultigridData.from_matrices(zero_diag, rs, ps, smoother=1)
