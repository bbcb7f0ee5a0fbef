"""Per-right-hand-side shifts and batched solves over uneven meshes, on the GPU.

* coarse_solver = 2 keeps every level's operator the Laplacian (bit-exact with the oracle's
  L) and solves the coarsest level through its eigendecomposition, so each right-hand side can
  carry its own shift: the solutions of (L + c_j I) u_j = b_j match a direct sparse solve.
* For one common shift and the damped-Jacobi smoother (whose sweeps do not depend on the
  spectral bound, which coarse_solver 2 takes from the unshifted Laplacian), the
  eigendecomposition coarse solve gives the same cycles as the dense inverse.
* A batch over icospheres and a planar grid solves every group to the requested residual, each
  solution matching the direct solve, before and after per-group autotuning.
"""
import numpy as np
import pytest

from conftest import csc, uniform

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def grid9(O):
    return O.triangulated_grid(8, 8, 1.0, 1.0, False)  # 9 x 9 vertices


GROUPS = {
    # name: (coarse builder, levels, radius)
    "ico4": (lambda O: O.icosahedron(), 4, 1.0),
    "grid33": (grid9, 2, 0.0),
    "ico3": (lambda O: O.icosahedron(), 3, 1.0),
}


def _pair(O, dec, name, precision=1):
    mk, levels, radius = GROUPS[name]
    coarse = mk(O)
    md = O.build_mg(coarse, levels, O.CIRCUMCENTER, 0.0, radius, 3)
    mg = dec.MultigridData(coarse, levels, shift=0.0, center="circumcenter", project_radius=radius,
                           coarse_solver=2, precision=precision, coarse_max=170)
    return md, mg


def _check_solutions(L, B, U, shifts, rtol):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    n = L.shape[0]
    for j, c in enumerate(shifts):
        A = (L + c * sp.identity(n)).tocsc()
        assert np.linalg.norm(B[j] - A @ U[j]) / np.linalg.norm(B[j]) <= rtol * 1.0001
        exact = spla.spsolve(A, B[j])
        assert np.linalg.norm(U[j] - exact) / np.linalg.norm(exact) < 1e-7


@pytest.mark.parametrize("name", list(GROUPS))
@pytest.mark.parametrize("precision", [1, 2])
def test_shifted_solve_matches_direct(O, dec, name, precision):
    md, mg = _pair(O, dec, name, precision)
    L = csc(md.op(0))
    # every level stores the Laplacian itself
    ref = L.tocsr()
    ref.sort_indices()
    rp, ci, v, _ = mg.level_op(0).csr()
    np.testing.assert_array_equal(ci, ref.indices)
    np.testing.assert_array_equal(v, ref.data)
    n = L.shape[0]
    shifts = np.array([0.1, 1.0, 10.0, 0.37, 3.3])
    B = np.stack([uniform(300 + j, n) for j in range(len(shifts))])
    U, rep = mg.solve(torch.zeros((len(shifts), n), dtype=torch.float64, device="cuda"),
                      torch.tensor(B, device="cuda"), rtol=1e-10, max_iters=60, shifts=shifts)
    assert rep.converged == 1
    _check_solutions(L, B, U.cpu().numpy(), shifts, 1e-10)


def test_eigen_coarse_solve_matches_dense_inverse(O, dec):
    coarse = O.icosahedron()
    kw = dict(shift=1.0, center="circumcenter", project_radius=1.0, precision=0, coarse_max=170, smoother=0)
    mg0 = dec.MultigridData(coarse, 4, coarse_solver=0, **kw)
    mg2 = dec.MultigridData(coarse, 4, coarse_solver=2, **kw)
    n = mg0.n
    B = torch.tensor(np.stack([uniform(320 + j, n) for j in range(3)]), device="cuda")
    u0 = mg0.cycles(torch.zeros_like(B), B, 3).cpu().numpy()
    u2 = mg2.cycles(torch.zeros_like(B), B, 3).cpu().numpy()
    np.testing.assert_allclose(u2, u0, rtol=1e-11, atol=1e-11 * np.abs(u0).max())


def test_shifts_need_eigen_coarse_solver(O, dec):
    mg = dec.MultigridData(O.icosahedron(), 2, shift=1.0, center="circumcenter", project_radius=1.0)
    b = torch.ones((2, mg.n), dtype=torch.float64, device="cuda")
    with pytest.raises(dec.DecError, match="coarse_solver"):
        mg.solve(torch.zeros_like(b), b, shifts=[1.0, 2.0])
    md, mg2 = _pair(O, dec, "ico3")
    with pytest.raises(dec.DecError, match="positive"):
        mg2.solve(torch.zeros((2, mg2.n), dtype=torch.float64, device="cuda"),
                  torch.ones((2, mg2.n), dtype=torch.float64, device="cuda"), shifts=[1.0, 0.0])


def test_batch_over_uneven_meshes(O, dec):
    names = list(GROUPS)
    pairs = [_pair(O, dec, nm) for nm in names]
    batch = dec.Batch([mg for _, mg in pairs])
    rng = np.random.default_rng(3)
    nrhs = [5, 3, 7]
    Bs, Us, shifts = [], [], []
    for q, (md, mg) in enumerate(pairs):
        n = mg.n
        Bs.append(np.stack([uniform(400 + 10 * q + j, n) for j in range(nrhs[q])]))
        shifts.append(np.exp(rng.uniform(np.log(0.1), np.log(10.0), nrhs[q])))
    for autotuned in (False, True):
        if autotuned:
            batch.autotune(nrhs, reps=2)
        Us = [torch.zeros((nrhs[q], pairs[q][1].n), dtype=torch.float64, device="cuda") for q in range(3)]
        reps, tot = batch.solve(Us, [torch.tensor(B, device="cuda") for B in Bs], shifts=shifts, rtol=1e-9)
        assert tot.converged == 1 and tot.launches > 0
        # algorithmic bytes: at least every caller vector in and out, and linear in the steps
        by0, by1, byk = batch.traffic(0), batch.traffic(1), batch.traffic(tot.iterations)
        assert by0 > 3 * 8 * sum(nrhs[q] * pairs[q][1].n for q in range(3)) and by1 > by0
        assert byk == pytest.approx(by0 + tot.iterations * (by1 - by0), rel=1e-12)
        for q, (md, mg) in enumerate(pairs):
            assert reps[q].converged == 1 and reps[q].iterations <= tot.iterations
            _check_solutions(csc(md.op(0)), Bs[q], Us[q].cpu().numpy(), shifts[q], 1e-9)
            # every group takes the batch's steps; its own solve held to as many gives the same bits
            U1 = torch.zeros_like(Us[q])
            mg.solve(U1, torch.tensor(Bs[q], device="cuda"), rtol=1e-30, max_iters=tot.iterations, shifts=shifts[q])
            np.testing.assert_array_equal(U1.cpu().numpy(), Us[q].cpu().numpy())
    # the batch is one graph launch: its kernels are the graph's nodes outside the loop plus the
    # loop body's per step, and new caller buffers rebuild the graph with the same result
    again = [torch.zeros_like(U) for U in Us]
    reps2, tot2 = batch.solve(again, [torch.tensor(B, device="cuda") for B in Bs], shifts=shifts, rtol=1e-9)
    assert tot2.iterations == tot.iterations and tot2.launches == tot.launches
    for q in range(3):
        np.testing.assert_array_equal(again[q].cpu().numpy(), Us[q].cpu().numpy())
    capped, totc = batch.solve([torch.zeros_like(U) for U in Us], [torch.tensor(B, device="cuda") for B in Bs],
                               shifts=shifts, rtol=1e-30, max_iters=2)
    assert totc.converged == 0 and totc.iterations == 2


@pytest.mark.parametrize("kind,m,n", [("pp", 0, 1), ("pp", 1, 0), ("pp", 0, 2), ("pp", 2, 0), ("pp", 1, 1),
                                      ("dd", 0, 1), ("dd", 1, 0), ("pd", 0, 1), ("dp", 1, 0), ("pd", 1, 1),
                                      ("dp", 1, 1)])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_batched_wedge_equals_single_applications(dec, kind, m, n, dtype):
    """dec_wedge_apply_batched (one launch, pairs along grid.y) is bit-identical to applying the
    plan to each pair."""
    mesh = dec.meshes.icosphere(3)
    g = dec.Mesh(mesh.points, mesh.ev0, mesh.ev1, mesh.te0, mesh.te1, mesh.te2, mesh.edge_orientation,
                 mesh.tri_orientation, center="circumcenter")
    make = {"pp": dec.dec_wedge_product, "dd": dec.dec_wedge_product_dd, "pd": dec.dec_wedge_product_pd,
            "dp": dec.dec_wedge_product_dp}[kind]
    w = make(m, n, g, dtype)
    la, lb, lo = w.len_a, w.len_b, w.len_out
    tdt = torch.float64 if dtype == "float64" else torch.float32
    count = 7
    a = torch.tensor(np.stack([uniform(500 + j, la) for j in range(count)]), dtype=tdt, device="cuda")
    b = torch.tensor(np.stack([uniform(600 + j, lb) for j in range(count)]), dtype=tdt, device="cuda")
    out = torch.empty((count, lo), dtype=tdt, device="cuda")
    w.batched(a, b, out)
    for j in range(count):
        np.testing.assert_array_equal(out[j].cpu().numpy(), w(a[j], b[j]).cpu().numpy())
