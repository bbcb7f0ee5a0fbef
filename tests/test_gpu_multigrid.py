"""Parity of the GPU multigrid with the oracle.

* Hierarchy (MultigridData(s, BinarySubdivision(), levels, op, steps), Multigrid.jl:698-797):
  every level's orientation (what dualize's orient! produces) is bit-exact, and every level's
  operator A = L + shift I matches the oracle bit for bit.
* Cycles: the plain V-cycle (Chebyshev-Jacobi or damped Jacobi, dense coarsest solve) agrees with
  the oracle's CPU statement of the same algorithm to 1e-11 relative after 3 cycles (the GPU
  kernels contract FMAs; the oracle does not).
* Solves reach the requested relative residual ‖b - A u‖ / ‖b‖ (checked on the CPU with the
  oracle's operator) and the FP32-in-FP64 refinement solution is within 1e-7 of a direct FP64
  solve.
"""
import numpy as np
import pytest

from conftest import csc, uniform

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def icosahedron(O):
    return O.icosahedron()


CONFIGS = {
    # name: (coarse mesh builder, levels, center, shift, radius)
    "ico4_circum": (lambda O: O.icosahedron(), 4, "circumcenter", 1.0, 1.0),
    "grid_bary": (lambda O: O.triangulated_grid(1, 1, 1 / 4, np.sqrt(3) / 8, False), 3, "barycenter", 0.5, 0.0),
    "grid_circum_cw": (lambda O: O.tri_345(False), 4, "circumcenter", 2.0, 0.0),
}


def oracle_center(O, c):
    return O.CIRCUMCENTER if c == "circumcenter" else O.BARYCENTER


@pytest.fixture(scope="module")
def built(O, dec):
    out = {}
    for name, (mk, levels, center, shift, radius) in CONFIGS.items():
        coarse = mk(O)
        md = O.build_mg(coarse, levels, oracle_center(O, center), shift, radius, 3)
        mg = dec.MultigridData(coarse, levels, shift=shift, center=center, project_radius=radius)
        out[name] = (coarse, md, mg)
    return out


@pytest.mark.parametrize("name", list(CONFIGS))
def test_level_orientation_and_operator_bit_exact(O, built, name):
    coarse, md, mg = built[name]
    for lvl in range(md.nlevels):
        om = md.mesh(lvl)
        gm = mg.level_mesh(lvl)
        eo, to = gm.orientation()
        np.testing.assert_array_equal(eo, om.edge_orientation)
        np.testing.assert_array_equal(to, om.tri_orientation)
        ref = csc(md.op(lvl)).tocsr()
        ref.sort_indices()
        rp, ci, v, shape = mg.level_op(lvl).csr()
        np.testing.assert_array_equal(rp, ref.indptr)
        np.testing.assert_array_equal(ci, ref.indices)
        np.testing.assert_array_equal(v, ref.data)


def test_icosphere_level_counts(built):
    coarse, md, mg = built["ico4_circum"]
    for lvl in range(5):
        k = 4 - lvl
        nv, ne, nt, lmax = mg.level_info(lvl)
        assert (nv, ne, nt) == (10 * 4 ** k + 2, 30 * 4 ** k, 20 * 4 ** k)
        assert 1.0 < lmax < 2.2


@pytest.mark.parametrize("name", list(CONFIGS))
@pytest.mark.parametrize("smoother", [0, 1])
def test_plain_vcycles_match_oracle(O, dec, built, name, smoother):
    coarse, md, _ = built[name]
    mk, levels, center, shift, radius = CONFIGS[name]
    mg = dec.MultigridData(coarse, levels, shift=shift, center=center, project_radius=radius,
                           smoother=smoother, pre=2, post=2, omega=0.7, cheb_ratio=4.0)
    lmax = [mg.level_info(l)[3] for l in range(levels + 1)]
    n = mg.level_info(0)[0]
    b = uniform(5, n)
    u0 = uniform(6, n) * 0.1
    ref = O.plain_vcycles(md, u0, b, 3, smoother, 2, 2, 0.7, 4.0, lmax)
    u = mg.cycles(torch.tensor(u0, device="cuda"), torch.tensor(b, device="cuda"), 3).cpu().numpy()
    np.testing.assert_allclose(u, ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())


def test_wcycle_matches_oracle_structure(O, dec, built):
    """μ = 2: the coarse correction is computed twice (Multigrid.jl:866-869)."""
    coarse, md, _ = built["ico4_circum"]
    mgv = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, mu=1)
    mgw = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, mu=2)
    n = mgv.level_info(0)[0]
    A = csc(md.op(0))
    b = uniform(9, n)
    rel = lambda u: np.linalg.norm(b - A @ u) / np.linalg.norm(b)
    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    bt = torch.tensor(b, device="cuda")
    rv = rel(mgv.cycles(z.clone(), bt, 2).cpu().numpy())
    rw = rel(mgw.cycles(z.clone(), bt, 2).cpu().numpy())
    assert rw <= rv * 1.0001
    assert rw < 1e-2


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_solve_reaches_tolerance(O, dec, built, precision):
    """FP64, FP32 and FP16-storage V-cycles inside FP64 refinement all reach the requested residual
    and the direct FP64 solution."""
    import scipy.sparse.linalg as spla
    coarse, md, _ = built["ico4_circum"]
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=precision)
    n = mg.level_info(0)[0]
    A = csc(md.op(0)).tocsc()
    nrhs = 3
    B = np.stack([uniform(100 + j, n) for j in range(nrhs)])
    U = torch.zeros((nrhs, n), dtype=torch.float64, device="cuda")
    rtol = 1e-10
    U, rep = mg.solve(U, torch.tensor(B, device="cuda"), rtol=rtol, max_iters=60)
    assert rep.converged == 1
    U = U.cpu().numpy()
    for j in range(nrhs):
        rel = np.linalg.norm(B[j] - A @ U[j]) / np.linalg.norm(B[j])
        assert rel <= rtol * 1.0001
        exact = spla.spsolve(A, B[j])
        assert np.linalg.norm(U[j] - exact) / np.linalg.norm(exact) < 1e-7
    assert rep.max_rel_residual <= rtol


def test_panel_width_does_not_change_results(dec, built):
    coarse, md, _ = built["ico4_circum"]
    n = None
    res = []
    for K in (1, 4):
        mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, rhs_block=K)
        n = mg.level_info(0)[0]
        B = np.stack([uniform(200 + j, n) for j in range(4)])
        U = torch.zeros((4, n), dtype=torch.float64, device="cuda")
        mg.cycles(U, torch.tensor(B, device="cuda"), 2)
        res.append(U.cpu().numpy())
    np.testing.assert_allclose(res[0], res[1], rtol=1e-13, atol=1e-13)


def test_host_buffer_solve_matches_device(dec, built):
    coarse, md, _ = built["ico4_circum"]
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1)
    n = mg.level_info(0)[0]
    B = np.stack([uniform(300 + j, n) for j in range(2)])
    Uh = np.zeros_like(B)
    mg.solve_host(Uh, B, rtol=1e-8)
    Ud = torch.zeros((2, n), dtype=torch.float64, device="cuda")
    mg.solve(Ud, torch.tensor(B, device="cuda"), rtol=1e-8)
    np.testing.assert_array_equal(Uh, Ud.cpu().numpy())


def test_device_refinement_loop_steps(O, dec, built):
    """The refinement loop runs on the device (a graph whose WHILE node the residual test sets):
    the step count it reports is the first k at which a k-step solve meets rtol, a capped solve
    reports not-converged with the residual of the u it returns, and b = 0 needs no step."""
    coarse, md, _ = built["ico4_circum"]
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1)
    n = mg.n
    A = csc(md.op(0)).tocsc()
    B = np.stack([uniform(150 + j, n) for j in range(3)])
    Bd = torch.tensor(B, device="cuda")
    rtol = 1e-9
    U, rep = mg.solve(torch.zeros_like(Bd), Bd, rtol=rtol, max_iters=60)
    assert rep.converged == 1 and rep.iterations >= 2
    worst = []
    for k in range(1, rep.iterations + 1):
        Uk, rk = mg.solve(torch.zeros_like(Bd), Bd, rtol=rtol, max_iters=k)
        Uk = Uk.cpu().numpy()
        rel = max(np.linalg.norm(B[j] - A @ Uk[j]) / np.linalg.norm(B[j]) for j in range(3))
        assert rk.iterations == k
        assert rk.max_rel_residual == pytest.approx(rel, rel=1e-6)
        assert rk.converged == (1 if k == rep.iterations else 0)
        worst.append(rel)
    assert all(w > rtol for w in worst[:-1]) and worst[-1] <= rtol * 1.0001
    np.testing.assert_array_equal(Uk, U.cpu().numpy())
    Z, rz = mg.solve(torch.zeros_like(Bd), torch.zeros_like(Bd), rtol=rtol)
    assert rz.converged == 1 and rz.iterations == 0 and rz.max_rel_residual == 0.0
    assert float(Z.abs().max()) == 0.0


def test_host_driven_loop_matches_device_loop(dec, built):
    """device_loop = 0 (one graph launch per refinement step, the test on the host) takes the same
    steps and gives the same bits as the loop on the device."""
    coarse, md, _ = built["ico4_circum"]
    out = []
    for dl in (1, 0):
        mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1,
                               pre=0, post=2, cheb_ratio=3.0, inner_cycles=2, device_loop=dl)
        B = torch.tensor(np.stack([uniform(160 + j, mg.n) for j in range(3)]), device="cuda")
        U, rep = mg.solve(torch.zeros_like(B), B, rtol=1e-10, max_iters=60)
        out.append((U.cpu().numpy(), rep.iterations, rep.max_rel_residual, rep.converged))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1:] == out[1][1:] and out[0][3] == 1


@pytest.mark.parametrize("precision,device_loop", [(0, 1), (1, 1), (2, 1), (1, 0)])
def test_solve_from_zero_matches_zero_guess(dec, built, precision, device_loop):
    """dec_mg_solve_from_zero (u output only; the first residual is b itself) gives the same bits
    and steps as dec_mg_solve from a zeroed u, whatever u held before; b = 0 needs no step."""
    coarse, md, _ = built["ico4_circum"]
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=precision,
                           pre=0, post=2, cheb_ratio=3.0, inner_cycles=2, device_loop=device_loop)
    B = torch.tensor(np.stack([uniform(170 + j, mg.n) for j in range(5)]), device="cuda")
    B[3] = 0.0
    U0, r0 = mg.solve(torch.zeros_like(B), B, rtol=1e-10, max_iters=60)
    for _ in range(2):
        Uz, rz = mg.solve(torch.full_like(B, float("nan")), B, rtol=1e-10, max_iters=60, use_initial_guess=False)
        np.testing.assert_array_equal(Uz.cpu().numpy(), U0.cpu().numpy())
        assert (rz.iterations, rz.converged, rz.max_rel_residual) == (r0.iterations, 1, r0.max_rel_residual)
    assert float(Uz[3].abs().max()) == 0.0
    Z, rzz = mg.solve(torch.ones_like(B), torch.zeros_like(B), rtol=1e-10, use_initial_guess=False)
    assert rzz.iterations == 0 and rzz.converged == 1 and float(Z.abs().max()) == 0.0


def test_pipelined_host_solves_match_synchronous(dec, built):
    """solve_host_submit / wait: three solves in flight on the hierarchy's own streams give the
    same bits as the synchronous host-buffer solve; a fourth submit before a wait, a second wait on
    a ticket and the learned smoother are refused."""
    coarse, md, _ = built["ico4_circum"]
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1)
    n = mg.n
    sizes = [2, 3, 2, 1, 4]
    Bs = [torch.tensor(np.stack([uniform(700 + 10 * q + j, n) for j in range(m)])).pin_memory()
          for q, m in enumerate(sizes)]
    Us = [torch.zeros_like(B).pin_memory() for B in Bs]
    p0 = mg.solve_host_submit(Us[0], Bs[0], rtol=1e-9, use_initial_guess=False)
    p1 = mg.solve_host_submit(Us[1], Bs[1], rtol=1e-9, use_initial_guess=False)
    p2 = mg.solve_host_submit(Us[2], Bs[2], rtol=1e-9, use_initial_guess=False)
    with pytest.raises(dec.DecError, match="in flight"):
        mg.solve_host_submit(Us[3], Bs[3])
    _, r0 = p0.wait()
    p3 = mg.solve_host_submit(Us[3], Bs[3], rtol=1e-9, use_initial_guess=False)
    _, r1 = p1.wait()
    p4 = mg.solve_host_submit(Us[4], Bs[4], rtol=1e-9, use_initial_guess=False)
    reps = [r0, r1, p2.wait()[1], p3.wait()[1], p4.wait()[1]]
    with pytest.raises(dec.DecError, match="ticket"):
        rep = dec._capi.SolveReport()
        dec.check(dec.lib().dec_mg_solve_host_wait(mg._h, p4.ticket, dec._capi.C.byref(rep)))
    for q, m in enumerate(sizes):
        ref = np.zeros((m, n))
        _, rr = mg.solve_host(ref, Bs[q].numpy(), rtol=1e-9, use_initial_guess=False)
        np.testing.assert_array_equal(Us[q].numpy(), ref)
        assert reps[q].converged == 1 and reps[q].iterations == rr.iterations
        assert reps[q].max_rel_residual == rr.max_rel_residual and reps[q].seconds > 0
    # starting from the solution: no refinement step
    _, rg = mg.solve_host_submit(Us[0], Bs[0], rtol=1e-9, use_initial_guess=True).wait()
    assert rg.converged == 1 and rg.iterations == 0
    learned = dec.MultigridData(coarse, 2, shift=1.0, center="circumcenter", project_radius=1.0, smoother=3)
    with pytest.raises(dec.DecError, match="learned"):
        learned.solve_host_submit(np.zeros(learned.n), np.ones(learned.n))


def test_singular_coarse_operator_is_reported(O, dec):
    coarse = O.icosahedron()
    with pytest.raises(dec.DecError, match="singular"):
        dec.MultigridData(coarse, 1, shift=0.0, center="circumcenter", project_radius=1.0)


# ---- the reference's own algorithm on the GPU: V/W-cycles with the Krylov CG smoother ----------

def _ref_grid_setup(O, dec, steps, mu):
    # test/Multigrid.jl:54-90: triangulated_grid(1,1,1/4,√3/8), 4 binary levels, circumcentric
    # duals, the singular Laplacian (shift 0), steps CG iterations per smoothing.
    s = O.triangulated_grid(1, 1, 1 / 4, np.sqrt(3) / 8, False)
    md = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, steps)
    mg = dec.MultigridData(s, 4, shift=0.0, center="circumcenter", smoother=2, pre=steps, post=steps, mu=mu)
    L = csc(md.op(0))
    return md, mg, L


@pytest.mark.parametrize("mu", [1, 2])
def test_cg_cycles_match_oracle(O, dec, mu):
    """GPU mu-cycles with the Krylov CG smoother against the oracle's restatement of
    _multigrid_μ_cycle + Krylov.jl cg (reduction order differs: 1e-9 relative)."""
    md, mg, L = _ref_grid_setup(O, dec, 3, mu)
    n = L.shape[0]
    b = L @ ((uniform(0, n) + 1) / 2)
    u0 = np.zeros(n)
    for cycles in (1, 2, 4):
        ref = O.mu_cycles(md, u0, b, cycles, mu)
        u = mg.cycles(torch.zeros(n, dtype=torch.float64, device="cuda"), torch.tensor(b, device="cuda"), cycles)
        np.testing.assert_allclose(u.cpu().numpy(), ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


def test_cg_cycles_reference_thresholds(O, dec):
    """test/Multigrid.jl:67-78 on the GPU: 5 V-cycles and 5 W-cycles reach < 1e-7."""
    for mu in (1, 2):
        md, mg, L = _ref_grid_setup(O, dec, 3, mu)
        n = L.shape[0]
        b = L @ ((uniform(0, n) + 1) / 2)
        u = mg.cycles(torch.zeros(n, dtype=torch.float64, device="cuda"), torch.tensor(b, device="cuda"), 5)
        u = u.cpu().numpy()
        assert np.linalg.norm(L @ u - b) / np.linalg.norm(b) < 1e-7


def test_cg_zero_steps_does_no_smoothing(O, dec):
    """Issue #178 (test/Multigrid.jl:151-170): steps = 0 skips the smoother entirely."""
    md0, mg0, L = _ref_grid_setup(O, dec, 0, 1)
    md1, mg1, _ = _ref_grid_setup(O, dec, 1, 1)
    n = L.shape[0]
    b = L @ ((uniform(0, n) + 1) / 2)
    z = torch.zeros(n, dtype=torch.float64, device="cuda")
    bt = torch.tensor(b, device="cuda")
    r0 = np.linalg.norm(L @ mg0.cycles(z.clone(), bt, 5).cpu().numpy() - b)
    r1 = np.linalg.norm(L @ mg1.cycles(z.clone(), bt, 5).cpu().numpy() - b)
    assert r1 < r0
    np.testing.assert_allclose(mg0.cycles(z.clone(), bt, 5).cpu().numpy(), O.mu_cycles(md0, np.zeros(n), b, 5, 1),
                               rtol=1e-12, atol=1e-12)


def test_cg_cycles_multi_rhs_match_single(O, dec):
    md, mg, L = _ref_grid_setup(O, dec, 3, 1)
    n = L.shape[0]
    B = np.stack([L @ ((uniform(10 + j, n) + 1) / 2) for j in range(3)])
    U = mg.cycles(torch.zeros((3, n), dtype=torch.float64, device="cuda"), torch.tensor(B, device="cuda"), 3)
    for j in range(3):
        ref = O.mu_cycles(md, np.zeros(n), B[j], 3, 1)
        np.testing.assert_allclose(U[j].cpu().numpy(), ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


# ---- full multigrid (Multigrid.jl:826-855) ---------------------------------------------------

@pytest.mark.parametrize("mu", [1, 2])
def test_full_multigrid_cg_matches_oracle(O, dec, mu):
    """FMG with the reference's CG smoother against the oracle's full_multigrid, and the
    reference's thresholds (test/Multigrid.jl:79-83: FMG-V < 1e-6, FMG-W < 1e-7 after 5 cycles).
    The operator is the singular Laplacian (shift 0): constants are its null space, which the CG
    iterations leave to rounding, so the iterates are compared modulo a constant (1e-8)."""
    md, mg, L = _ref_grid_setup(O, dec, 3, mu)
    n = L.shape[0]
    b = L @ ((uniform(0, n) + 1) / 2)
    bt = torch.tensor(b, device="cuda")
    for cycles in (1, 5):
        ref = O.full_multigrid(md, b, cycles, mu)
        u = dec.full_multigrid(bt, mg, cycles).cpu().numpy()
        du, dr = u - u.mean(), ref - ref.mean()
        assert np.linalg.norm(du - dr) <= 1e-8 * np.linalg.norm(dr)
        assert np.linalg.norm(L @ (u - ref)) <= 1e-8 * np.linalg.norm(b)
    assert np.linalg.norm(L @ u - b) / np.linalg.norm(b) < (1e-6 if mu == 1 else 1e-7)


def test_full_multigrid_chebyshev(O, dec):
    """FMG with the stationary smoother and the dense coarsest solve: one FMG-V(3,3) pass on
    icosphere L5 Helmholtz already reduces the residual below 1e-2, and more cycles keep going."""
    coarse = O.icosahedron()
    md = O.build_mg(coarse, 5, O.CIRCUMCENTER, 1.0, 1.0, 3)
    mg = dec.MultigridData(coarse, 5, shift=1.0, center="circumcenter", project_radius=1.0, precision=0)
    A = csc(md.op(0))
    n = A.shape[0]
    B = np.stack([uniform(600 + j, n) for j in range(3)])
    rel = []
    for cycles in (1, 3):
        U = dec.full_multigrid(torch.tensor(B, device="cuda"), mg, cycles).cpu().numpy()
        rel.append(max(np.linalg.norm(B[j] - A @ U[j]) / np.linalg.norm(B[j]) for j in range(3)))
    assert rel[0] < 1e-2 and rel[1] < rel[0] * 1e-2


# ---- GalerkinMode (Multigrid.jl:740-748) ------------------------------------------------------

@pytest.mark.parametrize("mu", [1, 2])
def test_galerkin_hierarchy_and_cg_cycles(O, dec, mu):
    """Coarse operators R A P built by the library equal the oracle's bit for bit (the same
    column-by-column products in SparseArrays' order); the CG-smoother μ-cycles on them match
    the oracle's, and the reference's test_galerkin thresholds hold on the GPU."""
    s = O.triangulated_grid(1, 1, 1 / 4, np.sqrt(3) / 8, False)
    md = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, 3, galerkin=True)
    mg = dec.MultigridData(s, 4, shift=0.0, center="circumcenter", smoother=2, pre=3, post=3, mu=mu,
                           mode="galerkin")
    for k in range(5):
        ref = csc(md.op(k)).toarray()
        rp, ci, v, shape = mg.level_op(k).csr()
        import scipy.sparse as sp
        got = sp.csr_matrix((v, ci, rp), shape=shape).toarray()
        np.testing.assert_array_equal(got, ref)
    L = csc(md.op(0))
    n = L.shape[0]
    b = L @ ((uniform(0, n) + 1) / 2)
    u = mg.cycles(torch.zeros(n, dtype=torch.float64, device="cuda"), torch.tensor(b, device="cuda"), 5)
    u = u.cpu().numpy()
    ref = O.mu_cycles(md, np.zeros(n), b, 5, mu)
    assert np.linalg.norm((u - u.mean()) - (ref - ref.mean())) <= 1e-8 * np.linalg.norm(ref - ref.mean())
    rel = np.linalg.norm(L @ u - b) / np.linalg.norm(b)
    assert rel < (2e-6 if mu == 1 else 7e-7)
    f = dec.full_multigrid(torch.tensor(b, device="cuda"), mg, 5).cpu().numpy()
    assert np.linalg.norm(L @ f - b) / np.linalg.norm(b) < (1e-3 if mu == 1 else 5e-6)


def test_galerkin_mixed_precision_solve(O, dec):
    """GalerkinMode under the FP32-in-FP64 Chebyshev solve on an icosphere Helmholtz problem:
    reaches the tolerance and the direct solution; per-RHS shifts are refused."""
    import scipy.sparse.linalg as spla
    coarse = O.icosahedron()
    md = O.build_mg(coarse, 4, O.CIRCUMCENTER, 1.0, 1.0, 3, galerkin=True)
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1,
                           mode="galerkin")
    for k in (1, 4):
        rp, ci, v, shape = mg.level_op(k).csr()
        import scipy.sparse as sp
        np.testing.assert_array_equal(sp.csr_matrix((v, ci, rp), shape=shape).toarray(), csc(md.op(k)).toarray())
    A = csc(md.op(0)).tocsc()
    n = A.shape[0]
    B = np.stack([uniform(900 + j, n) for j in range(3)])
    U, rep = mg.solve(torch.zeros((3, n), dtype=torch.float64, device="cuda"), torch.tensor(B, device="cuda"),
                      rtol=1e-10, max_iters=60)
    assert rep.converged == 1
    U = U.cpu().numpy()
    for j in range(3):
        exact = spla.spsolve(A, B[j])
        assert np.linalg.norm(U[j] - exact) / np.linalg.norm(exact) < 1e-7
    with pytest.raises(dec.DecError, match="Galerkin"):
        dec.MultigridData(coarse, 2, shift=1.0, center="circumcenter", project_radius=1.0, coarse_solver=2,
                          mode="galerkin")


def test_solve_traffic_counts_the_graph(dec, built):
    """dec_mg_solve_traffic: linear in the refinement steps; a loop body moves at least its
    finest-level sweeps' bytes (dec_mg_time_kernel's figure for a middle Chebyshev step) and at most
    a few times a whole cycle's worth; a solve from zero moves fewer bytes than one from a guess."""
    coarse, md, _ = built["ico4_circum"]
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1,
                           pre=0, post=2, cheb_ratio=3.0, inner_cycles=2, rhs_block=4)
    B = torch.tensor(np.stack([uniform(180 + j, mg.n) for j in range(4)]), device="cuda")
    _, rep = mg.solve(torch.zeros_like(B), B, rtol=1e-9, use_initial_guess=False)
    t1, t2, t3 = (mg.solve_traffic(4, k) for k in (1, 2, 3))
    body = t2 - t1
    assert body > 0 and abs((t3 - t2) - body) <= 1e-9 * body
    _, sweep_bytes = mg.time_kernel(0, 0, 4, reps=1)
    assert body >= 2 * 2 * 0.9 * sweep_bytes          # inner_cycles x post finest sweeps
    assert body <= 8 * 2 * sweep_bytes
    assert mg.solve_traffic(4, 2, from_zero=True) < mg.solve_traffic(4, 2, from_zero=False)
    with pytest.raises(dec.DecError):
        dec.MultigridData(coarse, 2, shift=1.0, center="circumcenter", project_radius=1.0, smoother=2).solve_traffic(1, 1)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("smoother,pre,post", [(1, 0, 2), (1, 2, 2), (1, 1, 3), (0, 1, 1), (1, 0, 1)])
@pytest.mark.parametrize("nrhs,shifts", [(3, False), (32, False), (5, True)])
def test_prolongation_fused_into_sweeps(O, dec, precision, smoother, pre, post, nrhs, shifts):
    """The two Chebyshev steps after a prolongation with the prolonged iterate never stored
    (k_sweep_ap: A x0 = (A P) z; k_sweep_p: the previous iterate P z formed from the coarse panels;
    tuning key "pfuse": 1 where the level's iterate was zero, 2 also onto an iterate, 3 onto an iterate
    in correction form) against
    x (+)= P z stored by k_prolong and then swept: the same iterates up to the rounding of the
    regrouped products, on cycles from zero and from a guess, with per-RHS shifts, FP32 and FP64
    panels; the same refinement steps to 1e-9."""
    coarse = O.icosahedron()
    outs = []
    try:
        for fuse in (0, 1, 2, 3):
            dec.tune_set("pfuse", fuse)
            kw = dict(coarse_solver=2, coarse_max=170) if shifts else {}
            mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0,
                                   precision=precision, smoother=smoother, pre=pre, post=post, omega=0.7,
                                   cheb_ratio=3.0, inner_cycles=2, **kw)
            B = torch.tensor(np.stack([uniform(300 + j, mg.n) for j in range(nrhs)]), device="cuda")
            sh = np.exp(np.linspace(-1.0, 1.0, nrhs)) if shifts else None
            U = torch.tensor(np.stack([uniform(400 + j, mg.n) * 0.1 for j in range(nrhs)]), device="cuda")
            U, _ = mg.solve(U, B, rtol=1e-30, max_iters=3, shifts=sh)
            Uz, rep = mg.solve(torch.zeros_like(B), B, rtol=1e-9, max_iters=40, shifts=sh, use_initial_guess=False)
            assert rep.converged == 1
            outs.append((U.cpu().numpy(), Uz.cpu().numpy(), rep.iterations))
    finally:
        dec.tune_set("pfuse", 3)
    tol = 1e-12 if precision == 0 else 1e-5
    for o in outs[1:]:
        for a, b in ((outs[0][0], o[0]), (outs[0][1], o[1])):
            assert np.abs(a - b).max() <= tol * np.abs(a).max()
        assert outs[0][2] == o[2]
