"""The learned smoother on the GPU against the oracle.

* Initialisation: Xavier-uniform from the splitmix64 stream of the seed, bit for bit.
* Inference on the tensor cores (mma.sync, and tcgen05 with TMEM accumulators; BF16 operands,
  FP32 accumulation) and the CUDA-core forward agree with the oracle's mlp_forward (same BF16
  roundings; FP32 against FP64 accumulation); the two tensor-core engines agree with each other.
* The backward kernels' parameter gradient agrees with the oracle's mlp_backward, both for
  given (features, dL/dy) and for the full energy-norm training loss on a mesh.
* The features of a residual field are bit-exact with a float32 numpy statement of them.
* One learned V-cycle matches a numpy statement built on the oracle's hierarchy and MLP.
* Training lowers the loss; the trained network smooths better per cycle than damped Jacobi and
  than Chebyshev-Jacobi (the solver's plain smoother, the method without the network); a diverging
  network hands over to the plain smoother; checkpoints round-trip and reject corruption.
"""
import numpy as np
import pytest

from conftest import csc, uniform
from test_oracle_mlp import OFF_B1, OFF_B2, OFF_B3, OFF_W1, OFF_W2, OFF_W3, jacobi_net, xavier

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def np_features(A, r):
    """float32 statement of the feature kernel on a CSR operator with sorted columns."""
    A = A.tocsr()
    A.sort_indices()
    n = A.shape[0]
    F = np.zeros((n, 16), np.float32)
    dsc = np.zeros(n, np.float32)
    f32 = np.float32
    for i in range(n):
        cols = A.indices[A.indptr[i]:A.indptr[i + 1]]
        vals = A.data[A.indptr[i]:A.indptr[i + 1]]
        di = f32(vals[cols == i].sum())
        nb, cp, sabs = [], [], f32(0)
        for c, v in zip(cols, vals):
            if c == i:
                continue
            o = f32(v)
            sabs = f32(sabs + abs(o))
            if len(nb) < 6:
                nb.append(f32(r[c]))
                cp.append(f32(o / di))
        ri = f32(r[i])
        s = abs(ri)
        for v in nb:
            s = max(s, abs(v))
        if s == 0:
            s = f32(1)
        inv = f32(f32(1) / s)
        F[i, 0] = ri * inv
        for q, (v, c) in enumerate(zip(nb, cp)):
            F[i, 1 + q] = v * inv
            F[i, 7 + q] = c
        F[i, 13] = f32(1) - f32(sabs / di)
        F[i, 14] = f32(len(nb)) * (f32(1) / f32(6))
        dsc[i] = f32(s / di)
    return F, dsc


@pytest.fixture(scope="module")
def ico3(O, dec):
    """Icosphere L3 Helmholtz hierarchy (shift 1) on the GPU and in the oracle."""
    coarse = O.icosahedron()
    md = O.build_mg(coarse, 3, O.CIRCUMCENTER, 1.0, 1.0, 3)
    mg = dec.MultigridData(coarse, 3, shift=1.0, center="circumcenter", project_radius=1.0, precision=0)
    return md, mg


def test_xavier_init_bit_exact(dec):
    m = dec.SmootherMLP(4)
    np.testing.assert_array_equal(m.params, xavier(4))
    assert m.step == 0
    assert not np.array_equal(dec.SmootherMLP(5).params, m.params)


@pytest.mark.parametrize("tensor_cores", [True, False, 2])
def test_forward_matches_oracle(O, dec, tensor_cores):
    m = dec.SmootherMLP(4)
    rng = np.random.default_rng(3)
    p = m.params
    p[OFF_B1:OFF_W2] = rng.uniform(-0.2, 0.2, 64)
    p[OFF_B2:OFF_W3] = rng.uniform(-0.2, 0.2, 64)
    p[OFF_B3] = 0.1
    m.params = p
    n = 10007  # not a multiple of the 32-sample tile
    x = rng.uniform(-1, 1, (n, 16)).astype(np.float32)
    x[:5] = 0.0
    y = m.eval(torch.tensor(x, device="cuda"), tensor_cores=tensor_cores).cpu().numpy().astype(np.float64)
    ref = O.mlp_forward(p, x)
    err = np.abs(y - ref)
    scale = np.abs(ref).max()
    # FP32 against FP64 accumulation; a hidden unit whose BF16 rounding lands on the other side
    # of a tie moves y by a few 1e-4 of its scale at most
    assert err.max() <= 2e-3 * scale
    assert np.median(err) <= 2e-5 * scale


@pytest.mark.parametrize("tensor_cores", [1, 2])
def test_jacobi_network_on_tensor_cores(dec, tensor_cores):
    m = dec.SmootherMLP(4)
    m.params = jacobi_net(np.float32(0.8))
    x = torch.zeros((300, 16), dtype=torch.float32, device="cuda")
    x[:, 0] = torch.linspace(-1, 1, 300, device="cuda")
    y = m.eval(x, tensor_cores=tensor_cores).cpu().numpy()
    f0 = x[:, 0].to(torch.bfloat16).float().cpu().numpy()
    np.testing.assert_allclose(y, np.float32(0.8) * f0, rtol=0, atol=1e-7)


def test_tcgen05_matches_mma_sync(dec):
    """Both engines round the same products to BF16 and accumulate in FP32; only the order of
    the FP32 sums differs, so the outputs agree to a few FP32 ulps of the hidden sums except
    where a BF16 rounding of a hidden unit flips."""
    m = dec.SmootherMLP(7)
    rng = np.random.default_rng(8)
    for n in (1, 127, 128, 129, 70001):
        x = torch.tensor(rng.uniform(-1, 1, (n, 16)).astype(np.float32), device="cuda")
        y1 = m.eval(x, tensor_cores=1).cpu().numpy()
        y2 = m.eval(x, tensor_cores=2).cpu().numpy()
        d = np.abs(y1 - y2)
        scale = max(np.abs(y1).max(), 1e-30)
        assert d.max() <= 2e-3 * scale
        assert np.mean(d <= 1e-5 * scale) >= 0.99
    with pytest.raises(dec.DecError, match="engine"):
        dec.check(dec.lib().dec_mlp_set_engine(m._h, 2))


def test_grad_matches_oracle(O, dec):
    m = dec.SmootherMLP(11)
    rng = np.random.default_rng(5)
    p = m.params
    p[OFF_B1:OFF_W2] = rng.uniform(-0.2, 0.2, 64)
    p[OFF_B2:OFF_W3] = rng.uniform(-0.2, 0.2, 64)
    m.params = p
    n = 3000
    x = rng.uniform(-1, 1, (n, 16)).astype(np.float32)
    dy = rng.uniform(-1, 1, n).astype(np.float32)
    g = m.grad(torch.tensor(x, device="cuda"), torch.tensor(dy, device="cuda")).cpu().numpy().astype(np.float64)
    ref = O.mlp_backward(p, x, dy.astype(np.float64))
    for a, b in ((OFF_W1, OFF_B1), (OFF_B1, OFF_W2), (OFF_W2, OFF_B2), (OFF_B2, OFF_W3), (OFF_W3, OFF_B3),
                 (OFF_B3, OFF_B3 + 1)):
        np.testing.assert_allclose(g[a:b], ref[a:b], rtol=0, atol=2e-3 * np.abs(ref[a:b]).max() + 1e-6)
    assert np.linalg.norm(g - ref) <= 1e-3 * np.linalg.norm(ref)


def test_features_bit_exact(O, dec, ico3):
    md, mg = ico3
    op = mg.level_op(0)
    A = csc(md.op(0))
    n = A.shape[0]
    R = np.stack([uniform(40, n), uniform(41, n) * 1e-3])
    R[1, :7] = 0.0  # a patch of zero residuals (scale 1)
    F, sc = dec.SmootherMLP.features(op, torch.tensor(R, device="cuda"))
    F, sc = F.cpu().numpy(), sc.cpu().numpy()
    for s in range(2):
        Fr, dr = np_features(A, R[s])
        np.testing.assert_array_equal(F[s * n:(s + 1) * n], Fr)
        np.testing.assert_array_equal(sc[s * n:(s + 1) * n], dr)


def test_loss_and_gradient_match_oracle(O, dec, ico3):
    md, mg = ico3
    op = mg.level_op(0)
    A = csc(md.op(0)).tocsr()
    n = A.shape[0]
    star0 = O.hodge_diag(O.dualize(md.mesh(0), O.CIRCUMCENTER), 0)
    m = dec.SmootherMLP(4)
    p = m.params
    S = 3
    R = np.stack([uniform(60 + s, n) for s in range(S)])
    loss, g = m.loss_grad(op, torch.tensor(R, device="cuda"))
    g = g.cpu().numpy().astype(np.float64)
    # the loss on the CPU: features, oracle forward, A δ, energy terms, oracle backward
    diag = A.diagonal()
    ref_loss, X, DY = 0.0, [], []
    for s in range(S):
        F, dsc = np_features(A, R[s])
        d = dsc.astype(np.float64) * O.mlp_forward(p, F)
        q = A @ d
        ns = np.sum(star0 * R[s] ** 2 / diag)
        w = star0 / (ns * S)
        ref_loss += np.sum(w * d * (q - 2 * R[s]))
        X.append(F)
        DY.append(2 * w * (q - R[s]) * dsc)
    ref_g = O.mlp_backward(p, np.concatenate(X), np.concatenate(DY))
    assert loss == pytest.approx(ref_loss, rel=1e-3)
    assert np.linalg.norm(g - ref_g) <= 5e-3 * np.linalg.norm(ref_g)


def _learned_sweep(O, p, A, x, b):
    r = b - A @ x
    F, dsc = np_features(A, r)
    return x + dsc.astype(np.float64) * O.mlp_forward(p, F)


@pytest.mark.parametrize("engine", ["mma", "tcgen05"])
def test_learned_vcycle_matches_numpy(O, dec, engine):
    coarse = O.icosahedron()
    md = O.build_mg(coarse, 2, O.CIRCUMCENTER, 1.0, 1.0, 3)
    mg = dec.MultigridData(coarse, 2, shift=1.0, center="circumcenter", project_radius=1.0, precision=0,
                           smoother=3, pre=2, post=1)
    mlp = dec.SmootherMLP(4)
    p = mlp.params
    p[OFF_W3:OFF_B3] *= 0.3
    mlp.params = p
    mlp.set_engine(engine)
    mg.set_smoother_mlp(mlp)
    ops = [csc(md.op(l)).tocsr() for l in range(3)]
    Rs = [csc(md.restriction(l)).tocsr() for l in range(2)]
    Ps = [csc(md.prolongation(l)).tocsr() for l in range(2)]

    def cycle(l, x, b):
        if l == 2:
            return np.linalg.solve(ops[2].toarray(), b)
        for _ in range(2):
            x = _learned_sweep(O, p, ops[l], x, b)
        z = cycle(l + 1, np.zeros(ops[l + 1].shape[0]), Rs[l] @ (b - ops[l] @ x))
        x = x + Ps[l] @ z
        return _learned_sweep(O, p, ops[l], x, b)

    n = ops[0].shape[0]
    b = uniform(70, n)
    u0 = uniform(71, n) * 0.1
    ref = cycle(0, u0, b)
    u = mg.cycles(torch.tensor(u0, device="cuda"), torch.tensor(b, device="cuda"), 1).cpu().numpy()
    assert np.linalg.norm(u - ref) <= 1e-3 * np.linalg.norm(ref - u0)


@pytest.fixture(scope="module")
def trained(O, dec):
    """A network trained for 400 Adam steps on white-noise-error residuals of icosphere L4."""
    from dec_b200 import learned
    _, op, R = learned.residual_fields(4, 12, shift=1.0, cycles=(0,))
    mlp = dec.SmootherMLP(4)
    l0, _ = mlp.loss_grad(op, R[:6], grad=False)
    losses = mlp.train(op, R[:6], 400, lr=1e-3, batch=65536, seed=4, record_loss=True)
    l1, _ = mlp.loss_grad(op, R[6:], grad=False)  # held-out fields
    return mlp, l0, losses, l1


def test_training_lowers_loss(trained):
    mlp, l0, losses, l1 = trained
    assert mlp.step == 400
    assert losses[0] == pytest.approx(l0, rel=1e-9)
    assert losses[-1] < min(0.0, losses[0]) - 0.5
    assert l1 < 0  # on held-out fields the step lowers the energy error


def test_trained_network_beats_best_damped_jacobi_loss(dec, trained):
    """Damped Jacobi is one point of the network family; training goes past its best damping."""
    from dec_b200 import learned
    _, op, R = learned.residual_fields(4, 4, shift=1.0, cycles=(0,), seed=500)
    jac = dec.SmootherMLP(4)
    best = 0.0
    for omega in (0.5, 0.6, 0.67, 0.75, 0.8, 0.9, 1.0):
        jac.params = jacobi_net(np.float32(omega))
        best = min(best, jac.loss_grad(op, R, grad=False)[0])
    assert trained[0].loss_grad(op, R, grad=False)[0] < best


def _rates(dec, O, smoother, mlp=None, cycles=4, pre=2, post=2):
    coarse = O.icosahedron()
    mg = dec.MultigridData(coarse, 5, shift=1.0, center="circumcenter", project_radius=1.0, precision=0,
                           smoother=smoother, pre=pre, post=post, omega=0.8)
    if mlp is not None:
        mg.set_smoother_mlp(mlp)
    n = mg.n
    B = torch.tensor(np.stack([uniform(80 + j, n) for j in range(4)]), device="cuda")
    U = torch.zeros_like(B)
    mg.cycles(U, B, cycles)
    op = mg.level_op(0)
    r, bn = op.residual_norms(U, B)
    return np.max(r / bn)


def test_trained_network_beats_jacobi(O, dec, trained):
    """The gain: the same V(2,2) cycles with the network's sweeps in place of damped Jacobi."""
    mlp = trained[0]
    rel_learned = _rates(dec, O, 3, mlp)
    rel_jacobi = _rates(dec, O, 0)
    assert rel_learned < 0.5 * rel_jacobi


def test_trained_network_against_chebyshev(O, dec, trained):
    """The solver's plain smoother is Chebyshev-Jacobi: per V(2,2) cycle the network's sweeps against
    it (and damped Jacobi), 4 cycles on icosphere L5."""
    mlp = trained[0]
    rel = {"learned": _rates(dec, O, 3, mlp), "chebyshev": _rates(dec, O, 1), "jacobi": _rates(dec, O, 0),
           "learned V(1,1)": _rates(dec, O, 3, mlp, pre=1, post=1)}
    print("relative residual after 4 cycles:", rel)
    # measured on a B200: learned 1.2e-6, Chebyshev 2.7e-5, damped Jacobi 4.1e-5 (per cycle 0.033 / 0.072 /
    # 0.080), learned V(1,1) 2.6e-5: per cycle the network's sweeps beat the plain smoother's, though each
    # costs an MLP evaluation
    assert rel["learned"] < 0.25 * rel["chebyshev"]
    assert rel["learned V(1,1)"] < 2.0 * rel["chebyshev"]


@pytest.mark.parametrize("engine", ["mma", "tcgen05"])
def test_learned_solve_converges_without_fallback(O, dec, trained, engine):
    import scipy.sparse.linalg as spla
    mlp = trained[0]
    mlp.set_engine(engine)
    coarse = O.icosahedron()
    md = O.build_mg(coarse, 4, O.CIRCUMCENTER, 1.0, 1.0, 3)
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1,
                           smoother=3, pre=2, post=2, fallback_rho=0.5)
    mg.set_smoother_mlp(mlp)
    n = mg.n
    B = np.stack([uniform(90 + j, n) for j in range(2)])
    U, rep = mg.solve(torch.zeros((2, n), dtype=torch.float64, device="cuda"), torch.tensor(B, device="cuda"),
                      rtol=1e-10, max_iters=60)
    assert rep.converged == 1 and rep.fallback_iteration == -1
    A = csc(md.op(0)).tocsc()
    U = U.cpu().numpy()
    for j in range(2):
        exact = spla.spsolve(A, B[j])
        assert np.linalg.norm(U[j] - exact) / np.linalg.norm(exact) < 1e-7
    mlp.set_engine("mma")


def test_engine_switch_recaptures_cycles(O, dec, trained):
    """A multigrid object that has captured its cycles with one engine runs the other after
    set_engine: the two cycle results differ only by the engines' FP32 summation order."""
    mlp = trained[0]
    coarse = O.icosahedron()
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1,
                           smoother=3, pre=2, post=2)
    mg.set_smoother_mlp(mlp)
    n = mg.n
    B = torch.tensor(np.stack([uniform(97 + j, n) for j in range(3)]), device="cuda")
    out = {}
    for engine in ("mma", "tcgen05", "mma"):
        mlp.set_engine(engine)
        out.setdefault(engine, []).append(mg.cycles(torch.zeros_like(B), B, 2).cpu().numpy())
    np.testing.assert_array_equal(out["mma"][0], out["mma"][1])
    a, b = out["mma"][0], out["tcgen05"][0]
    assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(a)


def test_diverging_network_falls_back(O, dec):
    coarse = O.icosahedron()
    mg = dec.MultigridData(coarse, 4, shift=1.0, center="circumcenter", project_radius=1.0, precision=1,
                           smoother=3, pre=2, post=2)
    bad = dec.SmootherMLP(4)
    bad.params = jacobi_net(np.float32(3.0))  # over-relaxed Jacobi: amplifies the rough modes
    mg.set_smoother_mlp(bad)
    n = mg.n
    B = torch.tensor(np.stack([uniform(95 + j, n) for j in range(2)]), device="cuda")
    U, rep = mg.solve(torch.zeros_like(B), B, rtol=1e-9, max_iters=80)
    assert rep.fallback_iteration == 1
    assert rep.converged == 1 and rep.max_rel_residual <= 1e-9
    # without a network the learned smoother refuses to run
    mg2 = dec.MultigridData(coarse, 2, shift=1.0, center="circumcenter", project_radius=1.0, smoother=3)
    with pytest.raises(dec.DecError, match="network"):
        mg2.solve(torch.zeros_like(B[:, :mg2.n]).contiguous(), B[:, :mg2.n].contiguous())


def test_checkpoint_round_trip(dec, trained, tmp_path):
    mlp = trained[0]
    path = tmp_path / "smoother.ckpt"
    mlp.save(path)
    other = dec.SmootherMLP(99)
    other.load(path)
    np.testing.assert_array_equal(other.params, mlp.params)
    assert other.step == mlp.step
    raw = bytearray(path.read_bytes())
    raw[100] ^= 0x01
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(bytes(raw))
    with pytest.raises(dec.DecError, match="CRC"):
        other.load(bad)
    with pytest.raises(dec.DecError, match="size"):
        (tmp_path / "short.ckpt").write_bytes(bytes(raw[:50]))
        other.load(tmp_path / "short.ckpt")
