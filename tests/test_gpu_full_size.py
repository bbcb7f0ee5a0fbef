"""Parity at the workloads' full sizes, by the oracle where it finishes in seconds and by properties
that hold at any size.

* Config 4's wedge batch (1,024 FP32 ∧(1,1) pairs on icosphere L7, one batched launch): four pairs
  against the oracle bit for bit, every pair antisymmetric bit for bit (∧(β, α) = -∧(α, β): each
  output is c0 (a2 b1 - a1 b2) + ..., so swapping the forms negates every rounded difference exactly)
  and ∧(α, α) = 0 exactly.
* The learned smoother's L9 mesh (2,621,442 vertices): the FP64 ∧(1,1), ∧(0,1) and the Laplacian
  against the oracle bit for bit, and the Laplacian's FP32 apply linear to within its rounding.
"""
import numpy as np
import pytest

from conftest import uniform

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def ico(O, level):
    m = O.icosahedron()
    for _ in range(level):
        m = O.refine_binary(m, 1.0)
    return m


@pytest.fixture(scope="module")
def l7(O, dec):
    m = ico(O, 7)
    d = O.dualize(m, O.CIRCUMCENTER)
    return m, d, dec.Mesh.from_oracle(m, center="circumcenter")


def test_config4_wedge_batch_l7(O, dec, l7):
    m, d, g = l7
    w = dec.dec_wedge_product(1, 1, g, "float32")
    count = 1024
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)
    a = torch.rand((count, d.ne), dtype=torch.float32, device="cuda", generator=gen) * 2 - 1
    b = torch.rand((count, d.ne), dtype=torch.float32, device="cuda", generator=gen) * 2 - 1
    out = torch.empty((count, d.nt), dtype=torch.float32, device="cuda")
    w.autotune(count, reps=2)
    w.batched(a, b, out)
    swap = torch.empty_like(out)
    w.batched(b, a, swap)
    assert torch.equal(swap, -out)
    self_ = torch.empty_like(out)
    w.batched(a, a, self_)
    assert not torch.any(self_ != 0)
    for j in (0, 1, 511, 1023):
        ref = O.wedge_f32(d, 11, a[j].cpu().numpy(), b[j].cpu().numpy())
        np.testing.assert_array_equal(out[j].cpu().numpy(), ref)


@pytest.fixture(scope="module")
def l9(O, dec):
    m = ico(O, 9)
    d = O.dualize(m, O.CIRCUMCENTER)
    return m, d, dec.Mesh.from_oracle(m, center="circumcenter")


def test_l9_operators_against_oracle(O, dec, l9):
    m, d, g = l9
    assert (d.nv, d.ne, d.nt) == (2621442, 7864320, 5242880)
    f, a, b = uniform(11, d.nv), uniform(12, d.ne), uniform(13, d.ne)
    t = lambda x: torch.tensor(x, device="cuda")
    w11 = dec.dec_wedge_product(1, 1, g)
    np.testing.assert_array_equal(w11(t(a), t(b)).cpu().numpy(), O.wedge(d, 11, a, b))
    w01 = dec.dec_wedge_product(0, 1, g)
    np.testing.assert_array_equal(w01(t(f), t(a)).cpu().numpy(), O.wedge(d, 1, f, a))
    L = dec.laplace_beltrami(g)
    np.testing.assert_array_equal(L.apply(t(f)).cpu().numpy(), O.csc_matvec(O.laplace_beltrami0(d), f))


def test_l9_laplacian_fp32_linear(dec, l9):
    m, d, g = l9
    L = dec.laplace_beltrami(g, "float32")
    x = torch.tensor(uniform(21, d.nv), dtype=torch.float32, device="cuda")
    y = torch.tensor(uniform(22, d.nv), dtype=torch.float32, device="cuda")
    lhs = L.apply(2.0 * x + y).double()
    rhs = 2.0 * L.apply(x).double() + L.apply(y).double()
    scale = lhs.abs().max().item()
    assert (lhs - rhs).abs().max().item() <= 1e-5 * scale
