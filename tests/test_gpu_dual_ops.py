"""Dual-dual operators of a 2D complex on the GPU (FastDEC.jl:762-853) against the same
compositions of the oracle's operators, ♭♯ as a stand-alone operator, and dec_Δ⁻¹
(FastDEC.jl:866-869) against the oracle's full multigrid.

Oracle side: ♭♯_mat, wedge_pd_01_mat, the FastDEC geometric ⋆1, the diagonal stars, d, dual d and
∧11 from the oracle, applied with its CSC product (the reference's column order); the inverse
geometric ⋆1 is a direct sparse solve of -⋆1 (the reference's `factorize`).  Tolerances:
compositions without the inverse geometric ⋆1 agree to 1e-13 relative (♭♯ alone bit for bit);
with it, the GPU's Krylov solve against the direct one gives 1e-9.
"""
import numpy as np
import pytest

from conftest import csc, uniform
from test_gpu_parity_ops import cuda, meshes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

NAMES = ["grid_compressed_circum", "ico3_circum", "grid_345_bary", "grid128_bary"]


@pytest.fixture(scope="module")
def cases(O, dec):
    out = {}
    for name, (m, center) in meshes(O).items():
        if name not in NAMES:
            continue
        d = O.dualize(m, center)
        g = dec.Mesh.from_oracle(m, center="barycenter" if center == O.BARYCENTER else "circumcenter")
        out[name] = (d, g)
    return out


class Ref:
    """The reference's compositions over the oracle's operators (FastDEC.jl:762-853)."""

    def __init__(self, O, d):
        import scipy.sparse.linalg as spla
        self.O, self.d = O, d
        self.mv = O.csc_matvec
        self.star2 = O.hodge_diag(d, 2)
        self.istar0 = O.inv_hodge_diag(d, 0)
        self.G1 = O.hodge_geometric1_fast(d)
        self.lu = spla.splu((-csc(self.G1)).tocsc())
        self.FS = O.flat_sharp_mat(d)
        self.M01 = O.wedge_pd_01_mat(d)
        self.DD0, self.DD1 = O.dec_dual_derivative(d, 0), O.dec_dual_derivative(d, 1)
        self.D0, self.D1 = O.dec_differential(d, 0), O.dec_differential(d, 1)

    def ihs1(self, x):
        return self.lu.solve(x)

    def i1(self, f, g):  # ⋆2 ∧pd11(⋆1⁻¹ g, f), ∧pd11(a, b) = ∧11(a, ♭♯ b)
        return self.star2 * self.O.wedge(self.d, 11, self.ihs1(g), self.mv(self.FS, f))

    def i2(self, f, g):  # ⋆1 ♭♯ ((Λpd01 ⋆0⁻¹ g) .* f)
        return self.mv(self.G1, self.mv(self.FS, self.mv(self.M01, self.istar0 * g) * f))

    def lie(self, f, g):
        return -self.mv(self.DD0, self.i1(f, g)) - self.i2(f, self.mv(self.DD1, g))

    def lap0(self, x):
        return self.star2 * self.mv(self.D1, self.ihs1(self.mv(self.DD0, x)))

    def lap1(self, x):
        a = self.mv(self.G1, self.mv(self.D0, self.istar0 * self.mv(self.DD1, x)))
        return a + self.mv(self.DD0, self.star2 * self.mv(self.D1, self.ihs1(x)))


def close(got, ref, tol):
    np.testing.assert_allclose(got, ref, rtol=0, atol=tol * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("name", NAMES)
def test_flat_sharp_operator(O, dec, cases, name):
    """♭♯_mat(sd) (DiscreteExteriorCalculus.jl:1992) as an operator: the matrix inside the
    pd/dp(1,1) wedges, bit for bit, and its apply in FP64."""
    d, g = cases[name]
    ref = csc(O.flat_sharp_mat(d)).tocsr()
    ref.sort_indices()
    rp, ci, v, shape = dec.flat_sharp(g).csr()
    assert shape == (d.ne, d.ne)
    np.testing.assert_array_equal(rp, ref.indptr)
    np.testing.assert_array_equal(ci, ref.indices)
    np.testing.assert_array_equal(v, ref.data)
    x = uniform(51, d.ne)
    np.testing.assert_array_equal(dec.flat_sharp(g)(cuda(x)).cpu().numpy(), O.csc_matvec(O.flat_sharp_mat(d), x))


@pytest.mark.parametrize("name", NAMES)
def test_interior_products(O, dec, cases, name):
    d, g = cases[name]
    R = Ref(O, d)
    f, h1, h2 = uniform(52, d.ne), uniform(53, d.ne), uniform(54, d.nv)
    i1 = dec.interior_product_dd(1, 1, g)(cuda(f), cuda(h1)).cpu().numpy()
    assert i1.shape == (d.nt,)
    close(i1, R.i1(f, h1), 1e-9)
    i2 = dec.interior_product_dd(1, 2, g)(cuda(f), cuda(h2)).cpu().numpy()
    assert i2.shape == (d.ne,)
    close(i2, R.i2(f, h2), 1e-13)
    with pytest.raises(ValueError):
        dec.interior_product_dd(2, 1, g)


@pytest.mark.parametrize("name", NAMES)
def test_lie_derivative(O, dec, cases, name):
    d, g = cases[name]
    R = Ref(O, d)
    f, h = uniform(55, d.ne), uniform(56, d.ne)
    got = dec.ℒ_dd(1, 1, g)(cuda(f), cuda(h)).cpu().numpy()
    close(got, R.lie(f, h), 1e-9)


@pytest.mark.parametrize("name", NAMES)
def test_dual_laplacians(O, dec, cases, name):
    d, g = cases[name]
    R = Ref(O, d)
    x0, x1 = uniform(57, d.nt), uniform(58, d.ne)
    close(dec.Δᵈ(0, g)(cuda(x0)).cpu().numpy(), R.lap0(x0), 1e-9)
    close(dec.Δᵈ(1, g)(cuda(x1)).cpu().numpy(), R.lap1(x1), 1e-9)


def test_inverse_laplacian(O, dec):
    """dec_Δ⁻¹(Val(0), s) = full_multigrid(b, md, 5, cg, μ=2) with 3 CG steps on the Laplacian
    hierarchy, against the oracle's full multigrid on the reference's test grid
    (test/Multigrid.jl:54-90), compared modulo the Laplacian's constant null space; it also meets
    the reference's FMG-W threshold (< 1e-7)."""
    s = O.triangulated_grid(1, 1, 1 / 4, np.sqrt(3) / 8, False)
    md = O.build_mg(s, 4, O.CIRCUMCENTER, 0.0, 0.0, 3)
    L = csc(md.op(0))
    n = L.shape[0]
    b = L @ ((uniform(0, n) + 1) / 2)
    inv = dec.dec_inverse_laplacian(0, s, 4)
    u = inv(cuda(b)).cpu().numpy()
    ref = O.full_multigrid(md, b, 5, 2)
    du, dr = u - u.mean(), ref - ref.mean()
    assert np.linalg.norm(du - dr) <= 1e-8 * np.linalg.norm(dr)
    assert np.linalg.norm(L @ u - b) / np.linalg.norm(b) < 1e-7
    assert inv.md.options.mu == 2 and inv.md.options.smoother == 2
    with pytest.raises(ValueError):
        dec.dec_inverse_laplacian(1, s, 4)
