"""Parity of the sm_100a library (through the C ABI) with the CPU oracle: orientation, dual
geometry, diagonal Hodge stars, d / ∂ / dual d, the Laplace-Beltrami / Helmholtz operator and
the wedge products, on seeded inputs.

Tolerances: integer work (orientation, operator patterns and ±1 values) is bit-exact.  The
geometry, ⋆, d-apply, Laplacian and the ∧01 / ∧11 / pd / dd wedges follow the reference's
operation order and are compared bit-exactly in FP64 and FP32.  ∧02 folds the two dual-triangle
coefficients at each vertex into one, so it is compared at 4 ulp-scale relative error (1e-14 FP64,
1e-6 FP32).
"""
import math

import numpy as np
import pytest

from conftest import csc, uniform

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def meshes(O):
    ico = O.icosahedron()
    for _ in range(3):
        ico = O.refine_binary(ico, 1.0)   # orientation left unset: the library runs orient!
    return {
        "grid128_bary": (O.triangulated_grid(127, 127, 1.0, 1.0, False), O.BARYCENTER),
        "grid_compressed_circum": (O.triangulated_grid(10, 7, 1.3, 0.9, True), O.CIRCUMCENTER),
        "ico3_circum": (ico, O.CIRCUMCENTER),
        "grid_345_bary": (O.grid_345(), O.BARYCENTER),
        "tri_345_false_bary": (O.tri_345(False), O.BARYCENTER),
    }


@pytest.fixture(scope="module")
def cases(O, dec):
    out = {}
    for name, (m, center) in meshes(O).items():
        d = O.dualize(m, center)
        g = dec.Mesh.from_oracle(m, center="barycenter" if center == O.BARYCENTER else "circumcenter")
        out[name] = (m, d, g)
    return out


NAMES = ["grid128_bary", "grid_compressed_circum", "ico3_circum", "grid_345_bary", "tri_345_false_bary"]


def cuda(a, dt=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


@pytest.mark.parametrize("name", NAMES)
def test_orientation_bit_exact(cases, name):
    m, d, g = cases[name]
    eo, to = g.orientation()
    np.testing.assert_array_equal(eo, d.mesh.edge_orientation)
    np.testing.assert_array_equal(to, d.mesh.tri_orientation)


@pytest.mark.parametrize("name", NAMES)
def test_geometry_bit_exact(cases, name):
    m, d, g = cases[name]
    np.testing.assert_array_equal(g.geometry("length"), d.length)
    np.testing.assert_array_equal(g.geometry("area"), d.area)
    np.testing.assert_array_equal(g.geometry("dual_area"), d.dual_area)
    np.testing.assert_array_equal(g.geometry("dual_point"), d.dual_point)
    # triangle-center -> edge-center dual edges are the D_edges12 block of the dual edges
    ne, nt = d.ne, d.nt
    np.testing.assert_array_equal(g.geometry("dual_length_te"), d.dual_length[2 * ne:2 * ne + 3 * nt])


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("k", [0, 1, 2])
def test_hodge_bit_exact(O, dec, cases, name, k):
    m, d, g = cases[name]
    np.testing.assert_array_equal(dec.dec_hodge_star(k, g).cpu().numpy(), O.hodge_diag(d, k))
    with np.errstate(divide="ignore"):
        ref_inv = O.inv_hodge_diag(d, k)
    np.testing.assert_array_equal(dec.dec_inv_hodge_star(k, g).cpu().numpy(), ref_inv)
    np.testing.assert_array_equal(dec.dec_hodge_star(k, g, dtype="float32").cpu().numpy(),
                                  O.hodge_diag(d, k).astype(np.float32))


OPS = [("d0", "dec_differential", 0), ("d1", "dec_differential", 1), ("b1", "dec_boundary", 1),
       ("b2", "dec_boundary", 2), ("dd0", "dec_dual_derivative", 0), ("dd1", "dec_dual_derivative", 1)]


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("op", OPS, ids=[o[0] for o in OPS])
def test_exterior_derivative_patterns_exact(O, dec, cases, name, op):
    m, d, g = cases[name]
    _, fn, n = op
    ref = csc(getattr(O, fn)(d, n)).tocsr()
    ref.sort_indices()
    rp, ci, v, shape = getattr(dec, fn)(n, g).csr()
    assert shape == ref.shape
    np.testing.assert_array_equal(rp, ref.indptr)
    np.testing.assert_array_equal(ci, ref.indices)
    np.testing.assert_array_equal(v, ref.data)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("op", OPS, ids=[o[0] for o in OPS])
@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_exterior_derivative_apply(O, dec, cases, name, op, dt):
    m, d, g = cases[name]
    _, fn, n = op
    t = getattr(O, fn)(d, n)
    A = getattr(dec, fn)(n, g, dtype=dt)
    x = uniform(7 + n, A.shape[1])
    if dt == "float64":
        y = A(cuda(x)).cpu().numpy()
        np.testing.assert_array_equal(y, O.csc_matvec(t, x))
    else:
        x32 = x.astype(np.float32)
        y = A(cuda(x32, torch.float32)).cpu().numpy()
        # ±1 coefficients: an FP32 sum in the same order as the FP64 one, rounded per step
        ref = (csc(t).astype(np.float32) @ x32.astype(np.float32))
        np.testing.assert_allclose(y, ref, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("name", NAMES)
def test_laplacian_bit_exact(O, dec, cases, name):
    m, d, g = cases[name]
    with np.errstate(divide="ignore", invalid="ignore"):
        t = O.laplace_beltrami0(d)
    ref = csc(t).tocsr()
    ref.sort_indices()
    L = dec.laplace_beltrami(g)
    rp, ci, v, shape = L.csr()
    np.testing.assert_array_equal(rp, ref.indptr)
    np.testing.assert_array_equal(ci, ref.indices)
    np.testing.assert_array_equal(v, ref.data)
    x = uniform(11, d.nv)
    if np.all(np.isfinite(ref.data)):
        np.testing.assert_array_equal(L(cuda(x)).cpu().numpy(), O.csc_matvec(t, x))


def test_helmholtz_shift_and_alpha_beta(O, dec, cases):
    m, d, g = cases["ico3_circum"]
    c = 0.37
    H = dec.helmholtz(g, c)
    L = csc(O.laplace_beltrami0(d))
    x, y0 = uniform(3, d.nv), uniform(4, d.nv)
    ref = 2.0 * ((L @ x) + c * x) - 0.5 * y0
    y = cuda(y0)
    H.apply(cuda(x), y, alpha=2.0, beta=-0.5)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_wedges(O, dec, cases, name, dt):
    m, d, g = cases[name]
    npdt = np.float64 if dt == "float64" else np.float32
    tdt = torch.float64 if dt == "float64" else torch.float32
    ref_fn = O.wedge if dt == "float64" else O.wedge_f32
    f = uniform(0, d.nv).astype(npdt)
    a = uniform(1, d.ne).astype(npdt)
    b = uniform(2, d.ne).astype(npdt)
    tt = uniform(3, d.nt).astype(npdt)
    # ∧(0,1) and ∧(1,0)
    w01 = dec.dec_wedge_product(0, 1, g, dt)
    np.testing.assert_array_equal(w01(cuda(f, tdt), cuda(a, tdt)).cpu().numpy(), ref_fn(d, 1, f, a))
    w10 = dec.dec_wedge_product(1, 0, g, dt)
    np.testing.assert_array_equal(w10(cuda(a, tdt), cuda(f, tdt)).cpu().numpy(), ref_fn(d, 1, f, a))
    # ∧(1,1)
    w11 = dec.dec_wedge_product(1, 1, g, dt)
    np.testing.assert_array_equal(w11(cuda(a, tdt), cuda(b, tdt)).cpu().numpy(), ref_fn(d, 11, a, b))
    # ∧(0,2) and ∧(2,0)
    tol = 1e-14 if dt == "float64" else 2e-6
    ref02 = ref_fn(d, 2, f, tt)
    w02 = dec.dec_wedge_product(0, 2, g, dt)
    out = w02(cuda(f, tdt), cuda(tt, tdt)).cpu().numpy()
    np.testing.assert_allclose(out, ref02, rtol=tol, atol=tol * np.abs(ref02).max())
    w20 = dec.dec_wedge_product(2, 0, g, dt)
    out = w20(cuda(tt, tdt), cuda(f, tdt)).cpu().numpy()
    np.testing.assert_allclose(out, ref02, rtol=tol, atol=tol * np.abs(ref02).max())


@pytest.mark.parametrize("name", NAMES)
def test_wedge_identities_on_device(O, dec, cases, name):
    """∧(1, β) = β (FastDEC.jl wdg01(1,1) == 1 in test/Backends.jl:152) and dx∧dy = area on planar meshes."""
    m, d, g = cases[name]
    one_v = cuda(np.ones(d.nv))
    one_e = cuda(np.ones(d.ne))
    np.testing.assert_array_equal(dec.dec_wedge_product(0, 1, g)(one_v, one_e).cpu().numpy(), np.ones(d.ne))
    if np.all(d.mesh.points[:, 2] == 0):
        p = d.mesh.points
        sg = np.where(d.mesh.edge_orientation == 1, 1.0, -1.0)
        dx = ((p[d.mesh.ev0] - p[d.mesh.ev1]) @ np.array([1.0, 0, 0])) * sg
        dy = ((p[d.mesh.ev0] - p[d.mesh.ev1]) @ np.array([0, 1.0, 0])) * sg
        w = dec.dec_wedge_product(1, 1, g)(cuda(dx), cuda(dy)).cpu().numpy()
        # the sign of dx∧dy follows each triangle's orientation relative to the plane
        np.testing.assert_allclose(np.abs(w), d.area, rtol=1e-12)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_pd_dd_wedges(O, dec, cases, name, dt):
    m, d, g = cases[name]
    npdt = np.float64 if dt == "float64" else np.float32
    tdt = torch.float64 if dt == "float64" else torch.float32
    Mpd = csc(O.wedge_pd_01_mat(d)).astype(npdt)
    Mdd = csc(O.wedge_dd_01_mat(d)).astype(npdt)
    gv = uniform(21, d.nv).astype(npdt)     # primal 0-form
    fe = uniform(22, d.ne).astype(npdt)     # dual 1-form
    ft = uniform(23, d.nt).astype(npdt)     # dual 0-form
    tol = 0 if dt == "float64" else 1e-6
    pd = dec.dec_wedge_product_pd(0, 1, g, dt)(cuda(gv, tdt), cuda(fe, tdt)).cpu().numpy()
    np.testing.assert_allclose(pd, (Mpd @ gv) * fe, rtol=tol, atol=tol)
    dp = dec.dec_wedge_product_dp(1, 0, g, dt)(cuda(fe, tdt), cuda(gv, tdt)).cpu().numpy()
    np.testing.assert_allclose(dp, fe * (Mpd @ gv), rtol=tol, atol=tol)
    dd01 = dec.dec_wedge_product_dd(0, 1, g, dt)(cuda(ft, tdt), cuda(fe, tdt)).cpu().numpy()
    np.testing.assert_allclose(dd01, (Mdd @ ft) * fe, rtol=tol, atol=tol)
    dd10 = dec.dec_wedge_product_dd(1, 0, g, dt)(cuda(fe, tdt), cuda(ft, tdt)).cpu().numpy()
    np.testing.assert_allclose(dd10, fe * (Mdd @ ft), rtol=tol, atol=tol)



@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_pd_dp_11_wedges(O, dec, cases, name, dt):
    """pd(1,1)(f, g) = ∧11(f, ♭♯ g) and dp(1,1)(f, g) = ∧11(♭♯ f, g) (FastDEC.jl:391-401) with
    ♭♯ = ♭(DPP) ♯(LLS) built on the GPU: bit-exact with the oracle in FP64."""
    m, d, g = cases[name]
    fs = O.flat_sharp_mat(d)
    npdt = np.float64 if dt == "float64" else np.float32
    tdt = torch.float64 if dt == "float64" else torch.float32
    f = uniform(21, d.ne)
    h = uniform(22, d.ne)
    ref_pd = O.wedge(d, 11, f, O.csc_matvec(fs, h))
    ref_dp = O.wedge(d, 11, O.csc_matvec(fs, f), h)
    pd = dec.dec_wedge_product_pd(1, 1, g, dt)(cuda(f.astype(npdt), tdt), cuda(h.astype(npdt), tdt)).cpu().numpy()
    dp = dec.dec_wedge_product_dp(1, 1, g, dt)(cuda(f.astype(npdt), tdt), cuda(h.astype(npdt), tdt)).cpu().numpy()
    if dt == "float64":
        np.testing.assert_array_equal(pd, ref_pd)
        np.testing.assert_array_equal(dp, ref_dp)
    else:
        for got, ref in ((pd, ref_pd), (dp, ref_dp)):
            np.testing.assert_allclose(got, ref, rtol=0, atol=2e-5 * max(1.0, np.abs(ref).max()))


def test_unsupported_degrees_raise(dec, cases):
    m, d, g = cases["grid_345_bary"]
    with pytest.raises(dec.DecError, match="Unsupported combination"):
        dec.dec_wedge_product(2, 1, g)
    with pytest.raises(dec.DecError):
        dec.dec_wedge_product_dd(1, 1, g)


def test_one_based_description_matches(O, dec, cases):
    """A Julia caller passes 1-based arrays (index_base = 1)."""
    m, d, g = cases["grid_345_bary"]
    g1 = dec.Mesh(m.points, m.ev0 + 1, m.ev1 + 1, m.te0 + 1, m.te1 + 1, m.te2 + 1, m.edge_orientation,
                  m.tri_orientation, center="barycenter", index_base=1)
    np.testing.assert_array_equal(g1.geometry("dual_area"), g.geometry("dual_area"))


@pytest.mark.parametrize("name", ["grid128_bary", "ico3_circum"])
def test_residual_norms(O, dec, cases, name):
    """‖b_j - A x_j‖ and ‖b_j‖ per right-hand side (the norm(L*u - b) / norm(b) test of
    test/Multigrid.jl:67), against numpy on the oracle's operator."""
    m, d, g = cases[name]
    H = dec.helmholtz(g, 0.75)
    A = csc(O.laplace_beltrami0(d)) + 0.75 * __import__("scipy.sparse", fromlist=["eye"]).eye(d.nv)
    nrhs = 5
    X = np.stack([uniform(40 + j, d.nv) for j in range(nrhs)])
    B = np.stack([uniform(60 + j, d.nv) for j in range(nrhs)])
    r, bn = H.residual_norms(cuda(X), cuda(B))
    ref_r = np.array([np.linalg.norm(B[j] - A @ X[j]) for j in range(nrhs)])
    ref_b = np.linalg.norm(B, axis=1)
    np.testing.assert_allclose(r, ref_r, rtol=1e-12)
    np.testing.assert_allclose(bn, ref_b, rtol=1e-13)
    with pytest.raises(dec.DecError, match="Laplacian, a Helmholtz operator or a square matrix"):
        dec.dec_differential(0, g).residual_norms(cuda(X), cuda(B))   # rejected before any device work


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("op", OPS, ids=[o[0] for o in OPS])
@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_unaligned_output_matches(dec, cases, name, op, dt):
    """Outputs that are not 16-byte aligned take the one-row-per-thread kernels; the result is the
    same bit for bit as the vectorised four-rows-per-thread path (and alpha/beta are honoured)."""
    m, d, g = cases[name]
    _, fn, n = op
    A = getattr(dec, fn)(n, g, dtype=dt)
    tdt = torch.float64 if dt == "float64" else torch.float32
    x = cuda(uniform(17 + n, A.shape[1]).astype(np.float64 if dt == "float64" else np.float32), tdt)
    rows = A.shape[0]
    buf = torch.zeros(rows + 1, dtype=tdt, device="cuda")
    ya = A(x)
    yu = A.apply(x, buf[1:])
    np.testing.assert_array_equal(yu.cpu().numpy(), ya.cpu().numpy())
    y0 = cuda(uniform(19, rows).astype(np.float64 if dt == "float64" else np.float32), tdt)
    za = y0.clone()
    A.apply(x, za, alpha=0.5, beta=2.0)
    buf[1:] = y0
    A.apply(x, buf[1:], alpha=0.5, beta=2.0)
    np.testing.assert_array_equal(buf[1:].cpu().numpy(), za.cpu().numpy())


@pytest.mark.parametrize("name", NAMES)
def test_geometric_hodge(O, dec, cases, name):
    """dec_hodge_star(1, sd, GeometricHodge()) (FastDEC.jl:660-716): the sparse ⋆1 built on the GPU
    is bit-exact with the oracle's statement, its apply too; the inverse (-⋆1)⁻¹ (a Krylov solve,
    as the reference's CUDA backend does, ext/CombinatorialSpacesCUDAExt.jl:93-96) agrees with a
    direct sparse solve to 1e-10 (test/Backends.jl:118-129 compares at atol 1e-10)."""
    import scipy.sparse.linalg as spla
    m, d, g = cases[name]
    ref = csc(O.hodge_geometric1_fast(d)).tocsr()
    ref.sort_indices()
    G = dec.hodge_operator(1, g, hodge="geometric")
    rp, ci, v, shape = G.csr()
    np.testing.assert_array_equal(rp, ref.indptr)
    np.testing.assert_array_equal(ci, ref.indices)
    np.testing.assert_array_equal(v, ref.data)
    x = uniform(31, d.ne)
    np.testing.assert_array_equal(G(cuda(x)).cpu().numpy(), O.csc_matvec(O.hodge_geometric1_fast(d), x))
    Gi = dec.hodge_operator(1, g, inverse=True, hodge="geometric")
    y = Gi(cuda(x)).cpu().numpy()
    exact = spla.spsolve((-ref).tocsc(), x)
    np.testing.assert_allclose(y, exact, rtol=0, atol=1e-10 * max(1.0, np.abs(exact).max()))
    y32 = dec.hodge_operator(1, g, inverse=True, hodge="geometric", dtype="float32")(
        cuda(x.astype(np.float32), torch.float32)).cpu().numpy()
    np.testing.assert_allclose(y32, exact, rtol=0, atol=1e-5 * max(1.0, np.abs(exact).max()))
