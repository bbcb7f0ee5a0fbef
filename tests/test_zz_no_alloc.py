"""The allocation-free residual-norm entry point.

`dec_op_residual_norms_noalloc` serves callers that cannot allocate device memory when they call
it (a fixed device-memory budget handed out up front, a real-time loop that must stay out of the
allocator, code that runs while another thread captures a CUDA graph).  Its scratch is a static
device array instead of cudaMalloc.  This test calls it through the C ABI and checks that, on two
calls in a row with different inputs and sizes, it returns the same norms as the allocating entry
point `dec_op_residual_norms` (relative tolerance 1e-12, as the other residual-norm test); that
it does so at the largest size its scratch holds (64 right-hand sides, whose norms sit right after
the last partial sums) and without the optional right-hand-side norms; and that it rejects more
right-hand sides than its scratch holds.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _norms(L, fn, op, X, B, with_bnorms=True):
    nrhs = X.shape[0]
    r = np.empty(nrhs)
    bn = np.empty(nrhs)
    st = getattr(L, fn)(op, C.c_void_p(X.data_ptr()), C.c_void_p(B.data_ptr()), nrhs,
                        r.ctypes.data_as(C.POINTER(C.c_double)),
                        bn.ctypes.data_as(C.POINTER(C.c_double)) if with_bnorms else None,
                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, L.dec_last_error()
    return r, (bn if with_bnorms else None)


def test_noalloc_residual_norms_match_allocating_entry_point(dec):
    L = dec.lib()
    m = dec.meshes.triangulated_grid(40, 40, 1.0, 1.0, False)
    g = dec.Mesh(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation, m.tri_orientation,
                 center="barycenter")
    H = dec.helmholtz(g, 0.5)
    n = g.nv
    for call, nrhs in enumerate((7, 3)):   # two calls in a row; the second is smaller
        X = torch.tensor(np.stack([dec.meshes.uniform(500 + 10 * call + j, n) for j in range(nrhs)]),
                         device="cuda")
        B = torch.tensor(np.stack([dec.meshes.uniform(600 + 10 * call + j, n) for j in range(nrhs)]),
                         device="cuda")
        r0, b0 = _norms(L, "dec_op_residual_norms", H._h, X, B)
        r1, b1 = _norms(L, "dec_op_residual_norms_noalloc", H._h, X, B)
        np.testing.assert_allclose(r1, r0, rtol=1e-12)
        np.testing.assert_allclose(b1, b0, rtol=1e-12)
        assert np.all(r0 > 0)


def test_noalloc_residual_norms_at_the_scratch_limit(dec):
    L = dec.lib()
    m = dec.meshes.triangulated_grid(20, 20, 1.0, 1.0, False)
    g = dec.Mesh(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation, m.tri_orientation,
                 center="barycenter")
    H = dec.helmholtz(g, 0.5)
    n = g.nv
    nrhs = 64
    X = torch.tensor(np.stack([dec.meshes.uniform(800 + j, n) for j in range(nrhs)]), device="cuda")
    B = torch.tensor(np.stack([dec.meshes.uniform(900 + j, n) for j in range(nrhs)]), device="cuda")
    r0, b0 = _norms(L, "dec_op_residual_norms", H._h, X, B)
    r1, b1 = _norms(L, "dec_op_residual_norms_noalloc", H._h, X, B)
    np.testing.assert_allclose(r1, r0, rtol=1e-12)
    np.testing.assert_allclose(b1, b0, rtol=1e-12)
    r2, none = _norms(L, "dec_op_residual_norms_noalloc", H._h, X[:5], B[:5], with_bnorms=False)
    assert none is None
    np.testing.assert_allclose(r2, r0[:5], rtol=1e-12)


def test_noalloc_rejects_too_many_rhs(dec):
    L = dec.lib()
    m = dec.meshes.triangulated_grid(6, 6, 1.0, 1.0, False)
    g = dec.Mesh(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation, m.tri_orientation)
    H = dec.helmholtz(g, 0.5)
    nrhs = 65
    X = torch.zeros((nrhs, g.nv), dtype=torch.float64, device="cuda")
    r = np.empty(nrhs)
    st = L.dec_op_residual_norms_noalloc(H._h, C.c_void_p(X.data_ptr()), C.c_void_p(X.data_ptr()), nrhs,
                                         r.ctypes.data_as(C.POINTER(C.c_double)), None,
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 1
    assert b"static scratch" in L.dec_last_error()
