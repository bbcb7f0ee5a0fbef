"""dec_b200: the CombinatorialSpaces.jl DEC hot path on B200 (sm_100a).

A Python mirror of the reference's backend entry points for this path, each calling the C ABI
of ``libdec_b200.so`` (include/dec_b200.h):

    dec_wedge_product(m, n, sd, dtype)          FastDEC.jl:255-289 (closure (a, b) -> a ∧ b)
    dec_wedge_product_pd / _dp / _dd            FastDEC.jl:291-401
    dec_differential / dec_boundary /
      dec_dual_derivative(n, sd, dtype)         ext/CombinatorialSpacesCUDAExt.jl:30-61
    dec_hodge_star / dec_inv_hodge_star         ext/CombinatorialSpacesCUDAExt.jl:70-96
    laplace_beltrami(sd) / helmholtz(sd, c)     test/Multigrid.jl:46-48
    MultigridData(s, levels, ...)               Multigrid.jl:698-797
    multigrid_vcycles / multigrid_wcycles       Multigrid.jl:814-824

Forms are torch CUDA tensors in the reference's element order; work runs on torch's current
stream.  There is no CPU fallback: every call goes to the CUDA library and raises if it is
missing or fails.
"""
import ctypes as C

import numpy as np

from . import _capi
from . import meshes  # noqa: F401
from . import mesh_io  # noqa: F401
from ._capi import check, lib, DecError  # noqa: F401

__all__ = ["Mesh", "Operator", "MultigridData", "dec_wedge_product", "dec_wedge_product_pd",
           "dec_wedge_product_dp", "dec_wedge_product_dd", "dec_differential", "dec_boundary",
           "dec_dual_derivative", "dec_hodge_star", "dec_inv_hodge_star", "laplace_beltrami",
           "helmholtz", "multigrid_vcycles", "multigrid_wcycles", "full_multigrid", "SmootherMLP", "Batch",
           "DecError"]

CENTERS = {"barycenter": _capi.DEC_BARYCENTER, "circumcenter": _capi.DEC_CIRCUMCENTER}


def _torch():
    import torch
    return torch


def _dtype_code(dtype):
    torch = _torch()
    if dtype in (torch.float64, np.float64, "f64", "float64"):
        return _capi.DEC_F64
    if dtype in (torch.float32, np.float32, "f32", "float32"):
        return _capi.DEC_F32
    raise ValueError(f"unsupported dtype {dtype}")


def _torch_dtype(code):
    torch = _torch()
    return torch.float64 if code == _capi.DEC_F64 else torch.float32


def _stream():
    torch = _torch()
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _check_form(t, n, code, what):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{what}: expected a CUDA tensor")
    if t.dtype != _torch_dtype(code):
        raise TypeError(f"{what}: expected {_torch_dtype(code)}, got {t.dtype}")
    if t.numel() != n or not t.is_contiguous():
        raise ValueError(f"{what}: expected a contiguous form of length {n}, got shape {tuple(t.shape)}")


class Mesh:
    """An embedded 2D delta set with its dual complex, resident on the GPU.

    Arguments are host arrays: ``points`` (nv, 3), edge faces ``ev0`` (∂v0, target) and
    ``ev1`` (∂v1, source), triangle faces ``te0, te1, te2`` (∂e0, ∂e1, ∂e2), the orientations
    (None = unset, as after ``topo_to_mesh``) and the dual-subdivision ``center``.
    """

    def __init__(self, points, ev0, ev1, te0, te1, te2, edge_orientation=None, tri_orientation=None,
                 center="barycenter", index_base=0):
        self._keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a.ctypes.data_as(C.c_void_p)

        pts = np.ascontiguousarray(points, dtype=np.float64)
        if pts.ndim == 2 and pts.shape[1] == 2:
            pts = np.concatenate([pts, np.zeros((pts.shape[0], 1))], axis=1)
        d = _capi.MeshDesc()
        d.nv, d.ne, d.nt = pts.shape[0], len(ev0), len(te0)
        d.index_base = index_base
        d.points = arr(pts, np.float64)
        d.e_v0, d.e_v1 = arr(ev0, np.int32), arr(ev1, np.int32)
        d.t_e0, d.t_e1, d.t_e2 = arr(te0, np.int32), arr(te1, np.int32), arr(te2, np.int32)
        d.edge_orientation = None if edge_orientation is None else arr(edge_orientation, np.int8)
        d.tri_orientation = None if tri_orientation is None else arr(tri_orientation, np.int8)
        d.center = CENTERS[center] if isinstance(center, str) else int(center)
        self.desc = d
        h = C.c_void_p()
        check(lib().dec_mesh_create(C.byref(d), C.byref(h)))
        self._h = h
        self._owned = True
        self.nv, self.ne, self.nt = int(d.nv), int(d.ne), int(d.nt)
        self._keep = []  # host arrays were copied by the library
        self.desc = None

    @classmethod
    def _borrow(cls, handle):
        self = cls.__new__(cls)
        self._h = handle
        self._owned = False
        nv, ne, nt = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().dec_mesh_counts(handle, C.byref(nv), C.byref(ne), C.byref(nt)))
        self.nv, self.ne, self.nt = nv.value, ne.value, nt.value
        return self

    @classmethod
    def from_oracle(cls, m, center="barycenter"):
        """Build from an object with the oracle Mesh attributes (0-based arrays)."""
        return cls(m.points, m.ev0, m.ev1, m.te0, m.te1, m.te2, m.edge_orientation,
                   m.tri_orientation, center=center, index_base=0)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_owned", False) and _capi is not None and _capi._lib is not None:
            _capi._lib.dec_mesh_destroy(h)
            self._h = None

    def orientation(self):
        eo = np.empty(self.ne, np.int8)
        to = np.empty(self.nt, np.int8)
        check(lib().dec_mesh_orientation(self._h, eo.ctypes.data_as(C.c_void_p), to.ctypes.data_as(C.c_void_p)))
        return eo, to

    def geometry(self, which):
        n = {"length": self.ne, "area": self.nt, "dual_area": 6 * self.nt, "dual_length_te": 3 * self.nt,
             "dual_point": 3 * (self.nv + self.ne + self.nt)}[which]
        code = {"length": 0, "area": 1, "dual_area": 2, "dual_length_te": 3, "dual_point": 4}[which]
        out = np.empty(n, np.float64)
        check(lib().dec_mesh_geometry(self._h, code, out.ctypes.data_as(C.c_void_p), n))
        return out.reshape(-1, 3) if which == "dual_point" else out


# ---- wedge products -------------------------------------------------------------------------

class WedgePlan:
    """Cached wedge coefficients on the device; calling it evaluates a ∧ b (allocating the output,
    as dec_c_wedge_product does, or into ``out``)."""

    def __init__(self, sd, kind, m, n, dtype):
        self.sd = sd
        self.code = _dtype_code(dtype)
        h = C.c_void_p()
        check(lib().dec_wedge_plan_create(sd._h, kind, m, n, self.code, C.byref(h)))
        self._h = h
        la, lb, lo = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().dec_wedge_lengths(h, C.byref(la), C.byref(lb), C.byref(lo)))
        self.len_a, self.len_b, self.len_out = la.value, lb.value, lo.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _capi is not None and _capi._lib is not None:
            _capi._lib.dec_wedge_plan_destroy(h)
            self._h = None

    def __call__(self, a, b, out=None):
        torch = _torch()
        _check_form(a, self.len_a, self.code, "wedge first form")
        _check_form(b, self.len_b, self.code, "wedge second form")
        if out is None:
            out = torch.empty(self.len_out, dtype=_torch_dtype(self.code), device=a.device)
        _check_form(out, self.len_out, self.code, "wedge output")
        check(lib().dec_wedge_apply(self._h, _ptr(a), _ptr(b), _ptr(out), _stream()))
        return out

    def batched(self, a, b, out):
        """out[j] = a[j] ∧ b[j] for j < count, one launch (a, b, out: (count, len) CUDA tensors)."""
        count = a.shape[0]
        for t, ln, what in ((a, self.len_a, "first forms"), (b, self.len_b, "second forms"),
                            (out, self.len_out, "outputs")):
            if tuple(t.shape) != (count, ln):
                raise ValueError(f"wedge batch {what}: expected shape {(count, ln)}, got {tuple(t.shape)}")
            _check_form(t, count * ln, self.code, f"wedge batch {what}")
        check(lib().dec_wedge_apply_batched(self._h, _ptr(a), _ptr(b), _ptr(out), count, _stream()))
        return out

    def autotune(self, count, reps=5):
        """Time the batched FP32 ∧(1,1)'s pairs-per-thread variants on min(count, 256) pairs and record
        the fastest in the tuning table (dec_wedge_autotune); returns the choice (0: nothing tuned)."""
        c = C.c_int32()
        check(lib().dec_wedge_autotune(self._h, count, reps, _stream(), C.byref(c)))
        return c.value


def dec_wedge_product(m, n, sd, dtype="float64"):
    """Primal-primal wedge of an m-form and an n-form (FastDEC.jl:255-289)."""
    return WedgePlan(sd, _capi.DEC_WEDGE_PP, m, n, dtype)


def dec_wedge_product_pd(m, n, sd, dtype="float64"):
    """Primal m-form ∧ dual n-form (FastDEC.jl:386-395)."""
    return WedgePlan(sd, _capi.DEC_WEDGE_PD, m, n, dtype)


def dec_wedge_product_dp(m, n, sd, dtype="float64"):
    """Dual m-form ∧ primal n-form (FastDEC.jl:381-384, :397-401)."""
    return WedgePlan(sd, _capi.DEC_WEDGE_DP, m, n, dtype)


def dec_wedge_product_dd(m, n, sd, dtype="float64"):
    """Dual m-form ∧ dual n-form (FastDEC.jl:317-325)."""
    return WedgePlan(sd, _capi.DEC_WEDGE_DD, m, n, dtype)


def dec_c_wedge_product(j, k, a, b, p, c, n_out, out=None, index_base=0):
    """dec_c_wedge_product!(Val(j), Val(k), res, α, β, p, c) (FastDEC.jl:217-232): the wedge kernel
    on caller caches (the reference's cache_wedge matrices; p an int32 CUDA tensor, c a CUDA tensor
    of the forms' dtype or None for (0,1)), for (0,1), (0,2), (0,3), (1,1) and (2,1).  p, c are
    passed in Julia's column-major order: a (R, n_out) torch tensor's transpose-contiguous layout,
    i.e. shape (n_out, R) row-major (for (0,1): shape (2, n_out))."""
    torch = _torch()
    code = _dtype_code(a.dtype)
    if out is None:
        out = torch.empty(n_out, dtype=a.dtype, device=a.device)
    for t, what in ((a, "α"), (b, "β"), (out, "result")):
        if t.dtype != a.dtype or not t.is_contiguous():
            raise ValueError(f"c_wedge: {what} must be contiguous {a.dtype}")
    if p.dtype != torch.int32 or not p.is_contiguous():
        raise ValueError("c_wedge: p must be a contiguous int32 tensor")
    if c is not None and (c.dtype != a.dtype or not c.is_contiguous()):
        raise ValueError("c_wedge: c must be a contiguous tensor of the forms' dtype")
    check(lib().dec_c_wedge_apply(j, k, n_out, _ptr(p), _ptr(c) if c is not None else None, code, _ptr(a),
                                  _ptr(b), _ptr(out), index_base, _stream()))
    return out


# ---- operators ------------------------------------------------------------------------------

class Operator:
    """A sparse DEC operator on the device: ``op(x)`` / ``op @ x`` returns Op x."""

    def __init__(self, sd, kind, dtype="float64", shift=0.0, handle=None, owned=False, code=None):
        self.sd = sd
        if handle is not None:
            self._h, self._owned = handle, owned
            self.code = _capi.DEC_F64 if code is None else code
        else:
            self.code = _dtype_code(dtype)
            h = C.c_void_p()
            check(lib().dec_op_create(sd._h, kind, float(shift), self.code, C.byref(h)))
            self._h, self._owned = h, True
        r, c = C.c_int64(), C.c_int64()
        check(lib().dec_op_shape(self._h, C.byref(r), C.byref(c)))
        self.shape = (r.value, c.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_owned", False) and _capi is not None and _capi._lib is not None:
            _capi._lib.dec_op_destroy(h)
            self._h = None

    def apply(self, x, y=None, alpha=1.0, beta=0.0):
        torch = _torch()
        _check_form(x, self.shape[1], self.code, "operator input")
        if y is None:
            y = torch.empty(self.shape[0], dtype=_torch_dtype(self.code), device=x.device)
        _check_form(y, self.shape[0], self.code, "operator output")
        check(lib().dec_op_apply(self._h, _ptr(x), _ptr(y), float(alpha), float(beta), _stream()))
        return y

    __call__ = apply

    def __matmul__(self, x):
        return self.apply(x)

    def residual_norms(self, x, b):
        """(‖b_j - Op x_j‖, ‖b_j‖) per right-hand side; x, b float64 CUDA tensors (n,) or (nrhs, n)."""
        nrhs = 1 if b.dim() == 1 else b.shape[0]
        r = np.empty(nrhs)
        bn = np.empty(nrhs)
        check(lib().dec_op_residual_norms(self._h, _ptr(x), _ptr(b), nrhs,
                                          r.ctypes.data_as(C.POINTER(C.c_double)),
                                          bn.ctypes.data_as(C.POINTER(C.c_double)), _stream()))
        return r, bn

    def autotune(self, reps=10):
        """Time the apply's rows-per-thread variants and record the fastest in the tuning table
        (dec_op_autotune); returns the choice (0: this operator's kernel has no variants)."""
        c = C.c_int32()
        check(lib().dec_op_autotune(self._h, reps, _stream(), C.byref(c)))
        return c.value

    def csr(self):
        """(indptr, indices, data, shape) of the operator, exported to the host."""
        nnz = C.c_int64()
        check(lib().dec_op_export_csr(self._h, C.byref(nnz), None, None, None))
        rp = np.empty(self.shape[0] + 1, np.int32)
        ci = np.empty(nnz.value, np.int32)
        v = np.empty(nnz.value, np.float64)
        check(lib().dec_op_export_csr(self._h, C.byref(nnz), rp.ctypes.data_as(C.c_void_p),
                                      ci.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p)))
        return rp, ci, v, self.shape


def _csc_struct(A, keep, index_base=0):
    """dec_csc of a scipy sparse matrix or an (colptr, rowval, nzval, (m, n)) tuple (0-based)."""
    if isinstance(A, tuple):
        cp, rv, nz, shape = A
    else:
        A = A.tocsc()
        A.sort_indices()
        cp, rv, nz, shape = A.indptr, A.indices, A.data, A.shape
    cp = np.ascontiguousarray(np.asarray(cp) + index_base, np.int32)
    rv = np.ascontiguousarray(np.asarray(rv) + index_base, np.int32)
    nz = np.ascontiguousarray(nz, np.float64)
    keep += [cp, rv, nz]
    c = _capi.Csc()
    c.m, c.n, c.index_base = int(shape[0]), int(shape[1]), index_base
    c.colptr, c.rowval, c.nzval = (cp.ctypes.data_as(C.c_void_p), rv.ctypes.data_as(C.c_void_p),
                                   nz.ctypes.data_as(C.c_void_p))
    return c


def sparse_operator(A, dtype="float64", index_base=0):
    """A caller's sparse matrix (scipy sparse, or a CSC tuple) as a device operator
    (dec_op_create_csc): ``op @ x`` is the reference's ``A * x`` on a SparseMatrixCSC."""
    keep = []
    c = _csc_struct(A, keep, index_base)
    h = C.c_void_p()
    check(lib().dec_op_create_csc(C.byref(c), _dtype_code(dtype), C.byref(h)))
    return Operator(None, 0, handle=h, owned=True, code=_dtype_code(dtype))


def tune_set(key, value):
    """Set an entry of the autotuner's table (dec_tune_set)."""
    check(lib().dec_tune_set(key.encode(), int(value)))


def tune_get(key):
    """The tuning table's entry for `key`, or None (dec_tune_get)."""
    v, found = C.c_int32(), C.c_int32()
    check(lib().dec_tune_get(key.encode(), C.byref(v), C.byref(found)))
    return v.value if found.value else None


def tune_clear():
    check(lib().dec_tune_clear())


def tune_entries():
    """The autotuner's table as a dict (through dec_tune_save into a temporary file)."""
    import json
    import os
    import tempfile
    fd, path = tempfile.mkstemp(suffix=".json")
    os.close(fd)
    try:
        tune_save(path)
        with open(path) as f:
            return json.load(f)["entries"]
    finally:
        os.unlink(path)


def tune_save(path):
    """Write the autotuner's table as JSON (dec_tune_save)."""
    check(lib().dec_tune_save(str(path).encode()))


def tune_load(path):
    """Merge a saved tuning table into the current one; returns the entries read (dec_tune_load)."""
    n = C.c_int32()
    check(lib().dec_tune_load(str(path).encode(), C.byref(n)))
    return n.value


def dec_differential(n, sd, dtype="float64"):
    return Operator(sd, {0: _capi.DEC_OP_D0, 1: _capi.DEC_OP_D1}[n], dtype)


def dec_boundary(n, sd, dtype="float64"):
    return Operator(sd, {1: _capi.DEC_OP_BOUNDARY1, 2: _capi.DEC_OP_BOUNDARY2}[n], dtype)


def dec_dual_derivative(n, sd, dtype="float64"):
    return Operator(sd, {0: _capi.DEC_OP_DUAL_D0, 1: _capi.DEC_OP_DUAL_D1}[n], dtype)


def dec_hodge_star(n, sd, dtype="float64"):
    """Diagonal Hodge star ⋆n as a device vector (the CuArray of the reference's CUDA backend)."""
    return _hodge(n, sd, 0, dtype)


def dec_inv_hodge_star(n, sd, dtype="float64"):
    return _hodge(n, sd, 1, dtype)


def _hodge(n, sd, inverse, dtype):
    torch = _torch()
    code = _dtype_code(dtype)
    size = {0: sd.nv, 1: sd.ne, 2: sd.nt}[n]
    out = torch.empty(size, dtype=_torch_dtype(code), device="cuda")
    check(lib().dec_hodge_diag(sd._h, n, inverse, code, _ptr(out), _stream()))
    return out


def hodge_operator(n, sd, inverse=False, dtype="float64", hodge="diagonal"):
    """⋆n (or its inverse) as an operator.  hodge="geometric" with n = 1 is the sparse
    GeometricHodge ⋆1 (FastDEC.jl:660-716); its inverse is a Krylov solve with -⋆1 (the
    reference's dec_inv_hodge_star(1, sd, GeometricHodge()))."""
    if hodge == "geometric" and n == 1:
        kind = _capi.DEC_OP_INV_STAR1_GEOMETRIC if inverse else _capi.DEC_OP_STAR1_GEOMETRIC
    elif hodge in ("diagonal", "geometric"):
        kind = (_capi.DEC_OP_INV_STAR0 if inverse else _capi.DEC_OP_STAR0) + n
    else:
        raise ValueError(f"unknown hodge {hodge!r}")
    return Operator(sd, kind, dtype)


def laplace_beltrami(sd, dtype="float64"):
    """fast_laplace_beltrami(sd) = -⋆0⁻¹ dual_d(1) ⋆1 d(0) = ⋆0⁻¹ d0ᵀ ⋆1 d0 (test/Multigrid.jl:46-48)."""
    return Operator(sd, _capi.DEC_OP_LAPLACE0, dtype)


def helmholtz(sd, shift, dtype="float64"):
    """laplace_beltrami(sd) + shift * I."""
    return Operator(sd, _capi.DEC_OP_HELMHOLTZ0, dtype, shift=shift)


def flat_sharp(sd, dtype="float64"):
    """♭♯_mat(sd) (DiscreteExteriorCalculus.jl:1992): dual 1-form -> primal 1-form, as an operator."""
    return Operator(sd, _capi.DEC_OP_FLAT_SHARP, dtype)


# ---- dual-dual interior product, Lie derivative and dual Laplacians (2D) ----------------------
# The reference composes these from its operators (FastDEC.jl:762-853); so does this mirror, with
# every factor a device operator of this library.  GeometricHodge throughout: ⋆1 is the sparse
# geometric star and its inverse the (-⋆1)⁻¹ Krylov solve; ⋆0, ⋆2 and their inverses are diagonal.

def _diag(v):
    return lambda x: v * x


def interior_product_dd(m, n, sd):
    """interior_product_dd(Val(m), Val(n), sd) (FastDEC.jl:765-790), FP64.
    (1,1): (f, g) -> ⋆2 ∧pd11(⋆1⁻¹ g, f), dual 1-forms f, g -> dual 0-form.
    (1,2): (f, g) -> ⋆1 ♭♯ ((Λpd01 (⋆0⁻¹ g)) .* f), dual 1-form f, dual 2-form g -> dual 1-form."""
    if (m, n) == (1, 1):
        ihs1 = hodge_operator(1, sd, inverse=True, hodge="geometric")
        w11 = dec_wedge_product_pd(1, 1, sd)
        hs2 = _diag(dec_hodge_star(2, sd))
        return lambda f, g: hs2(w11(ihs1(g), f))
    if (m, n) == (1, 2):
        ihs0 = _diag(dec_inv_hodge_star(0, sd))
        hs1 = hodge_operator(1, sd, hodge="geometric")
        fs = flat_sharp(sd)
        w01 = dec_wedge_product_pd(0, 1, sd)  # (g, f) -> (Λpd01 g) .* f
        return lambda f, g: hs1(fs(w01(ihs0(g), f)))
    raise ValueError(f"interior_product_dd: unsupported degrees ({m}, {n})")


def lie_derivative_dd(m, n, sd):
    """ℒ_dd(Val(1), Val(1), sd) (FastDEC.jl:795-802): (f, g) -> -(dd0 i1(f, g)) - i2(f, dd1 g), with
    i1 = interior_product_dd(1, 1), i2 = interior_product_dd(1, 2), ddk the dual derivatives."""
    if (m, n) != (1, 1):
        raise ValueError(f"lie_derivative_dd: unsupported degrees ({m}, {n})")
    dd0, dd1 = dec_dual_derivative(0, sd), dec_dual_derivative(1, sd)
    i1, i2 = interior_product_dd(1, 1, sd), interior_product_dd(1, 2, sd)

    def lie(f, g):
        a = dd0(i1(f, g))
        b = i2(f, dd1(g))
        return -a - b
    return lie


ℒ_dd = lie_derivative_dd


def dual_laplacian(k, sd):
    """Δᵈ(Val(k), sd) on a 2D complex (FastDEC.jl:812-853), FP64.
    k = 0: x -> ⋆2 d1 ⋆1⁻¹ (dd0 x) (dual 0-forms, length nt).
    k = 1: x -> ⋆1 d0 ⋆0⁻¹ dd1 x + dd0 ⋆2 d1 ⋆1⁻¹ x (dual 1-forms, length ne)."""
    dd0 = dec_dual_derivative(0, sd)
    ihs1 = hodge_operator(1, sd, inverse=True, hodge="geometric")
    d1 = dec_differential(1, sd)
    hs2 = _diag(dec_hodge_star(2, sd))
    if k == 0:
        return lambda x: hs2(d1(ihs1(dd0(x))))
    if k == 1:
        dd1 = dec_dual_derivative(1, sd)
        ihs0 = _diag(dec_inv_hodge_star(0, sd))
        d0 = dec_differential(0, sd)
        hs1 = hodge_operator(1, sd, hodge="geometric")
        return lambda x: hs1(d0(ihs0(dd1(x)))) + dd0(hs2(d1(ihs1(x))))
    raise ValueError(f"dual_laplacian: unsupported degree {k}")


Δᵈ = dual_laplacian


# ---- multigrid ------------------------------------------------------------------------------

def default_mg_options():
    o = _capi.MGOptions()
    lib().dec_mg_default_options(C.byref(o))
    return o


class MultigridData:
    """MultigridData(s, BinarySubdivision(), levels, op = L + shift I, steps) on the device.

    ``coarse`` is a host mesh description (anything with the oracle Mesh attributes or a
    ``Mesh``-compatible tuple); options follow ``dec_mg_options``.
    """

    def __init__(self, coarse, levels, shift=0.0, center="circumcenter", project_radius=0.0, mode="direct",
                 **opts):
        """mode: "direct" (DirectMode: every level discretised on its own mesh) or "galerkin"
        (GalerkinMode: coarse operators R A P, Multigrid.jl:740-748)."""
        o = default_mg_options()
        if mode not in ("direct", "galerkin"):
            raise ValueError(f"unknown multigrid mode {mode!r}")
        o.galerkin = 1 if mode == "galerkin" else 0
        o.levels = levels
        o.center = CENTERS[center] if isinstance(center, str) else int(center)
        o.project_radius = project_radius
        o.shift = shift
        for k, v in opts.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown multigrid option {k}")
            setattr(o, k, v)
        self.options = o
        keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data_as(C.c_void_p)

        d = _capi.MeshDesc()
        pts = np.ascontiguousarray(coarse.points, np.float64)
        d.nv, d.ne, d.nt = pts.shape[0], len(coarse.ev0), len(coarse.te0)
        d.index_base = 0
        d.points = arr(pts, np.float64)
        d.e_v0, d.e_v1 = arr(coarse.ev0, np.int32), arr(coarse.ev1, np.int32)
        d.t_e0, d.t_e1, d.t_e2 = (arr(coarse.te0, np.int32), arr(coarse.te1, np.int32),
                                  arr(coarse.te2, np.int32))
        d.edge_orientation = None if coarse.edge_orientation is None else arr(coarse.edge_orientation, np.int8)
        d.tri_orientation = None if coarse.tri_orientation is None else arr(coarse.tri_orientation, np.int8)
        d.center = o.center
        h = C.c_void_p()
        check(lib().dec_mg_create(C.byref(d), C.byref(o), C.byref(h)))
        self._h = h
        self.nlevels = levels + 1

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _capi is not None and _capi._lib is not None:
            _capi._lib.dec_mg_destroy(h)
            self._h = None

    @classmethod
    def from_matrices(cls, operators, restrictions, prolongations, steps=None, index_base=0, **opts):
        """MultigridData(g, r, p, s) (Multigrid.jl:538-546) from caller matrices, finest first:
        square operators, restrictions (n_{k+1} x n_k), prolongations (n_k x n_{k+1}), each a scipy
        sparse matrix or a CSC tuple; steps: one int for every level, a list per level, or None
        (opts pre / post).  dec_mg_create_from_csc."""
        o = default_mg_options()
        for k, v in opts.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown multigrid option {k}")
            setattr(o, k, v)
        nl = len(operators)
        if len(restrictions) != nl - 1 or len(prolongations) != nl - 1:
            raise ValueError("one restriction and one prolongation per level pair")
        keep = []
        ops = (_capi.Csc * nl)(*[_csc_struct(A, keep, index_base) for A in operators])
        rs = (_capi.Csc * max(1, nl - 1))(*[_csc_struct(A, keep, index_base) for A in restrictions])
        ps = (_capi.Csc * max(1, nl - 1))(*[_csc_struct(A, keep, index_base) for A in prolongations])
        st = None
        if steps is not None:
            sv = [int(steps)] * nl if np.isscalar(steps) else [int(x) for x in steps]
            if len(sv) != nl:
                raise ValueError("one steps entry per level")
            st = (C.c_int32 * nl)(*sv)
        h = C.c_void_p()
        check(lib().dec_mg_create_from_csc(nl, ops, rs, ps, st, C.byref(o), C.byref(h)))
        self = cls.__new__(cls)
        self.options = o
        self._h = h
        self.nlevels = nl
        return self

    def set_level_steps(self, steps):
        """MultigridData.steps: smoother steps before and after the coarse correction per level
        (None restores the options' pre / post).  dec_mg_set_level_steps."""
        if steps is None:
            check(lib().dec_mg_set_level_steps(self._h, None))
            return
        sv = [int(steps)] * self.nlevels if np.isscalar(steps) else [int(x) for x in steps]
        if len(sv) != self.nlevels:
            raise ValueError("one steps entry per level")
        check(lib().dec_mg_set_level_steps(self._h, (C.c_int32 * len(sv))(*sv)))

    def level_info(self, level):
        nv, ne, nt, lm = C.c_int64(), C.c_int64(), C.c_int64(), C.c_double()
        check(lib().dec_mg_level_info(self._h, level, C.byref(nv), C.byref(ne), C.byref(nt), C.byref(lm)))
        return nv.value, ne.value, nt.value, lm.value

    def level_mesh(self, level):
        h = C.c_void_p()
        check(lib().dec_mg_level_mesh(self._h, level, C.byref(h)))
        m = Mesh._borrow(h)
        m._parent = self
        return m

    def level_op(self, level):
        h = C.c_void_p()
        check(lib().dec_mg_level_op(self._h, level, C.byref(h)))
        op = Operator(None, 0, handle=h)
        op._parent = self
        return op

    @property
    def n(self):
        return self.level_info(0)[0]

    def cycles(self, u, b, cycles):
        """u <- `cycles` V- (or W-) cycles on A u = b; u, b float64 CUDA tensors (n,) or (nrhs, n)."""
        nrhs = 1 if b.dim() == 1 else b.shape[0]
        check(lib().dec_mg_cycles(self._h, _ptr(u), _ptr(b), nrhs, cycles, _stream()))
        return u

    def autotune(self, nrhs, reps=3):
        """Pick the fastest panel width for `nrhs` right-hand sides (dec_mg_autotune)."""
        k = C.c_int32()
        check(lib().dec_mg_autotune(self._h, nrhs, reps, _stream(), C.byref(k)))
        return k.value

    def solve_traffic(self, nrhs, iterations, from_zero=True):
        """Algorithmic bytes of a device-loop solve of `nrhs` right-hand sides that ran `iterations`
        refinement steps (dec_mg_solve_traffic)."""
        by = C.c_double()
        check(lib().dec_mg_solve_traffic(self._h, nrhs, 1 if from_zero else 0, iterations, C.byref(by)))
        return by.value

    def set_smoother_mlp(self, mlp):
        """Attach the learned smoother network used by smoother=DEC_SMOOTH_LEARNED (None detaches)."""
        check(lib().dec_mg_set_smoother_mlp(self._h, None if mlp is None else mlp._h))
        self._mlp = mlp  # keep the network alive while the hierarchy uses it

    def time_kernel(self, kernel, level, nrhs, reps=20):
        """(ms per launch, algorithmic bytes per launch) of one V-cycle kernel (dec_mg_time_kernel)."""
        ms, by = C.c_double(), C.c_double()
        check(lib().dec_mg_time_kernel(self._h, kernel, level, nrhs, reps, _stream(), C.byref(ms), C.byref(by)))
        return ms.value, by.value

    def solve(self, u, b, rtol=1e-8, max_iters=100, shifts=None, use_initial_guess=True):
        """FP64-refined solve of A u = b (u in/out); with `shifts` (coarse_solver=2 hierarchies)
        right-hand side j solves (L + (shift + shifts[j]) I) u_j = b_j.  use_initial_guess=False
        starts from u = 0 (u is output only; dec_mg_solve_from_zero)."""
        nrhs = 1 if b.dim() == 1 else b.shape[0]
        rep = _capi.SolveReport()
        if shifts is not None:
            sh = np.ascontiguousarray(shifts, np.float64)
            if sh.size != nrhs:
                raise ValueError("one shift per right-hand side")
            if not use_initial_guess:
                u.zero_()
            st = lib().dec_mg_solve_shifted(self._h, _ptr(u), _ptr(b), nrhs, sh.ctypes.data_as(C.c_void_p), rtol,
                                            max_iters, C.byref(rep), _stream())
            if st not in (_capi.DEC_OK, 4):
                check(st)
            return u, rep
        fn = lib().dec_mg_solve if use_initial_guess else lib().dec_mg_solve_from_zero
        st = fn(self._h, _ptr(u), _ptr(b), nrhs, rtol, max_iters, C.byref(rep), _stream())
        if st not in (_capi.DEC_OK, 4):
            check(st)
        return u, rep

    def solve_host(self, u, b, rtol=1e-8, max_iters=100, use_initial_guess=True):
        """Same solve on host float64 arrays ((n,) or (nrhs, n); numpy or pinned torch CPU tensors);
        the host<->device copies are part of the call.  use_initial_guess=False starts from zero
        and treats u as output only."""
        nrhs = 1 if b.ndim == 1 else b.shape[0]
        rep = _capi.SolveReport()

        def hp(a):
            return C.c_void_p(a.data_ptr()) if hasattr(a, "data_ptr") else a.ctypes.data_as(C.c_void_p)

        st = lib().dec_mg_solve_host(self._h, hp(u), hp(b), nrhs, rtol, max_iters, int(use_initial_guess),
                                     C.byref(rep), _stream())
        if st not in (_capi.DEC_OK, 4):
            check(st)
        return u, rep

    def solve_host_submit(self, u, b, rtol=1e-8, max_iters=100, use_initial_guess=True):
        """Pipelined solve_host: enqueues the copies and the solve on the hierarchy's own streams
        and returns a PendingSolve at once; three may be in flight, so neighbouring solves'
        host<->device copies overlap each one's compute (pinned torch CPU tensors give the
        overlap).  u and b must stay alive until PendingSolve.wait()."""
        nrhs = 1 if b.ndim == 1 else b.shape[0]
        hp = (lambda a: C.c_void_p(a.data_ptr()) if hasattr(a, "data_ptr") else a.ctypes.data_as(C.c_void_p))
        t = C.c_uint64()
        check(lib().dec_mg_solve_host_submit(self._h, hp(u), hp(b), nrhs, rtol, max_iters, int(use_initial_guess),
                                             C.byref(t)))
        return PendingSolve(self, t.value, u, b)


class PendingSolve:
    """A submitted host-buffer solve (MultigridData.solve_host_submit)."""

    def __init__(self, mg, ticket, u, b):
        self.mg, self.ticket, self.u, self.b = mg, ticket, u, b
        self.report = None

    def wait(self):
        """Blocks until u holds the solution; returns (u, SolveReport)."""
        if self.report is None:
            rep = _capi.SolveReport()
            st = lib().dec_mg_solve_host_wait(self.mg._h, self.ticket, C.byref(rep))
            if st not in (_capi.DEC_OK, 4):
                check(st)
            self.report = rep
        return self.u, self.report


class Batch:
    """Batched solves over several MultigridData hierarchies (dec_batch_*): each refinement step
    of every group runs as one CUDA graph with a concurrent branch per group."""

    def __init__(self, groups):
        self.groups = list(groups)
        arr = (C.c_void_p * len(self.groups))(*[g._h.value for g in self.groups])
        h = C.c_void_p()
        check(lib().dec_batch_create(arr, len(self.groups), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _capi is not None and _capi._lib is not None:
            _capi._lib.dec_batch_destroy(h)
            self._h = None

    def autotune(self, nrhs, reps=3):
        n = (C.c_int32 * len(nrhs))(*nrhs)
        check(lib().dec_batch_autotune(self._h, n, reps, _stream()))

    def solve(self, us, bs, shifts=None, rtol=1e-8, max_iters=100):
        """us, bs: per group float64 CUDA tensors (nrhs_g, n_g) (us in/out); shifts: per group
        host arrays or None.  Returns (per-group reports, total report)."""
        G = len(self.groups)
        nrhs = [1 if b.dim() == 1 else b.shape[0] for b in bs]
        up = (C.c_void_p * G)(*[u.data_ptr() for u in us])
        bp = (C.c_void_p * G)(*[b.data_ptr() for b in bs])
        nr = (C.c_int32 * G)(*nrhs)
        keep = []
        sp = None
        if shifts is not None:
            ptrs = []
            for sh in shifts:
                if sh is None:
                    ptrs.append(None)
                else:
                    a = np.ascontiguousarray(sh, np.float64)
                    keep.append(a)
                    ptrs.append(a.ctypes.data)
            sp = (C.c_void_p * G)(*ptrs)
        reps = (_capi.SolveReport * G)()
        tot = _capi.SolveReport()
        st = lib().dec_batch_solve(self._h, up, bp, nr, sp, rtol, max_iters, reps, C.byref(tot), _stream())
        if st not in (_capi.DEC_OK, 4):
            check(st)
        return list(reps), tot

    def traffic(self, iterations):
        """Algorithmic bytes of the captured batch graph run for `iterations` refinement steps
        (dec_batch_traffic)."""
        by = C.c_double()
        check(lib().dec_batch_traffic(self._h, iterations, C.byref(by)))
        return by.value


class SmootherMLP:
    """The learned smoother's network (dec_mlp_*): per-vertex MLP 16 -> 64 -> 64 -> 1, ReLU,
    BF16 weights and activations on the tensor cores with FP32 accumulation, FP32 master
    parameters trained with Adam by the library's own forward / backward kernels."""

    NPARAM = _capi.DEC_MLP_NPARAM

    def __init__(self, seed=4):
        h = C.c_void_p()
        check(lib().dec_mlp_create(C.c_uint64(seed), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _capi is not None and _capi._lib is not None:
            _capi._lib.dec_mlp_destroy(h)
            self._h = None

    @property
    def params(self):
        p = np.empty(self.NPARAM, np.float32)
        check(lib().dec_mlp_get_params(self._h, p.ctypes.data_as(C.c_void_p)))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.NPARAM:
            raise ValueError(f"expected {self.NPARAM} parameters")
        check(lib().dec_mlp_set_params(self._h, p.ctypes.data_as(C.c_void_p)))

    @property
    def step(self):
        s = C.c_int64()
        check(lib().dec_mlp_step(self._h, C.byref(s)))
        return s.value

    def eval(self, x, tensor_cores=True):
        """y = MLP(x) for x a float32 CUDA tensor (n, 16); tensor_cores: False (CUDA cores),
        True / 1 (mma.sync) or 2 (tcgen05 with TMEM accumulators)."""
        torch = _torch()
        x = x.contiguous()
        y = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        check(lib().dec_mlp_eval(self._h, _ptr(x), x.shape[0], _ptr(y), int(tensor_cores), _stream()))
        return y

    def set_engine(self, engine):
        """Kernel engine of the learned smoothing step: "tcgen05" (the default; TMEM accumulators,
        eight 128-sample tile chains per SM) or "mma" (mma.sync)."""
        check(lib().dec_mlp_set_engine(self._h, {"mma": 0, "tcgen05": 1}[engine]))

    def grad(self, x, dy):
        """Σ_q dy_q ∂MLP(x_q)/∂params as a float32 CUDA tensor (NPARAM,)."""
        torch = _torch()
        g = torch.empty(self.NPARAM, dtype=torch.float32, device=x.device)
        check(lib().dec_mlp_grad(self._h, _ptr(x.contiguous()), _ptr(dy.contiguous()), x.shape[0], _ptr(g),
                                 _stream()))
        return g

    @staticmethod
    def features(op, r):
        """(features (n*S, 16), scales s/a_ii (n*S,)) of residual fields r (S, n) float64."""
        torch = _torch()
        S = 1 if r.dim() == 1 else r.shape[0]
        n = op.shape[0]
        f = torch.empty((n * S, 16), dtype=torch.float32, device=r.device)
        sc = torch.empty(n * S, dtype=torch.float32, device=r.device)
        check(lib().dec_mlp_features(op._h, _ptr(r.contiguous()), S, _ptr(f), _ptr(sc), _stream()))
        return f, sc

    def loss_grad(self, op, r, grad=True):
        """(energy-norm loss, full parameter gradient or None) on residual fields r (S, n)."""
        torch = _torch()
        S = 1 if r.dim() == 1 else r.shape[0]
        loss = C.c_double()
        g = torch.empty(self.NPARAM, dtype=torch.float32, device=r.device) if grad else None
        check(lib().dec_mlp_loss_grad(self._h, op._h, _ptr(r.contiguous()), S, C.byref(loss),
                                      None if g is None else _ptr(g), _stream()))
        return loss.value, g

    def train(self, op, r, steps, lr=1e-3, batch=65536, seed=4, record_loss=False):
        """`steps` Adam steps on residual fields r (S, n) of op's mesh; returns the per-step losses
        (before each update) when record_loss, else None."""
        S = 1 if r.dim() == 1 else r.shape[0]
        losses = np.empty(steps) if record_loss else None
        check(lib().dec_mlp_train(self._h, op._h, _ptr(r.contiguous()), S, steps, float(lr), int(batch),
                                  C.c_uint64(seed), None if losses is None else losses.ctypes.data_as(C.c_void_p),
                                  _stream()))
        return losses

    def save(self, path):
        check(lib().dec_mlp_save(self._h, str(path).encode()))

    def load(self, path):
        check(lib().dec_mlp_load(self._h, str(path).encode()))


def multigrid_vcycles(u, b, md, cycles):
    """multigrid_vcycles(u, b, md, cycles) (Multigrid.jl:814): returns the updated u (a copy)."""
    u = u.clone()
    return md.cycles(u, b, cycles)


def full_multigrid(b, md, cycles):
    """full_multigrid(b, md, cycles, alg, μ) (Multigrid.jl:826-855): returns u; μ is the
    hierarchy's `mu` option."""
    torch = _torch()
    u = torch.empty_like(b)
    nrhs = 1 if b.dim() == 1 else b.shape[0]
    check(lib().dec_mg_full_multigrid(md._h, _ptr(u), _ptr(b.contiguous()), nrhs, cycles, _stream()))
    return u


def dec_inverse_laplacian(k, coarse, levels, steps=3, cycles=5, mu=2, center="circumcenter", project_radius=0.0):
    """dec_Δ⁻¹(Val(0), s; scheme=BinarySubdivision(), steps=3, cycles=5, alg=cg, μ=2)
    (FastDEC.jl:866-869): a hierarchy of `levels` binary subdivisions of `coarse` with the
    Laplacian ∇²(0) on every level and the reference's CG smoother, returned as
    b -> full_multigrid(b, md, cycles, cg, μ).  The hierarchy is the closure's `md`."""
    if k != 0:
        raise ValueError("dec_inverse_laplacian: only 0-forms (Val(0))")
    md = MultigridData(coarse, levels, shift=0.0, center=center, project_radius=project_radius,
                       smoother=_capi.DEC_SMOOTH_CG, pre=steps, post=steps, mu=mu, precision=0)

    def solve(b):
        return full_multigrid(b, md, cycles)
    solve.md = md
    return solve


def multigrid_wcycles(u, b, md, cycles):
    if md.options.mu != 2:
        raise ValueError("build the MultigridData with mu=2 for W-cycles")
    u = u.clone()
    return md.cycles(u, b, cycles)
