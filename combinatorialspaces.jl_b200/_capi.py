"""ctypes declarations of the C ABI in include/dec_b200.h."""
import ctypes as C
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent / "_lib" / "libdec_b200.so"

DEC_OK = 0
STATUS = {0: "DEC_OK", 1: "DEC_ERR_INVALID_ARG", 2: "DEC_ERR_OOM", 3: "DEC_ERR_CUDA",
          4: "DEC_ERR_NOT_CONVERGED", 5: "DEC_ERR_TIMEOUT", 6: "DEC_ERR_UNSUPPORTED",
          7: "DEC_ERR_NON_ORIENTABLE"}
DEC_F64, DEC_F32 = 0, 1
DEC_BARYCENTER, DEC_CIRCUMCENTER = 0, 1
DEC_WEDGE_PP, DEC_WEDGE_PD, DEC_WEDGE_DP, DEC_WEDGE_DD = 0, 1, 2, 3
(DEC_OP_D0, DEC_OP_D1, DEC_OP_BOUNDARY1, DEC_OP_BOUNDARY2, DEC_OP_DUAL_D0, DEC_OP_DUAL_D1,
 DEC_OP_STAR0, DEC_OP_STAR1, DEC_OP_STAR2, DEC_OP_INV_STAR0, DEC_OP_INV_STAR1, DEC_OP_INV_STAR2,
 DEC_OP_LAPLACE0, DEC_OP_HELMHOLTZ0, DEC_OP_STAR1_GEOMETRIC, DEC_OP_INV_STAR1_GEOMETRIC,
 DEC_OP_FLAT_SHARP, DEC_OP_GENERAL) = range(18)
DEC_GEOM_LENGTH, DEC_GEOM_AREA, DEC_GEOM_DUAL_AREA, DEC_GEOM_DUAL_LENGTH_TE, DEC_GEOM_DUAL_POINT = range(5)
DEC_SMOOTH_JACOBI, DEC_SMOOTH_CHEBYSHEV, DEC_SMOOTH_CG, DEC_SMOOTH_LEARNED = 0, 1, 2, 3
(DEC_KERNEL_SWEEP, DEC_KERNEL_RESIDUAL, DEC_KERNEL_RESTRICT, DEC_KERNEL_PROLONG, DEC_KERNEL_MLP, DEC_KERNEL_SWEEP_PAIR,
 DEC_KERNEL_SWEEP_PROLONGED0, DEC_KERNEL_SWEEP_PROLONGED1) = range(8)
DEC_MLP_NPARAM = 5313


class MeshDesc(C.Structure):
    _fields_ = [("nv", C.c_int32), ("ne", C.c_int32), ("nt", C.c_int32), ("index_base", C.c_int32),
                ("points", C.c_void_p), ("e_v0", C.c_void_p), ("e_v1", C.c_void_p),
                ("t_e0", C.c_void_p), ("t_e1", C.c_void_p), ("t_e2", C.c_void_p),
                ("edge_orientation", C.c_void_p), ("tri_orientation", C.c_void_p),
                ("center", C.c_int32)]


class MGOptions(C.Structure):
    _fields_ = [("levels", C.c_int32), ("center", C.c_int32), ("project_radius", C.c_double),
                ("shift", C.c_double), ("smoother", C.c_int32), ("pre", C.c_int32), ("post", C.c_int32),
                ("omega", C.c_double), ("cheb_ratio", C.c_double), ("coarse_solver", C.c_int32),
                ("precision", C.c_int32), ("rhs_block", C.c_int32), ("mu", C.c_int32),
                ("inner_cycles", C.c_int32), ("reorder", C.c_int32), ("coarse_max", C.c_int32),
                ("fallback_rho", C.c_double), ("galerkin", C.c_int32), ("device_loop", C.c_int32)]


class Csc(C.Structure):
    """dec_csc: a SparseMatrixCSC{Float64, Int32} in host memory."""
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("index_base", C.c_int32),
                ("colptr", C.c_void_p), ("rowval", C.c_void_p), ("nzval", C.c_void_p)]


class SolveReport(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32),
                ("max_rel_residual", C.c_double), ("seconds", C.c_double),
                ("launches", C.c_int64), ("rhs_block", C.c_int32), ("fallback_iteration", C.c_int32)]


P = C.c_void_p
PP = C.POINTER(C.c_void_p)
I32, I64, F64 = C.c_int32, C.c_int64, C.c_double
PI64 = C.POINTER(C.c_int64)
PF64 = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol declared in include/dec_b200.h
SIGNATURES = {
    "dec_last_error": (C.c_char_p, []),
    "dec_version": (I32, []),
    "dec_mesh_create": (I32, [C.POINTER(MeshDesc), PP]),
    "dec_mesh_destroy": (I32, [P]),
    "dec_mesh_counts": (I32, [P, PI64, PI64, PI64]),
    "dec_mesh_orientation": (I32, [P, P, P]),
    "dec_mesh_geometry": (I32, [P, I32, P, I64]),
    "dec_hodge_diag": (I32, [P, I32, I32, I32, P, P]),
    "dec_wedge_plan_create": (I32, [P, I32, I32, I32, I32, PP]),
    "dec_wedge_apply": (I32, [P, P, P, P, P]),
    "dec_wedge_lengths": (I32, [P, PI64, PI64, PI64]),
    "dec_wedge_apply_batched": (I32, [P, P, P, P, I32, P]),
    "dec_wedge_autotune": (I32, [P, I32, I32, P, C.POINTER(C.c_int32)]),
    "dec_wedge_plan_destroy": (I32, [P]),
    "dec_op_create": (I32, [P, I32, F64, I32, PP]),
    "dec_op_create_csc": (I32, [C.POINTER(Csc), I32, PP]),
    "dec_op_shape": (I32, [P, PI64, PI64]),
    "dec_op_apply": (I32, [P, P, P, F64, F64, P]),
    "dec_op_export_csr": (I32, [P, PI64, P, P, P]),
    "dec_op_residual_norms": (I32, [P, P, P, I32, PF64, PF64, P]),
    "dec_op_residual_norms_noalloc": (I32, [P, P, P, I32, PF64, PF64, P]),
    "dec_op_destroy": (I32, [P]),
    "dec_mg_default_options": (None, [C.POINTER(MGOptions)]),
    "dec_mg_create": (I32, [C.POINTER(MeshDesc), C.POINTER(MGOptions), PP]),
    "dec_mg_create_from_csc": (I32, [I32, C.POINTER(Csc), C.POINTER(Csc), C.POINTER(Csc), C.POINTER(C.c_int32),
                                     C.POINTER(MGOptions), PP]),
    "dec_mg_set_level_steps": (I32, [P, C.POINTER(C.c_int32)]),
    "dec_mg_destroy": (I32, [P]),
    "dec_mg_level_info": (I32, [P, I32, PI64, PI64, PI64, PF64]),
    "dec_mg_level_mesh": (I32, [P, I32, PP]),
    "dec_mg_level_op": (I32, [P, I32, PP]),
    "dec_mg_cycles": (I32, [P, P, P, I32, I32, P]),
    "dec_mg_full_multigrid": (I32, [P, P, P, I32, I32, P]),
    "dec_mg_solve": (I32, [P, P, P, I32, F64, I32, C.POINTER(SolveReport), P]),
    "dec_mg_solve_from_zero": (I32, [P, P, P, I32, F64, I32, C.POINTER(SolveReport), P]),
    "dec_mg_solve_host": (I32, [P, P, P, I32, F64, I32, I32, C.POINTER(SolveReport), P]),
    "dec_c_wedge_apply": (I32, [I32, I32, I64, P, P, I32, P, P, P, I32, P]),
    "dec_mg_solve_host_submit": (I32, [P, P, P, I32, F64, I32, I32, C.POINTER(C.c_uint64)]),
    "dec_mg_solve_host_wait": (I32, [P, C.c_uint64, C.POINTER(SolveReport)]),
    "dec_mg_time_kernel": (I32, [P, I32, I32, I32, I32, P, PF64, PF64]),
    "dec_mg_autotune": (I32, [P, I32, I32, P, C.POINTER(C.c_int32)]),
    "dec_mg_solve_traffic": (I32, [P, I32, I32, I32, PF64]),
    "dec_op_autotune": (I32, [P, I32, P, C.POINTER(C.c_int32)]),
    "dec_tune_set": (I32, [C.c_char_p, I32]),
    "dec_tune_get": (I32, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "dec_tune_clear": (I32, []),
    "dec_tune_save": (I32, [C.c_char_p]),
    "dec_tune_load": (I32, [C.c_char_p, C.POINTER(C.c_int32)]),
    "dec_mg_set_smoother_mlp": (I32, [P, P]),
    "dec_mg_solve_shifted": (I32, [P, P, P, I32, P, F64, I32, C.POINTER(SolveReport), P]),
    "dec_batch_create": (I32, [P, I32, PP]),
    "dec_batch_destroy": (I32, [P]),
    "dec_batch_autotune": (I32, [P, P, I32, P]),
    "dec_batch_traffic": (I32, [P, I32, C.POINTER(C.c_double)]),
    "dec_batch_solve": (I32, [P, P, P, P, P, F64, I32, P, C.POINTER(SolveReport), P]),
    "dec_mlp_create": (I32, [C.c_uint64, PP]),
    "dec_mlp_destroy": (I32, [P]),
    "dec_mlp_get_params": (I32, [P, P]),
    "dec_mlp_set_params": (I32, [P, P]),
    "dec_mlp_step": (I32, [P, PI64]),
    "dec_mlp_eval": (I32, [P, P, I64, P, I32, P]),
    "dec_mlp_grad": (I32, [P, P, P, I64, P, P]),
    "dec_mlp_features": (I32, [P, P, I32, P, P, P]),
    "dec_mlp_loss_grad": (I32, [P, P, P, I32, PF64, P, P]),
    "dec_mlp_train": (I32, [P, P, P, I32, I32, F64, I64, C.c_uint64, P, P]),
    "dec_mlp_save": (I32, [P, C.c_char_p]),
    "dec_mlp_set_engine": (I32, [P, I32]),
    "dec_mlp_load": (I32, [P, C.c_char_p]),
}


class DecError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib():
    """The loaded libdec_b200.so.  Raises if the library has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with combinatorialspaces.jl_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != DEC_OK:
        raise DecError(status, lib().dec_last_error().decode(errors="replace"))
