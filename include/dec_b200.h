/*
 * dec_b200.h - C ABI of libdec_b200.so, the sm_100a (B200) implementation of the
 * CombinatorialSpaces.jl DEC hot path: FastDEC wedge products, the exterior derivative /
 * boundary / Hodge star / Laplace-Beltrami operators, and the Multigrid.jl geometric V-cycle
 * over binary-subdivision hierarchies.
 *
 * Conventions
 *  - Every entry point returns a dec_status; on failure dec_last_error() holds a message
 *    (thread-local).  Nothing aborts or traps.
 *  - Forms (cochains) are caller-owned DEVICE arrays in the reference's element order
 *    (vertices, edges, triangles as numbered by the mesh description).  Work is enqueued on
 *    the caller's stream (a cudaStream_t passed as void*, NULL = legacy default stream).
 *  - Mesh, plan, operator and multigrid handles own their device memory.  A handle must not
 *    be used from two host threads at once.
 *  - Index arrays in dec_mesh_desc are int32 with a selectable base (1 for Julia callers).
 */
#ifndef DEC_B200_H
#define DEC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum dec_status {
  DEC_OK = 0,
  DEC_ERR_INVALID_ARG = 1,
  DEC_ERR_OOM = 2,
  DEC_ERR_CUDA = 3,
  DEC_ERR_NOT_CONVERGED = 4,
  DEC_ERR_TIMEOUT = 5,
  DEC_ERR_UNSUPPORTED = 6,
  DEC_ERR_NON_ORIENTABLE = 7
} dec_status;

typedef enum dec_dtype { DEC_F64 = 0, DEC_F32 = 1 } dec_dtype;

/* Barycenter() / Circumcenter(), src/DiscreteExteriorCalculus.jl:98-135 */
typedef enum dec_center { DEC_BARYCENTER = 0, DEC_CIRCUMCENTER = 1 } dec_center;

typedef struct dec_mesh dec_mesh;
typedef struct dec_wedge_plan dec_wedge_plan;
typedef struct dec_op dec_op;
typedef struct dec_mg dec_mg;
typedef struct dec_mlp dec_mlp;
typedef struct dec_batch dec_batch;

/*
 * A primal 2D delta set with embedding, i.e. the fields of EmbeddedDeltaSet2D{Bool,Point3d}
 * that the dual complex is built from (src/SimplicialSets.jl:221-411; the dual complex and its
 * geometry follow src/DiscreteExteriorCalculus.jl:545-608 and :935-990).
 */
typedef struct dec_mesh_desc {
  int32_t nv, ne, nt;
  int32_t index_base;              /* 1 (Julia) or 0 */
  const double* points;            /* nv x 3 row-major (x, y, z); host memory */
  const int32_t* e_v0;             /* ∂v0 of each edge (its target); host */
  const int32_t* e_v1;             /* ∂v1 of each edge (its source); host */
  const int32_t* t_e0;             /* ∂e0, ∂e1, ∂e2 of each triangle; host */
  const int32_t* t_e1;
  const int32_t* t_e2;
  const int8_t* edge_orientation;  /* ne; 1 true, 0 false, -1 unset (-> false); NULL = all unset */
  const int8_t* tri_orientation;   /* nt; NULL or any -1 => orient!(s, Val(2)) is run */
  int32_t center;                  /* dec_center */
} dec_mesh_desc;

const char* dec_last_error(void);
int32_t dec_version(void);

/* ---- mesh (replaces dualize(s, alg) + the per-operator host setup of FastDEC) ---------- */
dec_status dec_mesh_create(const dec_mesh_desc* desc, dec_mesh** out);
dec_status dec_mesh_destroy(dec_mesh* m);
dec_status dec_mesh_counts(const dec_mesh* m, int64_t* nv, int64_t* ne, int64_t* nt);
/* Orientation actually used (after orient!), copied to host arrays of ne / nt bytes. */
dec_status dec_mesh_orientation(const dec_mesh* m, int8_t* edge_orientation, int8_t* tri_orientation);

/* Geometry arrays copied to host (FP64), for parity checks:
 * 0 length[ne], 1 area[nt], 2 dual_area[6nt] (dual-triangle order of the reference),
 * 3 dual_length of the 3nt triangle-center -> edge-center dual edges, 4 dual_point[3(nv+ne+nt)] */
typedef enum dec_geometry { DEC_GEOM_LENGTH = 0, DEC_GEOM_AREA = 1, DEC_GEOM_DUAL_AREA = 2,
                            DEC_GEOM_DUAL_LENGTH_TE = 3, DEC_GEOM_DUAL_POINT = 4 } dec_geometry;
dec_status dec_mesh_geometry(const dec_mesh* m, int32_t which, double* host_out, int64_t len);

/* ---- Hodge star (replaces dec_hodge_star / dec_inv_hodge_star(n, sd, DiagonalHodge(),
 *      Val(:CUDA)), ext/CombinatorialSpacesCUDAExt.jl:70-96, which return a CuArray) ------- */
dec_status dec_hodge_diag(const dec_mesh* m, int32_t k, int32_t inverse, dec_dtype dtype,
                          void* out, void* stream);

/* ---- wedge products (replaces dec_wedge_product(m, n, sd, Val(:CUDA), CuArray, T) and
 *      dec_c_wedge_product!, src/FastDEC.jl:217-289, and the pd / dp / dd wedges :291-401) ---- */
typedef enum dec_wedge_kind {
  DEC_WEDGE_PP = 0, /* primal-primal (0,1) (1,0) (0,2) (2,0) (1,1), FastDEC.jl:255-279 */
  DEC_WEDGE_PD = 1, /* primal-dual (0,1) (1,1), FastDEC.jl:386-395 */
  DEC_WEDGE_DP = 2, /* dual-primal (1,0) (1,1), FastDEC.jl:381-384, :397-401 */
  DEC_WEDGE_DD = 3  /* dual-dual (0,1) (1,0), FastDEC.jl:317-325 */
} dec_wedge_kind;
dec_status dec_wedge_plan_create(dec_mesh* m, int32_t kind, int32_t deg_a, int32_t deg_b,
                                 dec_dtype dtype, dec_wedge_plan** out);
/* out = a ∧ b; a and b are device forms in the degrees given at plan creation. */
dec_status dec_wedge_apply(dec_wedge_plan* p, const void* a, const void* b, void* out, void* stream);
/* Lengths of the a, b and out forms of a plan. */
dec_status dec_wedge_lengths(const dec_wedge_plan* p, int64_t* len_a, int64_t* len_b, int64_t* len_out);
/* Batched launch: out_i = a_i ∧ b_i for `count` form pairs laid out back to back. */
dec_status dec_wedge_apply_batched(dec_wedge_plan* p, const void* a, const void* b, void* out,
                                   int32_t count, void* stream);
/* Autotuner (no reference counterpart): times the batched FP32 ∧(1,1) with 1, 2, 4, 8 and 16 form
 * pairs per thread on min(count, 256) pairs and stores the fastest in the tuning table under the
 * plan's triangle-count bucket (dec_tune_save keeps it); *choice = the pairs per thread, or 0 when
 * the plan is not an FP32 ∧(1,1) or count < 2 (nothing tuned).  Untuned batches use 4. */
dec_status dec_wedge_autotune(dec_wedge_plan* p, int32_t count, int32_t reps, void* stream, int32_t* choice);
dec_status dec_wedge_plan_destroy(dec_wedge_plan* p);
/* dec_c_wedge_product!(Val(j), Val(k), res, α, β, p, c) (FastDEC.jl:217-232): a wedge kernel on
 * caller caches in the reference's layout (cache_wedge output, Julia column-major), for
 * (j,k) = (0,1), (0,2), (0,3), (1,1), (2,1) -- the 3D kernels included:
 *   (0,1): p n_out x 2 (edge endpoints), c unused:   res[i] = ½ β[i] (α[p[i,1]] + α[p[i,2]])
 *   (0,2): p, c 6 x n_out:                            res[i] = β[i] Σ_j c[j,i] α[p[j,i]]
 *   (0,3): p, c 24 x n_out (tetrahedra):              res[i] = Σ_j β[i] c[j,i] α[p[j,i]]
 *   (1,1): p, c 3 x n_out (edges of triangle i):       wedge_kernel_11!
 *   (2,1): p 10 x n_out (6 edges, 4 triangles of tetrahedron i), c 12 x n_out: wedge_kernel_21!
 * p: device int32, index_base 0 or 1 (Julia); c, a (α), b (β), res: device arrays of dtype. */
dec_status dec_c_wedge_apply(int32_t j, int32_t k, int64_t n_out, const int32_t* p, const void* c, dec_dtype dtype,
                             const void* a, const void* b, void* res, int32_t index_base, void* stream);

/* ---- sparse operators (replaces dec_differential / dec_boundary / dec_dual_derivative(n, sd,
 *      Val(:CUDA)), ext/CombinatorialSpacesCUDAExt.jl:30-61, the diagonal Hodge stars, and
 *      the Laplacian fast_laplace_beltrami of test/Multigrid.jl:46-48 = ∇²(0),
 *      src/DiscreteExteriorCalculus.jl:1889) ----------------------------------------------- */
typedef enum dec_op_kind {
  DEC_OP_D0 = 0, DEC_OP_D1 = 1,                 /* dec_differential(0|1), FastDEC.jl:468-524 */
  DEC_OP_BOUNDARY1 = 2, DEC_OP_BOUNDARY2 = 3,   /* dec_boundary(1|2), FastDEC.jl:433-437 */
  DEC_OP_DUAL_D0 = 4, DEC_OP_DUAL_D1 = 5,       /* dec_dual_derivative(0|1), FastDEC.jl:443-453 */
  DEC_OP_STAR0 = 6, DEC_OP_STAR1 = 7, DEC_OP_STAR2 = 8,            /* FastDEC.jl:580-604 */
  DEC_OP_INV_STAR0 = 9, DEC_OP_INV_STAR1 = 10, DEC_OP_INV_STAR2 = 11, /* FastDEC.jl:732-737 */
  DEC_OP_LAPLACE0 = 12,   /* ⋆0⁻¹ d0ᵀ ⋆1 d0 (positive semidefinite, = -Δ(0)) */
  DEC_OP_HELMHOLTZ0 = 13, /* ⋆0⁻¹ d0ᵀ ⋆1 d0 + shift * I */
  DEC_OP_STAR1_GEOMETRIC = 14,     /* dec_hodge_star(1, sd, GeometricHodge()), FastDEC.jl:660-716 (sparse
                                      ne x ne; the diagonal ⋆1 on planar circumcentric duals) */
  DEC_OP_INV_STAR1_GEOMETRIC = 15  /* dec_inv_hodge_star(1, sd, GeometricHodge()), FastDEC.jl:745-748,
                                      CUDA ext :93-96: y = (-⋆1)⁻¹ x by a Jacobi-preconditioned
                                      BiCGSTAB solve in FP64 to 1e-14 relative residual (one host
                                      read-back per reduction; not capturable in a CUDA graph) */,
  DEC_OP_FLAT_SHARP = 16           /* ♭♯_mat(sd) (DiscreteExteriorCalculus.jl:1992; ♭ :687-714, ♯ :876-909):
                                      dual 1-form -> primal 1-form, ne x ne, <= 6 nnz per row (the
                                      matrix inside dec_wedge_product_pd/dp(1,1), FastDEC.jl:391-401) */,
  DEC_OP_GENERAL = 17              /* a caller's sparse matrix (dec_op_create_csc): the reference's A * x on a
                                      SparseMatrixCSC / CuSparseMatrixCSC (e.g. an operator of
                                      MultigridData.operators, src/Multigrid.jl:538-543) */
} dec_op_kind;

/* A sparse matrix in the layout of the reference's SparseMatrixCSC{Float64, Int32}
 * (src/Multigrid.jl:538-543): host arrays, column pointers and row indices with a selectable base. */
typedef struct dec_csc {
  int32_t m, n;            /* rows, columns */
  int32_t index_base;      /* 1 (Julia) or 0 */
  const int32_t* colptr;   /* n + 1 entries, colptr[0] == index_base */
  const int32_t* rowval;   /* row indices, strictly increasing within each column */
  const double* nzval;     /* values */
} dec_csc;
dec_status dec_op_create(dec_mesh* m, int32_t kind, double shift, dec_dtype dtype, dec_op** out);
/* A DEC_OP_GENERAL operator from a caller's sparse matrix (stored on the device as a slot-major ELL
 * with each row's columns in increasing order, so a row sums in SparseArrays' column order).
 * dec_op_apply, dec_op_shape and dec_op_export_csr work on it. */
dec_status dec_op_create_csc(const dec_csc* a, dec_dtype dtype, dec_op** out);
dec_status dec_op_shape(const dec_op* op, int64_t* rows, int64_t* cols);
/* y = alpha * Op x + beta * y  (beta == 0 overwrites y). */
dec_status dec_op_apply(dec_op* op, const void* x, void* y, double alpha, double beta, void* stream);
/* Residual norms ||b_j - Op x_j||_2 and ||b_j||_2 for nrhs right-hand sides (x, b: device FP64,
 * column-major rows x nrhs; norms, bnorms: host arrays of nrhs doubles, bnorms may be NULL): the
 * convergence test of the reference's multigrid tests, norm(L*u - b) / norm(b)
 * (test/Multigrid.jl:67).  Square FP64 operators only.  Uses device scratch for the per-block
 * partial sums (a deterministic two-stage reduction), allocated per call. */
dec_status dec_op_residual_norms(dec_op* op, const double* x, const double* b, int32_t nrhs, double* norms,
                                 double* bnorms, void* stream);
/* Allocation-free variant of dec_op_residual_norms (no counterpart in the reference).
 * For callers that cannot allocate device memory at the point of the call: an application
 * that hands the device a fixed memory budget up front, a real-time loop that must not enter
 * the allocator, or code running while another thread captures a CUDA graph.  It calls no
 * cudaMalloc / cudaFree: its scratch (the per-block partial sums, then the norms) is a file-scope
 * device array of DEC_RESIDUAL_NOALLOC_SCRATCH_DOUBLES doubles (about 264 KiB) that every GPU
 * which loads the library holds until the process exits.
 *  - nrhs above DEC_RESIDUAL_NOALLOC_MAX_RHS is rejected with DEC_ERR_INVALID_ARG.
 *  - The first call on a device looks up the array's device address (cudaGetSymbolAddress);
 *    make that first call before any stream capture on that device.  The address is kept for
 *    the life of the process: after cudaDeviceReset on a device, do not call it on that device
 *    again.
 *  - All calls share the one array, which keeps the last call's contents (every slot a call
 *    reads it has written first, so nothing needs clearing): calls that overlap on the GPU
 *    (concurrent streams or host threads) race. */
#define DEC_RESIDUAL_NOALLOC_MAX_RHS 64
#define DEC_RESIDUAL_BLOCKS 256 /* blocks of the residual-norm reduction: 2 partial sums each per RHS */
#define DEC_RESIDUAL_NOALLOC_SCRATCH_DOUBLES \
  (2 * DEC_RESIDUAL_BLOCKS * DEC_RESIDUAL_NOALLOC_MAX_RHS + 2 * DEC_RESIDUAL_NOALLOC_MAX_RHS)
dec_status dec_op_residual_norms_noalloc(dec_op* op, const double* x, const double* b, int32_t nrhs,
                                         double* norms, double* bnorms, void* stream);
/* CSR export to host, two-phase: call with rowptr == NULL to get nnz. */
dec_status dec_op_export_csr(const dec_op* op, int64_t* nnz, int32_t* rowptr, int32_t* colind, double* val);
dec_status dec_op_destroy(dec_op* op);

/* ---- geometric multigrid (replaces MultigridData(s, BinarySubdivision(), levels, op, steps;
 *      alg), src/Multigrid.jl:698-797, and multigrid_vcycles / multigrid_wcycles /
 *      full_multigrid, :814-855) --------------------------------------------------------- */
typedef enum dec_smoother {
  DEC_SMOOTH_JACOBI = 0,     /* damped Jacobi, `pre`/`post` sweeps */
  DEC_SMOOTH_CHEBYSHEV = 1,  /* Chebyshev-Jacobi of degree `pre`/`post` */
  DEC_SMOOTH_CG = 2,         /* Krylov.jl cg with itmax = steps (the reference's smoother) */
  DEC_SMOOTH_LEARNED = 3     /* per-vertex MLP correction on the tensor cores (dec_mg_set_smoother_mlp),
                                `pre`/`post` sweeps; Chebyshev-Jacobi is the fallback */
} dec_smoother;

typedef struct dec_mg_options {
  int32_t levels;          /* binary subdivisions above the coarse mesh */
  int32_t center;          /* dec_center of every level's dual complex (reference default: circumcenter) */
  double project_radius;   /* > 0: new vertices are projected onto this sphere (icospheres) */
  double shift;            /* operator A = L + shift * I on every level */
  int32_t smoother;        /* dec_smoother */
  int32_t pre, post;       /* sweeps / degree / CG steps */
  double omega;            /* Jacobi damping */
  double cheb_ratio;       /* Chebyshev interval [lmax / ratio, lmax] */
  int32_t coarse_solver;   /* 0: dense direct FP64 solve on the coarsest level; 1: the smoother;
                              2: exact solve through the coarsest Laplacian's eigendecomposition, which
                              admits a shift per right-hand side (every level then stores the
                              Laplacian, and RHS j solves (L + (shift + c_j) I) u = b; see
                              dec_mg_solve_shifted); Jacobi / Chebyshev smoothers only */
  int32_t precision;       /* 0: FP64 V-cycles; 1: FP32 V-cycles inside FP64 iterative refinement;
                              2: FP16-stored panels (FP32 arithmetic) inside FP64 refinement, each
                              step's residual scaled to unit RMS per RHS (Jacobi / Chebyshev only) */
  int32_t rhs_block;       /* right-hand sides per panel (1, 2, 4, 8, 16, 32; 0 = automatic) */
  int32_t mu;              /* 1 = V-cycle, 2 = W-cycle */
  int32_t inner_cycles;    /* cycles per refinement step of dec_mg_solve (>= 1) */
  int32_t reorder;         /* 1: store each level in a locality (Morton) order internally */
  int32_t coarse_max;      /* > 0: cycles stop at the first level with at most this many vertices
                              (<= 1024) and solve it directly; 0: at the hierarchy's coarsest level */
  double fallback_rho;     /* learned smoother: dec_mg_solve switches to the plain smoother for the
                              rest of the solve when a refinement step reduces the worst relative
                              residual by less than this factor (or it is not finite); that step is
                              undone and redone with the plain smoother */
  int32_t galerkin;        /* 0: DirectMode (every level's operator from its own mesh); 1: GalerkinMode
                              (Multigrid.jl:740-748): only the finest level's, the coarser ones
                              A_{k+1} = R_k A_k P_k (host sparse products in SparseArrays' order);
                              not with coarse_solver 2 */
  int32_t device_loop;     /* 1 (default): dec_mg_solve runs its refinement loop on the device (one graph
                              with a conditional WHILE node); 0: the host drives it, one graph launch
                              per step (profilers that do not follow kernels inside conditional graph
                              nodes see every kernel) */
} dec_mg_options;

typedef struct dec_solve_report {
  int32_t iterations;      /* outer iterations (cycles) run */
  int32_t converged;       /* all right-hand sides reached rtol */
  double max_rel_residual; /* max_j ||b_j - A u_j|| / ||b_j|| at exit (FP64) */
  double seconds;          /* device time of the solve */
  int64_t launches;        /* kernels launched by the solve */
  int32_t rhs_block;       /* panel width used */
  int32_t fallback_iteration; /* learned smoother: refinement step at which the plain smoother took
                                 over, -1 if it did not */
} dec_solve_report;

void dec_mg_default_options(dec_mg_options* o);
dec_status dec_mg_create(const dec_mesh_desc* coarse, const dec_mg_options* opts, dec_mg** out);
dec_status dec_mg_destroy(dec_mg* mg);
/* MultigridData(g, r, p, s) (src/Multigrid.jl:538-546): a hierarchy from the caller's matrices --
 * nlevels square operators, finest first (operators[k] n_k x n_k), nlevels - 1 restrictions
 * (restrictions[k] n_{k+1} x n_k) and prolongations (prolongations[k] n_k x n_{k+1}), and steps[k]
 * smoother steps before and after the coarse correction on level k (NULL: opts->pre / opts->post on
 * every level).  The cycle is _multigrid_μ_cycle (src/Multigrid.jl:857-872): smooth, r = b - A u,
 * r_c = R r, recurse (twice for μ = 2), u += P z, smooth, with each restriction and prolongation a
 * sparse product summed in SparseArrays' column order.  Smoothers: DEC_SMOOTH_CG (the reference's
 * Krylov cg, FP64), Jacobi and Chebyshev (every operator needs a nonzero diagonal; any precision);
 * coarse_solver 0 (dense) or 1.  opts->levels, center, project_radius, shift, galerkin and reorder
 * are not used: the operators are taken as given, in the caller's numbering.  Levels have no mesh
 * (dec_mg_level_mesh fails; dec_mg_level_info reports ne = nt = 0). */
dec_status dec_mg_create_from_csc(int32_t nlevels, const dec_csc* operators, const dec_csc* restrictions,
                                  const dec_csc* prolongations, const int32_t* steps, const dec_mg_options* opts,
                                  dec_mg** out);
/* The steps field of MultigridData (src/Multigrid.jl:542, :858-871): smoother steps before and after the
 * coarse correction on each level (steps[k] for level k, finest first, as many as the hierarchy has
 * levels; each in [0, 16]); NULL restores opts->pre / opts->post.  Any hierarchy, any smoother. */
dec_status dec_mg_set_level_steps(dec_mg* mg, const int32_t* steps);
/* level 0 = finest. */
dec_status dec_mg_level_info(const dec_mg* mg, int32_t level, int64_t* nv, int64_t* ne, int64_t* nt,
                             double* lmax);
dec_status dec_mg_level_mesh(const dec_mg* mg, int32_t level, const dec_mesh** out);
dec_status dec_mg_level_op(const dec_mg* mg, int32_t level, const dec_op** out);
/* u (in/out) and b: device FP64, column-major nv x nrhs (one contiguous vector per RHS). */
dec_status dec_mg_cycles(dec_mg* mg, double* u, const double* b, int32_t nrhs, int32_t cycles, void* stream);
/* full_multigrid(b, md, cycles, alg, μ) (Multigrid.jl:826-855): b restricted to the coarsest
 * level, then on the way up each level's solution is prolonged as the next level's initial guess
 * followed by `cycles` μ-cycles there; u (output) gets the finest level's result.  FP64. */
dec_status dec_mg_full_multigrid(dec_mg* mg, double* u, const double* b, int32_t nrhs, int32_t cycles,
                                 void* stream);
dec_status dec_mg_solve(dec_mg* mg, double* u, const double* b, int32_t nrhs, double rtol,
                        int32_t max_iters, dec_solve_report* report, void* stream);
/* dec_mg_solve from u = 0 (multigrid_vcycles(zeros(n), b, md, cycles), src/Multigrid.jl:814, as the
 * refined solve): u is output only and is not read.  The first refinement step's residual is b
 * itself, so it costs one pass over b instead of the FP64 update and residual passes (the same
 * iterates bit for bit). */
dec_status dec_mg_solve_from_zero(dec_mg* mg, double* u, const double* b, int32_t nrhs, double rtol,
                                  int32_t max_iters, dec_solve_report* report, void* stream);
/* Same solve with host u / b (pinned or pageable); copies are part of the call.  With
 * use_initial_guess = 0 the solve starts from u = 0 and u_host is output only (not copied in). */
dec_status dec_mg_solve_host(dec_mg* mg, double* u_host, const double* b_host, int32_t nrhs, double rtol,
                             int32_t max_iters, int32_t use_initial_guess, dec_solve_report* report,
                             void* stream);

/* Pipelined form of dec_mg_solve_host (Jacobi / Chebyshev smoothers): submit enqueues the copy of
 * b_host (and u_host) to the device, the solve and the copy of u back on the hierarchy's own
 * streams and returns a ticket at once; wait blocks until u_host holds the ticket's solution and
 * returns its report (seconds: first copy in to last copy out).  Three tickets may be in flight,
 * so the copies of neighbouring solves overlap each solve's compute; the host buffers must stay
 * valid (and, for the overlap, pinned) until the wait.  Other calls on the hierarchy first wait
 * for the pipeline. */
dec_status dec_mg_solve_host_submit(dec_mg* mg, double* u_host, const double* b_host, int32_t nrhs, double rtol,
                                    int32_t max_iters, int32_t use_initial_guess, uint64_t* ticket);
dec_status dec_mg_solve_host_wait(dec_mg* mg, uint64_t ticket, dec_solve_report* report);

/* dec_mg_solve with a shift per right-hand side (coarse_solver 2): RHS j solves
 * (L + (shift + shifts[j]) I) u_j = b_j; shifts is a host array of nrhs values (total shifts must
 * be positive). */
dec_status dec_mg_solve_shifted(dec_mg* mg, double* u, const double* b, int32_t nrhs, const double* shifts,
                                double rtol, int32_t max_iters, dec_solve_report* report, void* stream);

/* ---- batched solves over several hierarchies (meshes of uneven sizes; no counterpart in the
 *      reference): the whole solve of all groups is one CUDA graph -- a concurrent branch per group
 *      (FP32 or FP64 V-cycles per each hierarchy's options, FP64 refinement) and the refinement loop
 *      as a conditional WHILE node that a residual-test kernel over all groups sets, so a batch is one
 *      graph launch and one read-back of the loop state.  The graph holds the caller's u / rhs
 *      pointers: it is reused while a call passes the same buffers and sizes, and rebuilt otherwise.
 *      Groups use the Jacobi or Chebyshev smoother.
 * ------------------------------------------------------------------------------------------ */
/* The hierarchies are not owned and must outlive the batch. */
dec_status dec_batch_create(dec_mg* const* groups, int32_t ngroups, dec_batch** out);
dec_status dec_batch_destroy(dec_batch* batch);
/* Runs dec_mg_autotune on every group for its nrhs (panel width per group). */
dec_status dec_batch_autotune(dec_batch* batch, const int32_t* nrhs, int32_t reps, void* stream);
/* Group g: u[g] (in/out initial guess) and rhs[g] device FP64 column-major n_g x nrhs[g];
 * shifts[g] host per-RHS shifts (coarse_solver 2 groups) or NULL (shifts itself may be NULL).
 * Every group runs until all groups reach rtol or max_iters refinement steps; reports[g] gives the
 * step at which group g converged, total the whole batch (device seconds, kernels launched). */
dec_status dec_batch_solve(dec_batch* batch, double* const* u, const double* const* rhs, const int32_t* nrhs,
                           const double* const* shifts, double rtol, int32_t max_iters,
                           dec_solve_report* reports, dec_solve_report* total, void* stream);
/* Algorithmic bytes of the captured batch graph run for `iterations` refinement steps (total.iterations
 * of the last dec_batch_solve): every kernel's compulsory reads and writes, the caller vectors
 * into and out of the panels included; errors if no solve has been captured. */
dec_status dec_batch_traffic(const dec_batch* batch, int32_t iterations, double* bytes);

/* Learned smoother for DEC_SMOOTH_LEARNED: the hierarchy reads the network's weights at every
 * cycle (the network must outlive its use; retraining takes effect at the next cycle).  NULL
 * detaches it. */
dec_status dec_mg_set_smoother_mlp(dec_mg* mg, const dec_mlp* mlp);

/* ---- learned smoother network (no counterpart in the reference): per-vertex MLP 16 -> 64 -> 64
 *      -> 1 with ReLU; parameters flat FP32 W1[64][16] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3;
 *      inference with W1, W2, the features and the first hidden layer in BF16, FP32 accumulation.
 *      Features of vertex i from the residual field r and operator row i (Laplacian/Helmholtz):
 *      r_i/s, six neighbour residuals r_j/s, six couplings a_ij/a_ii (column order, zero-padded),
 *      1 - sum_j |a_ij|/a_ii, valence/6, 0; s = max |r| over the 1-ring.  The smoother applies
 *      x_i += (s / a_ii) y_i. ---------------------------------------------------------------- */
#define DEC_MLP_NPARAM 5313
/* Xavier-uniform weights (splitmix64 stream of `seed`), zero biases, Adam state zero. */
dec_status dec_mlp_create(uint64_t seed, dec_mlp** out);
dec_status dec_mlp_destroy(dec_mlp* mlp);
/* Host copies of the FP32 master parameters (DEC_MLP_NPARAM floats); either pointer may be NULL. */
dec_status dec_mlp_get_params(const dec_mlp* mlp, float* params);
dec_status dec_mlp_set_params(dec_mlp* mlp, const float* params);
dec_status dec_mlp_step(const dec_mlp* mlp, int64_t* step);
/* y[n] = MLP(x[n][16]) on device memory; tensor_cores = 0 evaluates on the CUDA cores, 1 with
 * mma.sync, 2 with tcgen05 / TMEM (this one synchronises the stream and returns DEC_ERR_TIMEOUT if
 * a bounded wait for the tensor core ran out). */
dec_status dec_mlp_eval(dec_mlp* mlp, const float* x, int64_t n, float* y, int32_t tensor_cores, void* stream);
/* Kernel engine of the learned smoothing step: 1 (the default) = tcgen05.mma with TMEM accumulators
 * (one 1024-thread CTA per SM, eight chains of 128-sample tiles); 0 = mma.sync (m16n8k16, warp tiles
 * of 32 samples). */
dec_status dec_mlp_set_engine(dec_mlp* mlp, int32_t engine);
/* grad[DEC_MLP_NPARAM] (device) = sum_q dy[q] d MLP(x_q) / d params. */
dec_status dec_mlp_grad(dec_mlp* mlp, const float* x, const float* dy, int64_t n, float* grad, void* stream);
/* Features (n*S x 16) and the correction scales s / a_ii (n*S) of S residual fields r (device,
 * column-major n x S) on an FP64 Laplacian / Helmholtz operator. */
dec_status dec_mlp_features(const dec_op* op, const double* r, int32_t S, float* features, float* scales,
                            void* stream);
/* Energy-norm loss of one smoothing step on S residual fields, and its full parameter gradient
 * (device, may be NULL):
 *   L = (1/S) sum_s (d_s' M A d_s - 2 d_s' M r_s) / n_s,  d = (s/a_ii) MLP(features),
 *   M = diag(star0), n_s = sum_i star0_i r_si^2 / a_ii. */
dec_status dec_mlp_loss_grad(dec_mlp* mlp, dec_op* op, const double* r, int32_t S, double* loss, float* grad,
                             void* stream);
/* `steps` Adam steps (lr; beta 0.9 / 0.999, eps 1e-8) on S residual fields; each step's gradient
 * comes from `batch` vertex samples (all of them when n*S <= batch, else drawn with replacement
 * from the stream of (seed, step)).  losses (host, may be NULL) receives each step's loss before
 * its update and then synchronises the stream every step. */
dec_status dec_mlp_train(dec_mlp* mlp, dec_op* op, const double* r, int32_t S, int32_t steps, double lr,
                         int64_t batch, uint64_t seed, double* losses, void* stream);
/* Checkpoint of parameters, Adam moments and step counter ("DECMLP01", version 1, CRC-32). */
dec_status dec_mlp_save(const dec_mlp* mlp, const char* path);
dec_status dec_mlp_load(dec_mlp* mlp, const char* path);

/* ---- profiling (no counterpart in the reference; its benchmarks print timings only,
 *      test/Benchmarks.jl:128-140) ------------------------------------------------------ */
typedef enum dec_mg_kernel {
  DEC_KERNEL_SWEEP = 0,     /* Chebyshev / Jacobi smoothing sweep */
  DEC_KERNEL_RESIDUAL = 1,  /* FP64 residual with norms */
  DEC_KERNEL_RESTRICT = 2,
  DEC_KERNEL_PROLONG = 3,
  DEC_KERNEL_MLP = 4,       /* learned smoothing step (the MLP kernel alone; 10,368 FLOP per sample,
                               10,240 of them on the tensor cores) */
  DEC_KERNEL_SWEEP_PAIR = 5, /* two Chebyshev steps as one temporal-blocked pass (FP32 panels of 16 or more,
                               rows of 6 slots); bytes: the pair's one-pass minimum (operator, x, b and the
                               result once) */
  DEC_KERNEL_SWEEP_PROLONGED0 = 6, /* first post-smoothing step from x = P z, the prolongation fused in
                                      (reads the coarse correction of level + 1; rows of 6 slots) */
  DEC_KERNEL_SWEEP_PROLONGED1 = 7  /* second Chebyshev step with its previous iterate P z formed the same
                                      way */
} dec_mg_kernel;
/* Times `reps` back-to-back launches of one V-cycle kernel at `level`, configured as in a solve
 * of `nrhs` right-hand sides, with CUDA events on `stream`.  Returns the mean milliseconds per
 * launch and the algorithmic bytes one launch moves (every array read or written once). */
dec_status dec_mg_time_kernel(dec_mg* mg, int32_t kernel, int32_t level, int32_t nrhs, int32_t reps,
                              void* stream, double* ms_per_launch, double* bytes_per_launch);
/* Algorithmic bytes of a whole dec_mg_solve / dec_mg_solve_from_zero (from_zero = 1) of nrhs
 * right-hand sides that ran `iterations` refinement steps (the report's iterations), with the
 * refinement loop on the device (Jacobi / Chebyshev smoothers): every kernel's streamed arrays
 * read or written once and each gathered vector once, summed over the solve graph's kernels, plus
 * the layout changes of b and u.  Captures the solve graph if no solve of this shape ran yet. */
dec_status dec_mg_solve_traffic(dec_mg* mg, int32_t nrhs, int32_t from_zero, int32_t iterations, double* bytes);
/* ---- the autotuner's table (no counterpart in the reference): the variant chosen per (kernel,
 *      dtype, shape, size bucket), process-wide, consulted when a kernel is launched or a solve graph
 *      captured.  Keys read "<kernel>/<dtype>/<shape>/n<floor(log2 size)>":
 *        ell/f32|f64/W7/n<rows>          rows per thread of the ELL apply (1, 2 or 4; 1 by default)
 *        sweep/f32/K<width>/W<slots>/n<rows>  lanes per row of the FP32 smoothing sweep: the vector
 *                                        width 4 (default) or 2 (twice the lanes on a row)
 *      Every variant computes the same bits; only the time differs. ------------------------------ */
/* Times each rows-per-thread variant of the operator's apply (operators stored as rows of 7 slots:
 * the Laplacian / Helmholtz operators of triangle meshes, a caller matrix of that width) on scratch
 * vectors, records the fastest in the table and returns it in *choice (0: the kernel has no variants). */
dec_status dec_op_autotune(dec_op* op, int32_t reps, void* stream, int32_t* choice);
dec_status dec_tune_set(const char* key, int32_t value);
/* *found = 0 (and *value untouched) when the key was never measured or set. */
dec_status dec_tune_get(const char* key, int32_t* value, int32_t* found);
dec_status dec_tune_clear(void);
/* The table as JSON ({"format": "dec_b200 tuning table", "version": 1, "device": ..., "entries": {...}});
 * loading merges a saved table into the current one (its entries win) and returns how many it read. */
dec_status dec_tune_save(const char* path);
dec_status dec_tune_load(const char* path, int32_t* entries);
/* Times each candidate panel width on one V-cycle and keeps the fastest for `nrhs` right-hand
 * sides (used when rhs_block = 0); for FP32 V-cycles on panels of 8 or more it then times the sweep's
 * lanes-per-row variants on the same cycle and records the winner in the tuning table for every
 * level.  Returns the chosen width. */
dec_status dec_mg_autotune(dec_mg* mg, int32_t nrhs, int32_t reps, void* stream, int32_t* rhs_block);

#ifdef __cplusplus
}
#endif
#endif /* DEC_B200_H */
