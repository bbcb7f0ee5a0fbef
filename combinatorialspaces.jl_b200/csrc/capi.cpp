// extern "C" entry points of libdec_b200.so (declared in include/dec_b200.h).  Each one turns
// exceptions from the implementation into a dec_status and a thread-local message.
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>

#include "mesh.cuh"
#include "mg.cuh"
#include "ops.cuh"
#include "tune.cuh"

// Implementations (wedge.cu, ops.cu).
dec_wedge_plan* wedge_plan_create_impl(dec_mesh* mh, int kind, int da, int db, dec_dtype dt);
void wedge_apply_impl(dec_wedge_plan* P, const void* a, const void* b, void* out, int count, void* stream);
int wedge_autotune_impl(dec_wedge_plan* P, int count, int reps, void* stream);
void wedge_plan_destroy_impl(dec_wedge_plan* P);
void wedge_lengths_impl(const dec_wedge_plan* P, int64_t* la, int64_t* lb, int64_t* lo);
void c_wedge_apply_impl(int j, int k, int64_t n, const int32_t* p, const void* c, dec_dtype dt, const void* a,
                        const void* b, void* res, int index_base, void* stream);
dec_op* op_create_impl(dec_mesh* mh, int kind, double shift, dec_dtype dt);
void op_apply_impl(dec_op* op, const void* x, void* y, double alpha, double beta, void* stream);
void op_export_csr_impl(const dec_op* op, int64_t* nnz, int32_t* rowptr, int32_t* colind, double* val);
void hodge_diag_impl(const dec_mesh* mh, int k, int inverse, dec_dtype dt, void* out, void* stream);
void op_residual_norms_impl(dec_op* op, const double* x, const double* b, int nrhs, double* norms, double* bnorms,
                            void* stream);
dec_mlp* mlp_create_impl(uint64_t seed);
void mlp_destroy_impl(dec_mlp* m);
void mlp_params_impl(dec_mlp* m, float* out, const float* in);
int64_t mlp_step_impl(const dec_mlp* m);
void mlp_eval_impl(dec_mlp* m, const float* x, int64_t n, float* y, int tensor_cores, void* stream);
void mlp_grad_impl(dec_mlp* m, const float* x, const float* dy, int64_t n, float* grad, void* stream);
void mlp_features_impl(const dec_op* op, const double* r, int S, float* feat, float* dscale, void* stream);
void mlp_loss_grad_impl(dec_mlp* m, dec_op* op, const double* r, int S, double* loss, float* grad, void* stream);
void mlp_train_impl(dec_mlp* m, dec_op* op, const double* r, int S, int steps, double lr, int64_t batch,
                    uint64_t seed, double* losses, void* stream);
void mlp_save_impl(const dec_mlp* m, const char* path);
void mlp_set_engine_impl(dec_mlp* m, int engine);
void mlp_load_impl(dec_mlp* m, const char* path);
void op_residual_norms_noalloc_impl(dec_op* op, const double* x, const double* b, int nrhs, double* norms,
                                    double* bnorms, void* stream);
dec_op* op_create_csc_impl(const dec_csc* a, dec_dtype dt);
int op_autotune_impl(dec_op* op, int reps, void* stream);

namespace {
thread_local std::string g_err;

template <class F>
dec_status guard(F&& f) {
  try {
    f();
    g_err.clear();
    return DEC_OK;
  } catch (const decb::Error& e) {
    g_err = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return DEC_ERR_OOM;
  } catch (const std::exception& e) {
    g_err = e.what();
    return DEC_ERR_INVALID_ARG;
  }
}
}  // namespace

extern "C" {

const char* dec_last_error(void) { return g_err.c_str(); }
int32_t dec_version(void) { return 1; }

dec_status dec_mesh_create(const dec_mesh_desc* desc, dec_mesh** out) {
  return guard([&] {
    decb::require(desc && out, "dec_mesh_create: null argument");
    *out = nullptr;
    auto* m = new dec_mesh();
    try {
      m->m.build(*desc);
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
  });
}

dec_status dec_mesh_destroy(dec_mesh* m) {
  return guard([&] { delete m; });
}

dec_status dec_mesh_counts(const dec_mesh* m, int64_t* nv, int64_t* ne, int64_t* nt) {
  return guard([&] {
    decb::require(m != nullptr, "dec_mesh_counts: null mesh");
    if (nv) *nv = m->m.nv;
    if (ne) *ne = m->m.ne;
    if (nt) *nt = m->m.nt;
  });
}

dec_status dec_mesh_orientation(const dec_mesh* m, int8_t* eo, int8_t* to) {
  return guard([&] {
    decb::require(m != nullptr, "dec_mesh_orientation: null mesh");
    m->m.ensure_host();
    if (eo) std::memcpy(eo, m->m.h_eo.data(), m->m.h_eo.size());
    if (to) std::memcpy(to, m->m.h_to.data(), m->m.h_to.size());
  });
}

dec_status dec_mesh_geometry(const dec_mesh* mh, int32_t which, double* out, int64_t len) {
  return guard([&] {
    decb::require(mh != nullptr && out != nullptr, "dec_mesh_geometry: null argument");
    const decb::Mesh& m = mh->m;
    std::vector<double> v;
    switch (which) {
      case DEC_GEOM_LENGTH: v = m.length.download(); break;
      case DEC_GEOM_AREA: v = m.area.download(); break;
      case DEC_GEOM_DUAL_AREA: v = m.dual_area.download(); break;
      case DEC_GEOM_DUAL_LENGTH_TE: v = m.dual_len_te.download(); break;
      case DEC_GEOM_DUAL_POINT: {
        m.ensure_host();
        auto tc = m.tri_center.download();
        v.resize(3 * ((size_t)m.nv + m.ne + m.nt));
        std::copy(m.h_pts.begin(), m.h_pts.end(), v.begin());
        for (int e = 0; e < m.ne; ++e)
          for (int k = 0; k < 3; ++k)
            v[3 * ((size_t)m.nv + e) + k] = (m.h_pts[3 * (size_t)m.h_ev0[e] + k] + m.h_pts[3 * (size_t)m.h_ev1[e] + k]) / 2;
        std::copy(tc.begin(), tc.end(), v.begin() + 3 * ((size_t)m.nv + m.ne));
        break;
      }
      default: throw decb::Error(DEC_ERR_INVALID_ARG, "dec_mesh_geometry: unknown array");
    }
    decb::require((int64_t)v.size() == len, "dec_mesh_geometry: length mismatch (expected " + std::to_string(v.size()) + ")");
    std::copy(v.begin(), v.end(), out);
  });
}

dec_status dec_hodge_diag(const dec_mesh* m, int32_t k, int32_t inverse, dec_dtype dt, void* out, void* stream) {
  return guard([&] { hodge_diag_impl(m, k, inverse, dt, out, stream); });
}

dec_status dec_wedge_plan_create(dec_mesh* m, int32_t kind, int32_t da, int32_t db, dec_dtype dt,
                                 dec_wedge_plan** out) {
  return guard([&] {
    decb::require(out != nullptr, "dec_wedge_plan_create: null output");
    *out = nullptr;
    *out = wedge_plan_create_impl(m, kind, da, db, dt);
  });
}

dec_status dec_wedge_apply(dec_wedge_plan* p, const void* a, const void* b, void* out, void* stream) {
  return guard([&] { wedge_apply_impl(p, a, b, out, 1, stream); });
}

dec_status dec_wedge_apply_batched(dec_wedge_plan* p, const void* a, const void* b, void* out, int32_t count,
                                   void* stream) {
  return guard([&] { wedge_apply_impl(p, a, b, out, count, stream); });
}

dec_status dec_wedge_autotune(dec_wedge_plan* p, int32_t count, int32_t reps, void* stream, int32_t* choice) {
  return guard([&] {
    const int c = wedge_autotune_impl(p, count, reps, stream);
    if (choice) *choice = c;
  });
}

dec_status dec_c_wedge_apply(int32_t j, int32_t k, int64_t n_out, const int32_t* p, const void* c, dec_dtype dtype,
                             const void* a, const void* b, void* res, int32_t index_base, void* stream) {
  return guard([&] { c_wedge_apply_impl(j, k, n_out, p, c, dtype, a, b, res, index_base, stream); });
}

dec_status dec_wedge_lengths(const dec_wedge_plan* p, int64_t* la, int64_t* lb, int64_t* lo) {
  return guard([&] { wedge_lengths_impl(p, la, lb, lo); });
}

dec_status dec_wedge_plan_destroy(dec_wedge_plan* p) {
  return guard([&] { wedge_plan_destroy_impl(p); });
}

dec_status dec_op_create(dec_mesh* m, int32_t kind, double shift, dec_dtype dt, dec_op** out) {
  return guard([&] {
    decb::require(out != nullptr, "dec_op_create: null output");
    *out = nullptr;
    *out = op_create_impl(m, kind, shift, dt);
  });
}

dec_status dec_op_create_csc(const dec_csc* a, dec_dtype dt, dec_op** out) {
  return guard([&] {
    decb::require(out != nullptr, "dec_op_create_csc: null output");
    *out = nullptr;
    *out = op_create_csc_impl(a, dt);
  });
}

dec_status dec_op_shape(const dec_op* op, int64_t* rows, int64_t* cols) {
  return guard([&] {
    decb::require(op != nullptr, "dec_op_shape: null operator");
    if (rows) *rows = op->rows;
    if (cols) *cols = op->cols;
  });
}

dec_status dec_op_apply(dec_op* op, const void* x, void* y, double alpha, double beta, void* stream) {
  return guard([&] { op_apply_impl(op, x, y, alpha, beta, stream); });
}

dec_status dec_op_residual_norms(dec_op* op, const double* x, const double* b, int32_t nrhs, double* norms,
                                 double* bnorms, void* stream) {
  return guard([&] { op_residual_norms_impl(op, x, b, nrhs, norms, bnorms, stream); });
}

dec_status dec_op_residual_norms_noalloc(dec_op* op, const double* x, const double* b, int32_t nrhs,
                                         double* norms, double* bnorms, void* stream) {
  return guard([&] { op_residual_norms_noalloc_impl(op, x, b, nrhs, norms, bnorms, stream); });
}

dec_status dec_op_export_csr(const dec_op* op, int64_t* nnz, int32_t* rowptr, int32_t* colind, double* val) {
  return guard([&] { op_export_csr_impl(op, nnz, rowptr, colind, val); });
}

dec_status dec_op_destroy(dec_op* op) {
  return guard([&] { delete op; });
}

void dec_mg_default_options(dec_mg_options* o) {
  if (o) decb::mg_default_options(*o);
}

dec_status dec_mg_create(const dec_mesh_desc* coarse, const dec_mg_options* opts, dec_mg** out) {
  return guard([&] {
    decb::require(coarse && opts && out, "dec_mg_create: null argument");
    *out = nullptr;
    *out = decb::mg_create(*coarse, *opts);
  });
}

dec_status dec_mg_create_from_csc(int32_t nlevels, const dec_csc* operators, const dec_csc* restrictions,
                                  const dec_csc* prolongations, const int32_t* steps, const dec_mg_options* opts,
                                  dec_mg** out) {
  return guard([&] {
    decb::require(opts && out, "dec_mg_create_from_csc: null argument");
    *out = nullptr;
    *out = decb::mg_create_from_csc(nlevels, operators, restrictions, prolongations, steps, *opts);
  });
}

dec_status dec_mg_set_level_steps(dec_mg* mg, const int32_t* steps) {
  return guard([&] { decb::mg_set_level_steps(mg, steps); });
}

dec_status dec_mg_destroy(dec_mg* mg) {
  return guard([&] { decb::mg_destroy(mg); });
}

dec_status dec_mg_level_info(const dec_mg* mg, int32_t level, int64_t* nv, int64_t* ne, int64_t* nt, double* lmax) {
  return guard([&] { decb::mg_level_info(mg, level, nv, ne, nt, lmax); });
}

dec_status dec_mg_level_mesh(const dec_mg* mg, int32_t level, const dec_mesh** out) {
  return guard([&] { *out = decb::mg_level_mesh(mg, level); });
}

dec_status dec_mg_level_op(const dec_mg* mg, int32_t level, const dec_op** out) {
  return guard([&] { *out = decb::mg_level_op(mg, level); });
}

dec_status dec_mg_cycles(dec_mg* mg, double* u, const double* b, int32_t nrhs, int32_t cycles, void* stream) {
  return guard([&] { decb::mg_cycles(mg, u, b, nrhs, cycles, stream); });
}

dec_status dec_mg_full_multigrid(dec_mg* mg, double* u, const double* b, int32_t nrhs, int32_t cycles, void* stream) {
  return guard([&] { decb::mg_full_multigrid(mg, u, b, nrhs, cycles, stream); });
}

dec_status dec_mg_solve(dec_mg* mg, double* u, const double* b, int32_t nrhs, double rtol, int32_t max_iters,
                        dec_solve_report* rep, void* stream) {
  dec_status st = DEC_OK;
  dec_status g = guard([&] { st = decb::mg_solve(mg, u, b, nrhs, rtol, max_iters, rep, stream, false, true); });
  return g != DEC_OK ? g : st;
}

dec_status dec_mg_solve_from_zero(dec_mg* mg, double* u, const double* b, int32_t nrhs, double rtol,
                                  int32_t max_iters, dec_solve_report* rep, void* stream) {
  dec_status st = DEC_OK;
  dec_status g = guard([&] { st = decb::mg_solve(mg, u, b, nrhs, rtol, max_iters, rep, stream, false, false); });
  return g != DEC_OK ? g : st;
}

dec_status dec_mg_solve_host(dec_mg* mg, double* u, const double* b, int32_t nrhs, double rtol, int32_t max_iters,
                             int32_t use_initial_guess, dec_solve_report* rep, void* stream) {
  dec_status st = DEC_OK;
  dec_status g = guard(
      [&] { st = decb::mg_solve(mg, u, b, nrhs, rtol, max_iters, rep, stream, true, use_initial_guess != 0); });
  return g != DEC_OK ? g : st;
}

dec_status dec_mg_solve_host_submit(dec_mg* mg, double* u, const double* b, int32_t nrhs, double rtol,
                                    int32_t max_iters, int32_t use_initial_guess, uint64_t* ticket) {
  return guard([&] {
    decb::require(ticket != nullptr, "dec_mg_solve_host_submit: null ticket");
    *ticket = decb::mg_solve_submit(mg, u, b, nrhs, rtol, max_iters, use_initial_guess != 0);
  });
}

dec_status dec_mg_solve_host_wait(dec_mg* mg, uint64_t ticket, dec_solve_report* rep) {
  dec_status st = DEC_OK;
  dec_status g = guard([&] { st = decb::mg_solve_wait(mg, ticket, rep); });
  return g != DEC_OK ? g : st;
}

dec_status dec_mg_time_kernel(dec_mg* mg, int32_t kernel, int32_t level, int32_t nrhs, int32_t reps, void* stream,
                              double* ms, double* bytes) {
  return guard([&] { decb::mg_time_kernel(mg, kernel, level, nrhs, reps, stream, ms, bytes); });
}

dec_status dec_mg_solve_traffic(dec_mg* mg, int32_t nrhs, int32_t from_zero, int32_t iterations, double* bytes) {
  return guard([&] {
    double b = decb::mg_solve_traffic(mg, nrhs, from_zero, iterations);
    if (bytes) *bytes = b;
  });
}

dec_status dec_op_autotune(dec_op* op, int32_t reps, void* stream, int32_t* choice) {
  return guard([&] {
    int c = op_autotune_impl(op, reps, stream);
    if (choice) *choice = c;
  });
}

dec_status dec_tune_set(const char* key, int32_t value) {
  return guard([&] {
    decb::require(key != nullptr && key[0] != 0, "dec_tune_set: empty key");
    decb::tune_set(key, value);
  });
}

dec_status dec_tune_get(const char* key, int32_t* value, int32_t* found) {
  return guard([&] {
    decb::require(key != nullptr && value != nullptr && found != nullptr, "dec_tune_get: null argument");
    constexpr int kMissing = -2147483647 - 1;
    const int v = decb::tune_get(key, kMissing);
    *found = v != kMissing;
    if (*found) *value = v;
  });
}

dec_status dec_tune_clear(void) {
  return guard([&] { decb::tune_clear(); });
}

dec_status dec_tune_save(const char* path) {
  return guard([&] {
    decb::require(path != nullptr, "dec_tune_save: null path");
    decb::tune_save(path);
  });
}

dec_status dec_tune_load(const char* path, int32_t* entries) {
  return guard([&] {
    decb::require(path != nullptr, "dec_tune_load: null path");
    const int n = decb::tune_load(path);
    if (entries) *entries = n;
  });
}

dec_status dec_mg_autotune(dec_mg* mg, int32_t nrhs, int32_t reps, void* stream, int32_t* rhs_block) {
  return guard([&] {
    int k = decb::mg_autotune(mg, nrhs, reps, stream);
    if (rhs_block) *rhs_block = k;
  });
}

dec_status dec_mg_solve_shifted(dec_mg* mg, double* u, const double* b, int32_t nrhs, const double* shifts,
                                double rtol, int32_t max_iters, dec_solve_report* rep, void* stream) {
  dec_status st = DEC_OK;
  dec_status g = guard([&] {
    decb::require(shifts != nullptr, "dec_mg_solve_shifted: null shifts");
    st = decb::mg_solve(mg, u, b, nrhs, rtol, max_iters, rep, stream, false, true, shifts);
  });
  return g != DEC_OK ? g : st;
}

dec_status dec_batch_create(dec_mg* const* groups, int32_t ngroups, dec_batch** out) {
  return guard([&] {
    decb::require(out != nullptr, "dec_batch_create: null argument");
    *out = nullptr;
    *out = decb::batch_create(groups, ngroups);
  });
}

dec_status dec_batch_destroy(dec_batch* batch) {
  return guard([&] { decb::batch_destroy(batch); });
}

dec_status dec_batch_autotune(dec_batch* batch, const int32_t* nrhs, int32_t reps, void* stream) {
  return guard([&] { decb::batch_autotune(batch, nrhs, reps, stream); });
}

dec_status dec_batch_traffic(const dec_batch* batch, int32_t iterations, double* bytes) {
  return guard([&] {
    decb::require(bytes != nullptr, "batch: null output");
    *bytes = decb::batch_traffic(batch, iterations);
  });
}

dec_status dec_batch_solve(dec_batch* batch, double* const* u, const double* const* rhs, const int32_t* nrhs,
                           const double* const* shifts, double rtol, int32_t max_iters, dec_solve_report* reports,
                           dec_solve_report* total, void* stream) {
  dec_status st = DEC_OK;
  dec_status g = guard(
      [&] { st = decb::batch_solve(batch, u, rhs, nrhs, shifts, rtol, max_iters, reports, total, stream); });
  return g != DEC_OK ? g : st;
}

dec_status dec_mg_set_smoother_mlp(dec_mg* mg, const dec_mlp* mlp) {
  return guard([&] { decb::mg_set_smoother_mlp(mg, mlp); });
}

dec_status dec_mlp_create(uint64_t seed, dec_mlp** out) {
  return guard([&] {
    decb::require(out != nullptr, "dec_mlp_create: null argument");
    *out = nullptr;
    *out = mlp_create_impl(seed);
  });
}

dec_status dec_mlp_destroy(dec_mlp* mlp) {
  return guard([&] { mlp_destroy_impl(mlp); });
}

dec_status dec_mlp_get_params(const dec_mlp* mlp, float* params) {
  return guard([&] { mlp_params_impl(const_cast<dec_mlp*>(mlp), params, nullptr); });
}

dec_status dec_mlp_set_params(dec_mlp* mlp, const float* params) {
  return guard([&] { mlp_params_impl(mlp, nullptr, params); });
}

dec_status dec_mlp_step(const dec_mlp* mlp, int64_t* step) {
  return guard([&] {
    decb::require(step != nullptr, "dec_mlp_step: null argument");
    *step = mlp_step_impl(mlp);
  });
}

dec_status dec_mlp_eval(dec_mlp* mlp, const float* x, int64_t n, float* y, int32_t tensor_cores, void* stream) {
  return guard([&] { mlp_eval_impl(mlp, x, n, y, tensor_cores, stream); });
}

dec_status dec_mlp_grad(dec_mlp* mlp, const float* x, const float* dy, int64_t n, float* grad, void* stream) {
  return guard([&] { mlp_grad_impl(mlp, x, dy, n, grad, stream); });
}

dec_status dec_mlp_features(const dec_op* op, const double* r, int32_t S, float* features, float* scales,
                            void* stream) {
  return guard([&] { mlp_features_impl(op, r, S, features, scales, stream); });
}

dec_status dec_mlp_loss_grad(dec_mlp* mlp, dec_op* op, const double* r, int32_t S, double* loss, float* grad,
                             void* stream) {
  return guard([&] { mlp_loss_grad_impl(mlp, op, r, S, loss, grad, stream); });
}

dec_status dec_mlp_train(dec_mlp* mlp, dec_op* op, const double* r, int32_t S, int32_t steps, double lr,
                         int64_t batch, uint64_t seed, double* losses, void* stream) {
  return guard([&] { mlp_train_impl(mlp, op, r, S, steps, lr, batch, seed, losses, stream); });
}

dec_status dec_mlp_set_engine(dec_mlp* mlp, int32_t engine) {
  return guard([&] { mlp_set_engine_impl(mlp, engine); });
}

dec_status dec_mlp_save(const dec_mlp* mlp, const char* path) {
  return guard([&] { mlp_save_impl(mlp, path); });
}

dec_status dec_mlp_load(dec_mlp* mlp, const char* path) {
  return guard([&] { mlp_load_impl(mlp, path); });
}

}  // extern "C"
