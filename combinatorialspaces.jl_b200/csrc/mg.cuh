// Geometric multigrid over binary-subdivision hierarchies (declarations for the C ABI).
#pragma once
#include "mesh.cuh"
#include "ops.cuh"

namespace decb {
void mg_default_options(dec_mg_options& o);
dec_mg* mg_create(const dec_mesh_desc& coarse, const dec_mg_options& opts);
dec_mg* mg_create_from_csc(int nl, const dec_csc* ops, const dec_csc* rs, const dec_csc* ps, const int* steps,
                           const dec_mg_options& o);
void mg_set_level_steps(dec_mg* mg, const int* steps);
void mg_destroy(dec_mg* mg);
void mg_level_info(const dec_mg* mg, int level, int64_t* nv, int64_t* ne, int64_t* nt, double* lmax);
const dec_mesh* mg_level_mesh(const dec_mg* mg, int level);
const dec_op* mg_level_op(const dec_mg* mg, int level);
void mg_cycles(dec_mg* mg, double* u, const double* b, int nrhs, int cycles, void* stream);
void mg_full_multigrid(dec_mg* mg, double* u, const double* b, int nrhs, int cycles, void* stream);
dec_status mg_solve(dec_mg* mg, double* u, const double* b, int nrhs, double rtol, int max_iters,
                    dec_solve_report* rep, void* stream, bool host_buffers, bool use_initial_guess,
                    const double* shifts = nullptr);
uint64_t mg_solve_submit(dec_mg* mg, double* u, const double* b, int nrhs, double rtol, int max_iters,
                         bool use_initial_guess);
dec_status mg_solve_wait(dec_mg* mg, uint64_t ticket, dec_solve_report* rep);
void mg_time_kernel(dec_mg* mg, int kernel, int level, int nrhs, int reps, void* stream, double* ms,
                    double* bytes);
int mg_autotune(dec_mg* mg, int nrhs, int reps, void* stream);
double mg_solve_traffic(dec_mg* mg, int nrhs, int from_zero, int iterations);
void mg_set_smoother_mlp(dec_mg* mg, const dec_mlp* mlp);
dec_batch* batch_create(dec_mg* const* groups, int ngroups);
void batch_destroy(dec_batch* b);
void batch_autotune(dec_batch* b, const int* nrhs, int reps, void* stream);
double batch_traffic(const dec_batch* b, int iterations);
dec_status batch_solve(dec_batch* b, double* const* u, const double* const* rhs, const int* nrhs,
                       const double* const* shifts, double rtol, int max_iters, dec_solve_report* reps,
                       dec_solve_report* total, void* stream);
}  // namespace decb
