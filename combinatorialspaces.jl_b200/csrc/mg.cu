#include "mg.cuh"
struct dec_mg {};
namespace decb {
void mg_default_options(dec_mg_options& o) { o = dec_mg_options{}; }
dec_mg* mg_create(const dec_mesh_desc&, const dec_mg_options&) { throw Error(DEC_ERR_UNSUPPORTED, "mg: not built"); }
void mg_destroy(dec_mg* mg) { delete mg; }
void mg_level_info(const dec_mg*, int, int64_t*, int64_t*, int64_t*, double*) { throw Error(DEC_ERR_UNSUPPORTED, "mg"); }
const dec_mesh* mg_level_mesh(const dec_mg*, int) { throw Error(DEC_ERR_UNSUPPORTED, "mg"); }
const dec_op* mg_level_op(const dec_mg*, int) { throw Error(DEC_ERR_UNSUPPORTED, "mg"); }
void mg_cycles(dec_mg*, double*, const double*, int, int, void*) { throw Error(DEC_ERR_UNSUPPORTED, "mg"); }
dec_status mg_solve(dec_mg*, double*, const double*, int, double, int, dec_solve_report*, void*, bool) { throw Error(DEC_ERR_UNSUPPORTED, "mg"); }
}
