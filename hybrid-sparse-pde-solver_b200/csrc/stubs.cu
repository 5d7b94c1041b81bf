// stubs.cu -- temporary: solvers not yet implemented.
#include "krylov.cuh"
namespace hamlss {
std::unique_ptr<Prec> make_amg(Ctx&, hamlss_mat*, const hamlss_params&) { fail(HAMLSS_ERR_INVALID, "AMG not built yet"); }
SolveResult mixed_solve(Ctx&, int, hamlss_mat*, Prec*, const double*, double*, const hamlss_params&, Workspace&, int*) { fail(HAMLSS_ERR_INVALID, "mixed not built yet"); }
}
extern "C" {
int hamlss_solve_adaptive(hamlss_ctx*, const hamlss_mat*, const double*, double*, int, const hamlss_params*, hamlss_stats*, hamlss_escalation*, int32_t, int32_t*, int32_t*) { return HAMLSS_ERR_INVALID; }
int hamlss_extract_features(hamlss_ctx*, const hamlss_mat*, double*, int32_t*) { return HAMLSS_ERR_INVALID; }
int hamlss_amg_aggregate(hamlss_ctx*, const hamlss_mat*, double, int32_t*, int32_t*) { return HAMLSS_ERR_INVALID; }
int hamlss_amg_num_levels(const hamlss_prec*, int32_t*) { return HAMLSS_ERR_INVALID; }
int hamlss_amg_level_matrix(const hamlss_prec*, int32_t, int32_t, int32_t*, int32_t*, int32_t*, int32_t*, int32_t*, double*) { return HAMLSS_ERR_INVALID; }
}
