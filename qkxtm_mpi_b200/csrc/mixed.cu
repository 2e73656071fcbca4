// mixed.cu -- even-odd mixed-precision CG (placeholder until implemented)
#include "qkx_ctx.cuh"
namespace qkx {
int invert_eo_mixed(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double2* const* b,
                    double2* const* x, qkx_solve_info* info) {
  set_error("CG_EO_MIXED not built yet");
  return QKX_ERR_UNSUPPORTED;
}
void mixed_free(qkx_ctx* c) {}
}  // namespace qkx
