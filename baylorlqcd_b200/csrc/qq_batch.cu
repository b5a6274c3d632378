// Batched mixed-precision propagators and loop traces (filled in below).
#include "qq_ctx.h"

namespace qq {

int batch_solve(qq_ctx* c, int nrhs, const double* be, const double* bo, const double kappa[2],
                const qq_method* method, double* xe, double* xo, qq_solve_info* infos) {
  (void)c; (void)nrhs; (void)be; (void)bo; (void)kappa; (void)method; (void)xe; (void)xo; (void)infos;
  return set_error(QQ_BAD_ARG, "batched solver not built yet");
}

int traces_level0(qq_ctx* c, const double* be, const double* bo, const double* xe,
                  const double* xo, double kappa, double* J) {
  (void)c; (void)be; (void)bo; (void)xe; (void)xo; (void)kappa; (void)J;
  return set_error(QQ_BAD_ARG, "traces not built yet");
}

}  // namespace qq
