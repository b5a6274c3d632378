// CPU oracle (test infrastructure): loop traces (filled in with the trace kernels).
#include <cstring>

#include "oracle_impl.h"

extern "C" void oq_twaverage_level0(const oq_geom* g, const double* be, const double* bo,
                                    const double* xe, const double* xo, const double* u,
                                    double kappa, double* J) {
  (void)be; (void)bo; (void)xe; (void)xo; (void)u; (void)kappa;
  std::memset(J, 0, sizeof(double) * 2 * g->n[3] * 6);
}
