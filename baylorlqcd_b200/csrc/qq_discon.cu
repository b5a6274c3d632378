// Batched disconnected loops (qq_discon_traces): the noise loop of twistdiscon
// (Q/disconloops.f90:3612-4170) at the unsubtracted level.  Per noise, in the
// reference's order: draw Z(2) or Z(4) noise from the lagged-Fibonacci stream
// (z2source / z4source, be then bo), solve the propagator, take the level-0 traces
// (twAverage at nsub = 0 with the kappa scaling of :4045-4049) and accumulate; at the
// end divide by the number of noises and by nx*ny*nz (:4161-4164).
//
// The solves run through the library's own paths: solver 0 = plain FP64 GMRES-DR per
// noise, solver 1 = batched mixed-precision BiCGStab on blocks of rhs_block noises,
// solver 2 = the reference's psc sequence (GMRES-DR on the first noise keeping its
// deflation space, GMRES-Proj to the fixed 1e-8 on the rest, :3783-3790, :3936).
// Noise, solutions and traces stay in device memory; only the generator runs on the
// host, as in the reference.
#include <algorithm>
#include <cstring>
#include <vector>

#include "qq_ctx.h"

namespace qq {
int sources_z(qq_ctx* c, double* be, double* bo, bool z4);
int batch_solve(qq_ctx* c, int nrhs, const double* be, const double* bo, const double kappa[2],
                const qq_method* method, double* xe, double* xo, qq_solve_info* infos);
int traces_level0(qq_ctx* c, const double* be, const double* bo, const double* xe,
                  const double* xo, double kappa, double delta, int dobndry, double* J);
}  // namespace qq

using namespace qq;

extern "C" int qq_discon_traces(qq_ctx* c, int noise_kind, int nnoise, const double kappa[2],
                                const qq_method* method, double delta, int dobndry, double* J,
                                qq_solve_info* infos) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!kappa || !method || !J) return set_error(QQ_BAD_ARG, "null argument");
  if (noise_kind != 2 && noise_kind != 4) return set_error(QQ_BAD_ARG, "noise_kind must be 2 or 4");
  if (nnoise < 1) return set_error(QQ_BAD_ARG, "nnoise must be >= 1");
  if (method->solver < 0 || method->solver > 2) return set_error(QQ_BAD_ARG, "solver must be 0, 1 or 2");
  QQ_CK(cudaSetDevice(c->device));
  const size_t nv = c->ref_doubles();
  const int nt = c->g.n[3];
  const int block = method->solver == 1 ? std::max(1, std::min(method->rhs_block, kMaxBatch)) : 1;
  // device copies of a block of noises and solutions (reference layout)
  DevBuf dbe, dbo, dxe, dxo;
  QQ_CK(dbe.alloc(sizeof(double) * nv * block));
  QQ_CK(dbo.alloc(sizeof(double) * nv * block));
  QQ_CK(dxe.alloc(sizeof(double) * nv * block));
  QQ_CK(dxo.alloc(sizeof(double) * nv * block));
  std::vector<double> hbe(nv), hbo(nv), Jn((size_t)12 * nt), Jsum((size_t)12 * nt, 0.0);
  qq_defl* defl = nullptr;
  if (method->solver == 2) QQ_TRY(qq_defl_create(c, method->m, method->k, &defl));
  int rc = QQ_OK;
  for (int i0 = 0; i0 < nnoise && rc == QQ_OK; i0 += block) {
    const int nb = std::min(block, nnoise - i0);
    for (int k = 0; k < nb; ++k) {  // the generator's order: noise by noise, be then bo
      QQ_TRY(sources_z(c, hbe.data(), hbo.data(), noise_kind == 4));
      QQ_CK(cudaMemcpyAsync(dbe.as<double>() + nv * k, hbe.data(), sizeof(double) * nv,
                            cudaMemcpyHostToDevice, c->st));
      QQ_CK(cudaMemcpyAsync(dbo.as<double>() + nv * k, hbo.data(), sizeof(double) * nv,
                            cudaMemcpyHostToDevice, c->st));
      QQ_CK(cudaStreamSynchronize(c->st));  // hbe / hbo are reused for the next noise
    }
    qq_solve_info* inf = infos ? infos + i0 : nullptr;
    std::vector<qq_solve_info> local;
    if (!inf) {
      local.resize(nb);
      inf = local.data();
    }
    int st = QQ_OK;
    if (method->solver == 2) {
      const int gm[2] = {method->m, method->k};
      QQ_CK(cudaMemsetAsync(dxe.p, 0, sizeof(double) * nv, c->st));
      QQ_CK(cudaMemsetAsync(dxo.p, 0, sizeof(double) * nv, c->st));
      st = qq_fermprop(c, dbe.as<double>(), dbo.as<double>(), kappa, 6, method->tol, 0, gm, dxe.as<double>(),
                       dxo.as<double>(), 0, i0 == 0 ? 1 : 2, defl, inf);
    } else {
      QQ_CK(cudaMemsetAsync(dxe.p, 0, sizeof(double) * nv * nb, c->st));
      QQ_CK(cudaMemsetAsync(dxo.p, 0, sizeof(double) * nv * nb, c->st));
      st = batch_solve(c, nb, dbe.as<double>(), dbo.as<double>(), kappa, method, dxe.as<double>(),
                       dxo.as<double>(), inf);
    }
    if (st != QQ_OK && st != QQ_NOT_CONVERGED) {
      rc = st;
      break;
    }
    if (st == QQ_NOT_CONVERGED) rc = QQ_NOT_CONVERGED;
    for (int k = 0; k < nb; ++k) {
      QQ_TRY(traces_level0(c, dbe.as<double>() + nv * k, dbo.as<double>() + nv * k, dxe.as<double>() + nv * k,
                           dxo.as<double>() + nv * k, kappa[0], delta, dobndry, Jn.data()));
      for (size_t e = 0; e < Jn.size(); ++e) Jsum[e] += Jn[e];
    }
  }
  if (defl) qq_defl_destroy(defl);
  if (rc != QQ_OK && rc != QQ_NOT_CONVERGED) return rc;
  const double norm = 1.0 / ((double)nnoise * c->g.n[0] * c->g.n[1] * c->g.n[2]);
  for (size_t e = 0; e < Jsum.size(); ++e) Jsum[e] *= norm;
  QQ_CK(cudaMemcpy(J, Jsum.data(), sizeof(double) * Jsum.size(), cudaMemcpyDefault));
  return rc;
}
