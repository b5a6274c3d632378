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
#include <functional>
#include <thread>
#include <vector>

#include "qq_ctx.h"

namespace qq {
int sources_z(qq_ctx* c, double* be, double* bo, bool z4);
int batch_solve(qq_ctx* c, int nrhs, const double* be, const double* bo, const double kappa[2],
                const qq_method* method, double* xe, double* xo, qq_solve_info* infos);
int traces_mom(qq_ctx* c, const double* be, const double* bo, const double* xe, const double* xo,
               double kappa, double delta, const int io[3], int dobndry, int nmom, double* J, int ir);

namespace {

// The noise loop: per noise (generator order), draw, solve, take the kappa-scaled traces
// J(2, nt, nmom, 6) and hand them to add().  pre (may be empty) runs on the calling
// thread while the first block of noises is drawn; it must not draw random numbers.
using PerNoise = std::function<int(const double* be, const double* bo, const double* xe, const double* xo)>;

// The noise loop: per noise (generator order), draw, solve and hand the device pair
// (noise, solution) to per_noise.  pre (may be empty) runs on the calling thread while the
// first block of noises is drawn; it must not draw random numbers.
int discon_loop_fn(qq_ctx* c, int noise_kind, int nnoise, const double kappa[2], const qq_method* method,
                   const PerNoise& per_noise, qq_solve_info* infos, const std::function<int()>& pre = {}) {
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
  // Host noise, double-buffered: a second thread draws the next block while the device
  // solves this one.  The generator has one user at a time and draws noise by noise,
  // be then bo, exactly as many noises as requested: the stream is the reference's.
  std::vector<double> hb[2] = {std::vector<double>(2 * nv * block), std::vector<double>(2 * nv * block)};
  const bool z4 = noise_kind == 4;
  auto draw = [c, nv, z4, &hb](int which, int nb) -> int {
    for (int k = 0; k < nb; ++k) {
      double* e = hb[which].data() + 2 * nv * k;
      const int st = sources_z(c, e, e + nv, z4);
      if (st != QQ_OK) return st;
    }
    return QQ_OK;
  };
  int gen_rc = QQ_OK;  // declared before the joiner, which joins the thread on every exit
  struct Joiner {
    std::thread t;
    ~Joiner() {
      if (t.joinable()) t.join();
    }
  } gen;
  struct DeflGuard {
    qq_defl* d = nullptr;
    ~DeflGuard() {
      if (d) qq_defl_destroy(d);
    }
  } defl;
  if (method->solver == 2) QQ_TRY(qq_defl_create(c, method->m, method->k, &defl.d));
  int cur = 0;
  if (pre) {
    gen.t = std::thread([&gen_rc, &draw, nb0 = std::min(block, nnoise), dev = c->device] {
      cudaSetDevice(dev);
      gen_rc = draw(0, nb0);
    });
    const int pre_rc = pre();
    gen.t.join();
    QQ_TRY(pre_rc);
    QQ_TRY(gen_rc);
  } else {
    QQ_TRY(draw(cur, std::min(block, nnoise)));
  }
  int rc = QQ_OK;
  for (int i0 = 0; i0 < nnoise && rc == QQ_OK; i0 += block) {
    const int nb = std::min(block, nnoise - i0);
    for (int k = 0; k < nb; ++k) {
      const double* e = hb[cur].data() + 2 * nv * k;
      QQ_CK(cudaMemcpyAsync(dbe.as<double>() + nv * k, e, sizeof(double) * nv, cudaMemcpyHostToDevice, c->st));
      QQ_CK(cudaMemcpyAsync(dbo.as<double>() + nv * k, e + nv, sizeof(double) * nv, cudaMemcpyHostToDevice,
                            c->st));
    }
    QQ_CK(cudaStreamSynchronize(c->st));  // hb[cur] may be redrawn from here on
    const int nb1 = std::min(block, nnoise - (i0 + nb));
    gen_rc = QQ_OK;
    if (nb1 > 0) gen.t = std::thread([&gen_rc, &draw, cur, nb1, dev = c->device] {
      cudaSetDevice(dev);
      gen_rc = draw(1 - cur, nb1);
    });
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
                       dxo.as<double>(), 0, i0 == 0 ? 1 : 2, defl.d, inf);
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
    for (int k = 0; k < nb; ++k)
      QQ_TRY(per_noise(dbe.as<double>() + nv * k, dbo.as<double>() + nv * k, dxe.as<double>() + nv * k,
                       dxo.as<double>() + nv * k));
    if (gen.t.joinable()) gen.t.join();
    if (gen_rc != QQ_OK) return gen_rc;
    cur = 1 - cur;
  }
  return rc;
}

// The twisted-mass form: the kappa-scaled level-0 traces J(2, nt, nmom, 6) of every noise
// handed to add().
int discon_loop(qq_ctx* c, int noise_kind, int nnoise, const double kappa[2], const qq_method* method,
                double delta, const int io[3], int dobndry, int ir, int nmom,
                const std::function<void(const double*)>& add, qq_solve_info* infos,
                const std::function<int()>& pre = {}) {
  std::vector<double> Jn((size_t)12 * c->g.n[3] * nmom);
  return discon_loop_fn(
      c, noise_kind, nnoise, kappa, method,
      [&](const double* be, const double* bo, const double* xe, const double* xo) -> int {
        QQ_TRY(traces_mom(c, be, bo, xe, xo, kappa[0], delta, io, dobndry, nmom, Jn.data(), ir));
        add(Jn.data());
        return QQ_OK;
      },
      infos, pre);
}

// Levels twAverage fills (:4519-4580): 1 always, 4 for nsub = 4 or 6, 6 for nsub = 6
// (0-based 0, 3, 5); with its subtraction switched off all carry the unsubtracted traces.
std::vector<int> filled_levels(int nsub) {
  std::vector<int> lv{0};
  if (nsub == 4 || nsub == 6) lv.push_back(3);
  if (nsub == 6) lv.push_back(5);
  return lv;
}

// J(2, nt, nmom, 6) -> add into Jl(2, nt, 6, nmom, nop) at the given levels.
void add_levels(const double* J, int nt, int nmom, int nop, const std::vector<int>& lv, double* Jl) {
  for (int iop = 0; iop < 6 && iop < nop; ++iop)
    for (int im = 0; im < nmom; ++im)
      for (int l : lv)
        for (int t = 0; t < nt; ++t)
          for (int ri = 0; ri < 2; ++ri) {
            const size_t src = (((size_t)iop * nmom + im) * nt + t) * 2 + ri;
            const size_t dst = ((((size_t)iop * nmom + im) * 6 + l) * nt + t) * 2 + ri;
            Jl[dst] = Jl[dst] + J[src];
          }
}

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_twvev(qq_ctx* c, double kappa, double delta, const int io[3], int dobndry, int ir, int nsub,
                        int nmom, int nop, double* Jvev);

extern "C" int qq_discon_traces(qq_ctx* c, int noise_kind, int nnoise, const double kappa[2],
                                const qq_method* method, double delta, int dobndry, double* J,
                                qq_solve_info* infos) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!kappa || !method || !J) return set_error(QQ_BAD_ARG, "null argument");
  const int nt = c->g.n[3];
  const int io[3] = {1, 1, 1};
  std::vector<double> Jsum((size_t)12 * nt, 0.0);
  const int rc = discon_loop(c, noise_kind, nnoise, kappa, method, delta, io, dobndry, 1, 1,
                             [&](const double* Jn) {
                               for (size_t e = 0; e < Jsum.size(); ++e) Jsum[e] += Jn[e];
                             },
                             infos);
  if (rc != QQ_OK && rc != QQ_NOT_CONVERGED) return rc;
  const double norm = 1.0 / ((double)nnoise * c->g.n[0] * c->g.n[1] * c->g.n[2]);
  for (size_t e = 0; e < Jsum.size(); ++e) Jsum[e] *= norm;
  QQ_CK(cudaMemcpy(J, Jsum.data(), sizeof(double) * Jsum.size(), cudaMemcpyDefault));
  return rc;
}

extern "C" int qq_twaverage(qq_ctx* c, const double* be, const double* bo, const double* xe, const double* xo,
                            double kappa, double delta, const int io[3], int dobndry, int ir, int nsub, int nmom,
                            int nop, double* Jave) {
  (void)kappa;  // enters only the subtraction levels, which the reference leaves switched off
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!be || !bo || !xe || !xo || !io || !Jave) return set_error(QQ_BAD_ARG, "null argument");
  if (nop < 6) return set_error(QQ_BAD_ARG, "nop must be at least 6");
  QQ_CK(cudaSetDevice(c->device));
  const int nt = c->g.n[3];
  std::vector<double> J((size_t)12 * nt * std::max(nmom, 1));
  QQ_TRY(traces_mom(c, be, bo, xe, xo, 1.0, delta, io, dobndry, nmom, J.data(), ir));
  std::vector<double> out((size_t)2 * nt * 6 * nmom * nop, 0.0);
  if (nsub == 0 || nsub == 4 || nsub == 6) add_levels(J.data(), nt, nmom, nop, filled_levels(nsub), out.data());
  QQ_CK(cudaMemcpy(Jave, out.data(), sizeof(double) * out.size(), cudaMemcpyDefault));
  return QQ_OK;
}

extern "C" int qq_twistdiscon(qq_ctx* c, int noise_kind, int nnoise, const double kappa[2],
                              const qq_method* method, double delta, const int io[3], int dobndry, int ir,
                              int nsub, int nmom, int nop, double* Jtotal, double* Jnoise, qq_solve_info* infos) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!kappa || !method || !io || !Jtotal) return set_error(QQ_BAD_ARG, "null argument");
  if (nop < 6) return set_error(QQ_BAD_ARG, "nop must be at least 6");
  if (nmom < 1 || nmom > 5) return set_error(QQ_BAD_ARG, "nmom must be 1..5");
  const int nt = c->g.n[3];
  const size_t n = (size_t)2 * nt * 6 * nmom * nop;
  auto at = [&](int ri, int t, int lv, int im, int iop) {
    return ((((size_t)iop * nmom + im) * 6 + lv) * nt + t) * 2 + ri;
  };
  // Jtotal = numnoises * Jvev (:3779-3839): twvev, kappa on every operator but 2 and 6,
  // the highest order combined with the first for nsub = 6 (run while the first block of
  // noises is drawn)
  std::vector<double> jt(n, 0.0), jvev;
  // per-noise values Jtemp(..., inoise) = Jave' + Jvev' (:4112-4114), kept when asked for
  std::vector<double> jn(Jnoise ? n * (size_t)nnoise : 0, 0.0);
  int inoise = 0;
  auto vev = [&]() -> int {
    if (nsub != 4 && nsub != 6) return QQ_OK;
    std::vector<double> jv(n);
    QQ_TRY(qq_twvev(c, kappa[0], delta, io, dobndry, ir, nsub, nmom, nop, jv.data()));
    for (int iop = 0; iop < nop; ++iop)
      if (iop != 1 && iop != 5)
        for (int im = 0; im < nmom; ++im)
          for (int lv = 0; lv < 6; ++lv)
            for (int t = 0; t < nt; ++t)
              for (int ri = 0; ri < 2; ++ri) jv[at(ri, t, lv, im, iop)] = kappa[0] * jv[at(ri, t, lv, im, iop)];
    if (nsub == 6)
      for (int iop = 0; iop < nop; ++iop)
        for (int im = 0; im < nmom; ++im)
          for (int t = 0; t < nt; ++t)
            for (int ri = 0; ri < 2; ++ri)
              jv[at(ri, t, 5, im, iop)] = jv[at(ri, t, 3, im, iop)] + jv[at(ri, t, 5, im, iop)];
    for (size_t e = 0; e < n; ++e) jt[e] = nnoise * jv[e];
    jvev.swap(jv);
    return QQ_OK;
  };
  // + the kappa-scaled traces of every noise at the levels twAverage fills (:4040-4045)
  const std::vector<int> lv = filled_levels(nsub);
  const bool any = nsub == 0 || nsub == 4 || nsub == 6;
  if (ir != 1 && ir != -1) return set_error(QQ_BAD_ARG, "ir must be 1 or -1");
  const int rc = discon_loop(c, noise_kind, nnoise, kappa, method, delta, io, dobndry, ir, nmom,
                             [&](const double* Jn) {
                               if (any) add_levels(Jn, nt, nmom, nop, lv, jt.data());
                               if (Jnoise && any) add_levels(Jn, nt, nmom, nop, lv, jn.data() + n * inoise);
                               ++inoise;
                             },
                             infos, vev);
  if (rc != QQ_OK && rc != QQ_NOT_CONVERGED) return rc;
  // :4161-4164
  for (size_t e = 0; e < n; ++e) jt[e] = jt[e] / (double)nnoise;
  const double nxyz = (double)c->g.n[0] * c->g.n[1] * c->g.n[2];
  for (size_t e = 0; e < n; ++e) jt[e] = jt[e] / nxyz;
  QQ_CK(cudaMemcpy(Jtotal, jt.data(), sizeof(double) * n, cudaMemcpyDefault));
  if (Jnoise) {  // written out as fac * Jtemp, fac = 1/(nx*ny*nz) (:4230-4233)
    const double fac = 1.0 / nxyz;
    for (int k = 0; k < nnoise; ++k)
      for (size_t e = 0; e < n; ++e) {
        double& v = jn[n * k + e];
        if (!jvev.empty()) v = v + jvev[e];
        v = fac * v;
      }
    QQ_CK(cudaMemcpy(Jnoise, jn.data(), sizeof(double) * jn.size(), cudaMemcpyDefault));
  }
  return rc;
}

extern "C" int qq_vev(qq_ctx* c, double kappa, const int io[3], double* Jvev, double* plaq, double* psi);

// discon, Q/disconloops.f90:3445-3608 (one run): Jtotal(isub >= 2) starts as the vev
// Jvev; every noise's average (nsub levels, nmom momenta with the momfacs factors about
// io) is added; the sum is divided by the number of noises (Jvev included, as the
// reference does) and by nx*ny*nz.  The reference solves its noises with QMR (inverter
// 2); here the method's solver runs.
extern "C" int qq_discon(qq_ctx* c, int noise_kind, int nnoise, double kappa, const qq_method* method,
                         const int io[3], int nsub, int nmom, int nop, double* Jtotal, double* Jvev_out,
                         qq_solve_info* infos) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!method || !io || !Jtotal) return set_error(QQ_BAD_ARG, "null argument");
  if (nsub < 1 || nsub > 6) return set_error(QQ_BAD_ARG, "nsub must be 1..6");
  if (nmom < 1 || nmom > 5) return set_error(QQ_BAD_ARG, "nmom must be 1..5");
  if (nop < 1 || nop > 9) return set_error(QQ_BAD_ARG, "nop must be 1..9");
  QQ_CK(cudaSetDevice(c->device));
  const int nt = c->g.n[3];
  const size_t n = (size_t)2 * nt * nsub * nmom * nop, n9 = (size_t)2 * nt * nsub * nmom * 9;
  std::vector<double> jv((size_t)2 * nt * 25), jt(n, 0.0), ja(n9);
  QQ_TRY(qq_vev(c, kappa, io, jv.data(), nullptr, nullptr));
  if (Jvev_out) QQ_CK(cudaMemcpy(Jvev_out, jv.data(), sizeof(double) * jv.size(), cudaMemcpyDefault));
  auto at = [&](int ri, int t, int isub, int im, int iop) {  // Jtotal(2, nt, nsub, nmom, nop), 0-based
    return ((((size_t)iop * nmom + im) * nsub + isub) * nt + t) * 2 + ri;
  };
  for (int iop = 0; iop < std::min(nop, 5); ++iop)  // :3545-3547
    for (int im = 0; im < nmom; ++im)
      for (int isub = 1; isub < nsub; ++isub)
        for (int t = 0; t < nt; ++t)
          for (int ri = 0; ri < 2; ++ri)
            jt[at(ri, t, isub, im, iop)] = jv[((((size_t)iop * 5) + im) * nt + t) * 2 + ri];
  DevBuf dmf;
  if (nmom > 1) {
    const size_t nmf = (size_t)5 * 4 * 16 * 2 * (c->g.vh / 16);
    std::vector<double> mf(nmf);
    QQ_TRY(qq_momfacs(c->g.n, io, mf.data()));
    QQ_CK(dmf.alloc(sizeof(double) * nmf));
    QQ_CK(cudaMemcpy(dmf.p, mf.data(), sizeof(double) * nmf, cudaMemcpyHostToDevice));
  }
  const double kap[2] = {kappa, 0.0};
  const int rc = discon_loop_fn(
      c, noise_kind, nnoise, kap, method,
      [&](const double* be, const double* bo, const double* xe, const double* xo) -> int {
        QQ_TRY(qq_average(c, be, bo, xe, xo, kappa, nsub, nmom, 9, nmom > 1 ? dmf.as<double>() : nullptr,
                          ja.data()));
        for (int iop = 0; iop < nop; ++iop)
          for (int im = 0; im < nmom; ++im)
            for (int isub = 0; isub < nsub; ++isub)
              for (int t = 0; t < nt; ++t)
                for (int ri = 0; ri < 2; ++ri) jt[at(ri, t, isub, im, iop)] += ja[((((size_t)iop * nmom + im) * nsub + isub) * nt + t) * 2 + ri];
        return QQ_OK;
      },
      infos);
  if (rc != QQ_OK && rc != QQ_NOT_CONVERGED) return rc;
  const double nxyz = (double)c->g.n[0] * c->g.n[1] * c->g.n[2];
  for (double& v : jt) v = v / (double)nnoise / nxyz;  // :3581-3584
  QQ_CK(cudaMemcpy(Jtotal, jt.data(), sizeof(double) * n, cudaMemcpyDefault));
  return rc;
}
