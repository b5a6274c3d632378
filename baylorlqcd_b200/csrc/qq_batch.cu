// Batched mixed-precision propagators (qq_fermprop_batch).
//
// Method for nrhs sources on one configuration:
//   1. source preparation and odd-half reconstruction exactly as fermprop
//      (Q/quark.f90:595-618, :787-824), in FP64;
//   2. the first right-hand side is solved with mixed-precision GMRES-DR(m, k), which
//      also yields an FP32 deflation space (k harmonic-Ritz vectors);
//   3. the other right-hand sides are first projected onto that space (the minimum-
//      residual step of GMRES-Proj) and then solved together, in blocks, by BiCGStab
//      in FP32 or FP16 with FP64 reliable updates: whenever the iterated residual has
//      dropped by `delta` since the last update, the FP64 solution is updated and the
//      FP64 true residual replaces the low-precision one (and is re-projected);
//   4. every answer is judged by its FP64 true residual.
// precision = 64 runs the plain FP64 GMRES-DR(m, k) of the reference on every RHS.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "qq_ctx.h"
#include "qq_mrhs.cuh"

namespace qq {

namespace {

struct PerRhs {
  Field b, x;                  // FP64 even-system source and solution
  Field r64;                   // FP64 residual
  Field r, rhat, p, v, t, xl;  // low precision BiCGStab vectors
  Field tmp;                   // odd-parity temporary (low precision)
  double bn = 0.0, rmax = 0.0, rn = 0.0;
  bool done = false;
  int slot = 0;
};

int alloc_field(qq_ctx* c, Field& f, int prec) {
  f.prec = prec;
  QQ_CK(f.data.alloc(field_bytes(prec, c->g.vh)));
  if (prec == P16) QQ_CK(f.norm.alloc(sizeof(float) * c->g.vh));
  return QQ_OK;
}

template <int P>
int launch_bicg_op(qq_ctx* c, const BatchArgs& A, int op) {
  dim3 grd(kRedBlocks, A.n);
  switch (op) {
    case OP_DOT_RHAT_R: bicg_kernel<P, OP_DOT_RHAT_R><<<grd, kRedThreads, 0, c->st>>>(A); break;
    case OP_P_UPDATE: bicg_kernel<P, OP_P_UPDATE><<<grd, kRedThreads, 0, c->st>>>(A); break;
    case OP_DOT_RHAT_V: bicg_kernel<P, OP_DOT_RHAT_V><<<grd, kRedThreads, 0, c->st>>>(A); break;
    case OP_S_UPDATE: bicg_kernel<P, OP_S_UPDATE><<<grd, kRedThreads, 0, c->st>>>(A); break;
    case OP_DOTS_T: bicg_kernel<P, OP_DOTS_T><<<grd, kRedThreads, 0, c->st>>>(A); break;
    case OP_XR_UPDATE: bicg_kernel<P, OP_XR_UPDATE><<<grd, kRedThreads, 0, c->st>>>(A); break;
    default: return set_error(QQ_BAD_ARG, "bad batched op");
  }
  QQ_CK(cudaGetLastError());
  return QQ_OK;
}

int bicg_op(qq_ctx* c, int prec, const BatchArgs& A, int op, const int* dslots, int step) {
  count_launch(step >= 0 ? 2 : 1);
  if (prec == P32)
    QQ_TRY(launch_bicg_op<P32>(c, A, op));
  else if (prec == P16)
    QQ_TRY(launch_bicg_op<P16>(c, A, op));
  else
    QQ_TRY(launch_bicg_op<P64>(c, A, op));
  if (step >= 0) {
    bicg_scalar_kernel<<<A.n, 256, 0, c->st>>>(A.S, dslots, A.partial, kRedBlocks, step);
    QQ_CK(cudaGetLastError());
  }
  return QQ_OK;
}

// Full-lattice FP64 residual ||b - M x|| / ||b|| of the unpreconditioned operator
// M = (1 + 2 i kappa mu gamma5) - kappa H on both parities (the system fermprop
// solves, Q/diracops.f90:10-40).
int full_residual(qq_ctx* c, Spinor be, Spinor bo, Spinor xe, Spinor xo, const double kappa[2],
                  double* rel) {
  Tmp h(c, P64), m(c, P64);
  const double tk = 2.0 * kappa[0] * kappa[1];
  double num = 0.0, den = 0.0;
  for (int par = 0; par < 2; ++par) {
    Spinor xs = par == 0 ? xe : xo, xother = par == 0 ? xo : xe, bs = par == 0 ? be : bo;
    QQ_TRY(op_hsingle(c, h.sp(), xother, 0, par));
    // m = x + tk J x - kappa H x_other ; then r = b - m
    QQ_CK(launch_spinmix(c->g.vh, xs, h.sp(), m.sp(), 1.0, tk, -kappa[0], 0.0, P64, c->st));
    double* s = c->scal.as<double>();
    QQ_TRY(lin(c, m.sp(), cimm(1.0), bs, cimm(-1.0), m.sp(), cimm(0), Spinor{nullptr, nullptr, P64}, s));
    double n2 = 0.0, b2 = 0.0;
    QQ_TRY(read_scalars(c, s, 1, &n2));
    QQ_TRY(norm2_host(c, bs, &b2));
    num += n2;
    den += b2;
  }
  *rel = std::sqrt(num / den);
  return QQ_OK;
}

}  // namespace

// Deflated mixed-precision BiCGStab on a set of right-hand sides (all active at once).
int bicgstab_mixed_batch(qq_ctx* c, std::vector<PerRhs*>& rhs, int prec, double tol, double delta,
                         int maxiter, const double kappa[2], const DeflSpace* defl,
                         std::vector<SolveStats>& stats) {
  const int n = (int)rhs.size();
  if (n == 0) return QQ_OK;
  if (n > kMaxBatch) return set_error(QQ_BAD_ARG, "too many right-hand sides in one block");
  DevBuf S, part, dslots;
  QQ_CK(S.alloc(sizeof(double) * kScal * kMaxBatch));
  QQ_CK(part.alloc(sizeof(double) * 3 * kRedBlocks * kMaxBatch));
  QQ_CK(dslots.alloc(sizeof(int) * kMaxBatch));
  Tmp tmp64(c, P64);
  std::vector<double> hS(kScal * kMaxBatch, 0.0);
  for (int i = 0; i < n; ++i) {
    PerRhs& R = *rhs[i];
    R.slot = i;
    QQ_TRY(norm2_host(c, R.b.sp(), &R.bn));
    R.bn = std::sqrt(R.bn);
    // r = b - A x, then project onto the deflation space
    {
      Tmp h(c, P64);
      QQ_TRY(op_dbletm(c, h.sp(), R.x.sp(), tmp64.sp(), 0, kappa));
      double* s = c->scal.as<double>();
      QQ_TRY(lin(c, R.r64.sp(), cimm(1.0), R.b.sp(), cimm(-1.0), h.sp(), cimm(0), Spinor{nullptr, nullptr, P64}, s));
      double n2;
      QQ_TRY(read_scalars(c, s, 1, &n2));
      R.rn = std::sqrt(n2);
      stats[i].mvp += 1;
    }
    if (defl && defl->k > 0) {
      QQ_TRY(defl_project(c, *defl, R.b.sp(), R.x.sp(), R.r64.sp(), kappa, &R.rn));
      stats[i].mvp += 1;
    }
    R.rmax = R.rn;
    R.done = !(R.bn > 0.0) || R.rn / R.bn <= tol;
    QQ_TRY(lin(c, R.r.sp(), cimm(1.0), R.r64.sp()));
    QQ_TRY(copy_field(c, R.rhat.sp(), R.r.sp()));
    QQ_TRY(zero_field(c, R.p.sp()));
    QQ_TRY(zero_field(c, R.v.sp()));
    QQ_TRY(zero_field(c, R.xl.sp()));
    double* s = &hS[(size_t)i * kScal];
    s[SC_RHO] = s[SC_ALPHA] = s[SC_OMEGA] = 1.0;
    s[SC_RHO + 1] = s[SC_ALPHA + 1] = s[SC_OMEGA + 1] = 0.0;
    stats[i].true_rel = R.bn > 0.0 ? R.rn / R.bn : 0.0;
  }
  QQ_CK(cudaMemcpyAsync(S.p, hS.data(), sizeof(double) * hS.size(), cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  std::vector<double> r2(kMaxBatch);
  for (int it = 0; it < maxiter; ++it) {
    std::vector<PerRhs*> act;
    for (auto* R : rhs)
      if (!R->done) act.push_back(R);
    if (act.empty()) break;
    BatchArgs A;
    std::memset(&A, 0, sizeof(A));
    A.vh = c->g.vh;
    A.n = (int)act.size();
    A.S = S.as<double>();
    A.partial = part.as<double>();
    std::vector<int> slots(A.n);
    std::vector<Spinor> pin(A.n), vout(A.n), rin(A.n), tout(A.n), tmpo(A.n);
    for (int k = 0; k < A.n; ++k) {
      PerRhs& R = *act[k];
      A.r[k] = R.r.sp();
      A.rhat[k] = R.rhat.sp();
      A.p[k] = R.p.sp();
      A.v[k] = R.v.sp();
      A.t[k] = R.t.sp();
      A.x[k] = R.xl.sp();
      A.slot[k] = R.slot;
      slots[k] = R.slot;
      pin[k] = R.p.sp();
      vout[k] = R.v.sp();
      rin[k] = R.r.sp();
      tout[k] = R.t.sp();
      tmpo[k] = R.tmp.sp();
    }
    QQ_CK(cudaMemcpyAsync(dslots.p, slots.data(), sizeof(int) * A.n, cudaMemcpyHostToDevice, c->st));
    const int* ds = dslots.as<int>();
    QQ_TRY(bicg_op(c, prec, A, OP_DOT_RHAT_R, ds, ST_BETA));
    QQ_TRY(bicg_op(c, prec, A, OP_P_UPDATE, ds, -1));
    QQ_TRY(op_dbletm_multi(c, vout.data(), pin.data(), tmpo.data(), A.n, 0, kappa));
    QQ_TRY(bicg_op(c, prec, A, OP_DOT_RHAT_V, ds, ST_ALPHA));
    QQ_TRY(bicg_op(c, prec, A, OP_S_UPDATE, ds, -1));
    QQ_TRY(op_dbletm_multi(c, tout.data(), rin.data(), tmpo.data(), A.n, 0, kappa));
    QQ_TRY(bicg_op(c, prec, A, OP_DOTS_T, ds, ST_OMEGA));
    QQ_TRY(bicg_op(c, prec, A, OP_XR_UPDATE, ds, ST_R2));
    // read ||r||^2 of the active right-hand sides
    QQ_CK(cudaMemcpyAsync(hS.data(), S.p, sizeof(double) * kScal * kMaxBatch, cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    std::vector<PerRhs*> upd;
    for (auto* R : act) {
      SolveStats& stt = stats[std::find(rhs.begin(), rhs.end(), R) - rhs.begin()];
      stt.itercount += 1;
      stt.mvp += 2;
      const double rn = std::sqrt(hS[(size_t)R->slot * kScal + SC_R2]);
      if (!std::isfinite(rn)) return set_error(QQ_NAN, "NaN residual in batched BiCGStab");
      if (rn < delta * R->rmax || rn / R->bn < 0.5 * tol) upd.push_back(R);
    }
    // reliable updates: x64 += xl ; r64 = b - A x64 (FP64) ; r = r64
    for (auto* R : upd) {
      SolveStats& stt = stats[std::find(rhs.begin(), rhs.end(), R) - rhs.begin()];
      QQ_TRY(lin(c, R->x.sp(), cimm(1.0), R->xl.sp(), cimm(1.0), R->x.sp()));
      QQ_TRY(zero_field(c, R->xl.sp()));
      Tmp h(c, P64);
      QQ_TRY(op_dbletm(c, h.sp(), R->x.sp(), tmp64.sp(), 0, kappa));
      double* s = c->scal.as<double>();
      QQ_TRY(lin(c, R->r64.sp(), cimm(1.0), R->b.sp(), cimm(-1.0), h.sp(), cimm(0), Spinor{nullptr, nullptr, P64}, s));
      double n2;
      QQ_TRY(read_scalars(c, s, 1, &n2));
      R->rn = std::sqrt(n2);
      stt.mvp += 1;
      if (defl && defl->k > 0 && R->rn / R->bn > tol) {
        // re-deflate: the low modes the iteration has re-excited are removed exactly
        QQ_TRY(defl_project(c, *defl, R->b.sp(), R->x.sp(), R->r64.sp(), kappa, &R->rn));
        stt.mvp += 1;
      }
      stt.true_rel = R->rn / R->bn;
      stt.hist.push_back(stt.true_rel);
      stt.hist_mvp.push_back(stt.mvp);
      if (R->rn / R->bn <= tol) {
        R->done = true;
        continue;
      }
      QQ_TRY(lin(c, R->r.sp(), cimm(1.0), R->r64.sp()));
      R->rmax = R->rn;
    }
  }
  int status = QQ_OK;
  for (auto* R : rhs)
    if (!R->done) status = QQ_NOT_CONVERGED;
  return status;
}

int batch_solve(qq_ctx* c, int nrhs, const double* be, const double* bo, const double kappa[2],
                const qq_method* meth, double* xe, double* xo, qq_solve_info* infos) {
  const int prec = meth->precision == 64 ? P64 : meth->precision == 32 ? P32 : meth->precision == 16 ? P16 : -1;
  if (prec < 0) return set_error(QQ_BAD_ARG, "precision must be 64, 32 or 16");
  if (meth->solver != 0 && meth->solver != 1) return set_error(QQ_BAD_ARG, "solver must be 0 or 1");
  if (meth->m < 2 || meth->k < 1 || meth->k >= meth->m || meth->m > 127)
    return set_error(QQ_BAD_ARG, "GMRES(m,k) out of range");
  if (!(meth->tol > 0.0)) return set_error(QQ_BAD_ARG, "tol must be > 0");
  const int block = std::max(1, std::min(meth->rhs_block, kMaxBatch));
  const size_t nv = c->ref_doubles();
  const double tk = 2.0 * kappa[0] * kappa[1];
  const double fac1 = 1.0 / (kappa[0] * kappa[0]);
  const double fac2 = 1.0 / (kappa[0] * (1.0 + tk * tk));
  // even-system tolerance: the full-lattice residual is checked at the end
  const double tol_even = meth->tol * 0.25;
  std::vector<std::unique_ptr<PerRhs>> R(nrhs);
  std::vector<SolveStats> stats(nrhs);
  std::vector<double> seconds(nrhs, 0.0);
  std::vector<int> status(nrhs, QQ_OK);
  Tmp fbe(c, P64), fbo(c, P64), h(c, P64);
  for (int i = 0; i < nrhs; ++i) {
    R[i].reset(new PerRhs());
    PerRhs& r = *R[i];
    QQ_TRY(alloc_field(c, r.b, P64));
    QQ_TRY(alloc_field(c, r.x, P64));
    QQ_TRY(alloc_field(c, r.r64, P64));
    QQ_TRY(zero_field(c, r.x.sp()));
    // fermprop source: b_e/kappa^2 + H_eo (1 - 2 i kappa mu gamma5) b_o / (kappa (1 + tk^2))
    const double* de = nullptr;
    const double* dO = nullptr;
    QQ_TRY(stage_in(c, 1, be + (size_t)i * nv, nv, &de));
    QQ_TRY(ref_to_field(c, de, 0, fbe.sp()));
    QQ_TRY(stage_in(c, 2, bo + (size_t)i * nv, nv, &dO));
    QQ_TRY(ref_to_field(c, dO, 1, fbo.sp()));
    QQ_CK(launch_spinmix(c->g.vh, fbo.sp(), Spinor{nullptr, nullptr, P64}, r.r64.sp(), 1.0, -tk, 0.0, 0.0, P64, c->st));
    QQ_TRY(op_hsingle(c, h.sp(), r.r64.sp(), 0, 0));
    QQ_TRY(lin(c, r.b.sp(), cimm(fac1), fbe.sp(), cimm(fac2), h.sp()));
  }
  cudaEvent_t e0, e1;
  QQ_CK(cudaEventCreate(&e0));
  QQ_CK(cudaEventCreate(&e1));
  auto tic = [&]() { cudaEventRecord(e0, c->st); };
  auto toc = [&]() {
    cudaEventRecord(e1, c->st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms * 1e-3;
  };
  int rc = QQ_OK;
  const int maxiter = meth->max_outer > 0 ? 1000 * meth->max_outer : 200000;
  if (meth->solver == 0) {
    for (int i = 0; i < nrhs && rc == QQ_OK; ++i) {
      tic();
      status[i] = gmresdr_fp64(c, R[i]->b.sp(), R[i]->x.sp(), meth->m, meth->k, tol_even, 0, kappa,
                               nullptr, &stats[i]);
      seconds[i] = toc();
      if (status[i] != QQ_OK && status[i] != QQ_NOT_CONVERGED) rc = status[i];
    }
  } else {
    DeflSpace defl;
    double defl_sec = 0.0;
    if (meth->deflate) {
      // deflation space from the first right-hand side; its partial solution is kept
      // as that right-hand side's initial guess
      tic();
      const double dt = meth->defl_tol > 0.0 ? meth->defl_tol : 1e-5;
      const int st0 = gmresdr_mixed(c, R[0]->b.sp(), R[0]->x.sp(), meth->m, meth->k, std::max(dt, tol_even),
                                    200, kappa, &defl, &stats[0]);
      defl_sec = toc();
      if (st0 != QQ_OK && st0 != QQ_NOT_CONVERGED) rc = st0;
    }
    for (int i0 = 0; i0 < nrhs && rc == QQ_OK; i0 += block) {
      const int nb = std::min(block, nrhs - i0);
      std::vector<PerRhs*> blk;
      std::vector<SolveStats> bst(nb);
      for (int k = 0; k < nb; ++k) {
        PerRhs& r = *R[i0 + k];
        QQ_TRY(alloc_field(c, r.r, prec));
        QQ_TRY(alloc_field(c, r.rhat, prec));
        QQ_TRY(alloc_field(c, r.p, prec));
        QQ_TRY(alloc_field(c, r.v, prec));
        QQ_TRY(alloc_field(c, r.t, prec));
        QQ_TRY(alloc_field(c, r.xl, prec));
        QQ_TRY(alloc_field(c, r.tmp, prec));
        blk.push_back(&r);
      }
      tic();
      const int st = bicgstab_mixed_batch(c, blk, prec, tol_even, 0.1, maxiter, kappa,
                                          defl.k > 0 ? &defl : nullptr, bst);
      const double sec = toc();
      for (int k = 0; k < nb; ++k) {
        // the deflation-building solve is charged to the first right-hand side
        if (i0 + k == 0 && meth->deflate) {
          bst[k].itercount += stats[0].itercount;
          bst[k].mvp += stats[0].mvp;
          bst[k].ritz = stats[0].ritz;
        }
        stats[i0 + k] = bst[k];
        seconds[i0 + k] = sec / nb + (i0 + k == 0 ? defl_sec : 0.0);
        status[i0 + k] = blk[k]->done ? QQ_OK : QQ_NOT_CONVERGED;
      }
      if (st != QQ_OK && st != QQ_NOT_CONVERGED) rc = st;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != QQ_OK) return rc;
  // odd reconstruction, full-lattice residual, output
  Tmp fxo(c, P64);
  for (int i = 0; i < nrhs; ++i) {
    PerRhs& r = *R[i];
    const double* de = nullptr;
    const double* dO = nullptr;
    QQ_TRY(stage_in(c, 1, be + (size_t)i * nv, nv, &de));
    QQ_TRY(ref_to_field(c, de, 0, fbe.sp()));
    QQ_TRY(stage_in(c, 2, bo + (size_t)i * nv, nv, &dO));
    QQ_TRY(ref_to_field(c, dO, 1, fbo.sp()));
    QQ_TRY(op_hsingle(c, h.sp(), r.x.sp(), 0, 1));
    const double f = 1.0 / (1.0 + tk * tk);
    QQ_CK(launch_spinmix(c->g.vh, fbo.sp(), h.sp(), fxo.sp(), f, -tk * f, f * kappa[0], -tk * f * kappa[0], P64, c->st));
    double rel = 0.0;
    QQ_TRY(full_residual(c, fbe.sp(), fbo.sp(), r.x.sp(), fxo.sp(), kappa, &rel));
    stats[i].true_rel = rel;
    if (rel > meth->tol && status[i] == QQ_OK) status[i] = QQ_NOT_CONVERGED;
    double* dxe = nullptr;
    double* dxo = nullptr;
    QQ_TRY(stage_out_begin(c, 1, xe + (size_t)i * nv, nv, &dxe));
    QQ_TRY(field_to_ref(c, r.x.sp(), 0, dxe));
    QQ_TRY(stage_out_end(c, 1, xe + (size_t)i * nv, nv, dxe));
    QQ_TRY(stage_out_begin(c, 2, xo + (size_t)i * nv, nv, &dxo));
    QQ_TRY(field_to_ref(c, fxo.sp(), 1, dxo));
    QQ_TRY(stage_out_end(c, 2, xo + (size_t)i * nv, nv, dxo));
    QQ_CK(cudaStreamSynchronize(c->st));
    if (infos) fill_info(&infos[i], status[i], stats[i], seconds[i]);
  }
  for (int i = 0; i < nrhs; ++i)
    if (status[i] != QQ_OK) return QQ_NOT_CONVERGED;
  return QQ_OK;
}

int traces_level0(qq_ctx* c, const double* be, const double* bo, const double* xe,
                  const double* xo, double kappa, double* J) {
  (void)c; (void)be; (void)bo; (void)xe; (void)xo; (void)kappa; (void)J;
  return set_error(QQ_BAD_ARG, "traces not built yet");
}

}  // namespace qq
