// Krylov solvers of the reference's inverters module, on the GPU.
//
//   GMRES-DR(m,k)   Q/inverters.f90:2871-3572  (Morgan 2002)
//   GMRES-Proj      Q/inverters.f90:7183-8304
//   GMRES-DR-shift  Q/inverters.f90:6041-7179 (multi-shift, on gamma5mult)
//   BiCGStab        Q/inverters.f90:302-487
//
// The Krylov basis lives in HBM in the GPU spinor layout.  Arnoldi orthogonalisation
// is classical Gram-Schmidt with one re-orthogonalisation (CGS2): each pass is one
// multi-vector kernel over the whole basis instead of the reference's j separate
// vecdot/axpy sweeps (modified Gram-Schmidt); both are backward stable to FP64.
// The Hessenberg matrix is built on the device; the host reads it once per cycle for
// the least-squares solve and the harmonic-Ritz restart, which is where the reference
// checks convergence with the true residual anyway.
#include <cmath>
#include <functional>
#include <cstring>

#include "qq_ctx.h"

namespace qq {

namespace {

constexpr int kCycleLimit = 5000;  // kcyclim, U/latdims.f90:70
constexpr int kMaxShifts = 512;   // per-shift norms live in the 1024-double scalar buffer

struct Arnoldi {
  qq_ctx* c;
  int pb;
  int m;         // Krylov dimension (m+1 vectors)
  size_t nel;    // 16-byte elements per vector
  DevBuf V, H, hscr, y;
  DevBuf Pdev;  // restart rotation ((m+1) x (k+1), k < m), allocated once
  // Krylov operator: Hdbletm, or gamma5mult - g5shift (gmresdrshift)
  bool g5 = false;
  double g5shift = 0.0;
  int init(qq_ctx* c_, int pb_, int m_) {
    c = c_;
    pb = pb_;
    m = m_;
    nel = (pb == P64 ? (size_t)12 : (size_t)6) * c->g.vh;
    QQ_CK(V.alloc((size_t)(m + 1) * nel * 16));
    QQ_CK(H.alloc(sizeof(double) * 2 * (size_t)(m + 1) * m));
    QQ_CK(hscr.alloc(sizeof(double) * 2 * 128));
    QQ_CK(y.alloc(sizeof(double) * 2 * 256));
    QQ_CK(Pdev.alloc(sizeof(double) * 2 * (size_t)(m + 1) * m));
    return QQ_OK;
  }
  void* vec(int i) const { return static_cast<char*>(V.p) + (size_t)i * nel * 16; }
  Spinor sp(int i) const { return Spinor{vec(i), nullptr, pb}; }
  BasisArgs basis() const { return BasisArgs{V.p, nel, nel}; }
  double* col(int j) const { return H.as<double>() + 2 * (size_t)(m + 1) * j; }
  int zeroH() {
    QQ_CK(cudaMemsetAsync(H.p, 0, H.bytes, c->st));
    return QQ_OK;
  }
};

// One Arnoldi step: v_{j+1} = normalised (I - V V^H) A src, H(:, j) filled; src = v_j
// for GMRES, the preconditioned z_j = M v_j for flexible GMRES.
int arnoldi_step_from(Arnoldi& A, int j, Spinor src, Spinor tmp_odd, const double kappa[2], double* nrm2_slot) {
  qq_ctx* c = A.c;
  if (A.g5)
    QQ_TRY(op_g5mult(c, A.sp(j + 1), src, tmp_odd, 0, kappa, A.g5shift));
  else
    QQ_TRY(op_dbletm(c, A.sp(j + 1), src, tmp_odd, 0, kappa));
  double* part = c->partial.as<double>();
  const int nv = j + 1;
  int ng = 0;
  BasisArgs B = A.basis();
  double* hcol = A.col(j);
  double* hscr = A.hscr.as<double>();
  void* w = A.vec(j + 1);
  QQ_CK(launch_multidot(A.pb, B, nv, w, part, &ng, c->st));
  QQ_CK(launch_finalize(part, kRedBlocks, ng * 16, 2 * nv, hcol, 0, c->st));
  QQ_CK(launch_multiaxpy(A.pb, B, nv, hcol, 1.0, w, w, part, c->st));
  QQ_CK(launch_multidot(A.pb, B, nv, w, part, &ng, c->st));
  QQ_CK(launch_finalize(part, kRedBlocks, ng * 16, 2 * nv, hscr, 0, c->st));
  QQ_CK(launch_multiaxpy(A.pb, B, nv, hscr, 1.0, w, w, part, c->st));
  QQ_CK(launch_finalize(part, kRedBlocks, 3, 1, nrm2_slot, 0, c->st));
  QQ_CK(launch_hcol_update(A.H.as<double>(), A.m + 1, j, hscr, nv, nrm2_slot, c->st));
  QQ_CK(launch_normalize(A.pb, A.nel, w, w, nrm2_slot, c->st));
  return QQ_OK;
}

int arnoldi_step(Arnoldi& A, int j, Spinor tmp_odd, const double kappa[2], double* nrm2_slot) {
  return arnoldi_step_from(A, j, A.sp(j), tmp_odd, kappa, nrm2_slot);
}

// Re-orthogonalise vector `idx` of the basis against vectors [0, idx) and normalise.
int reorth(Arnoldi& A, int idx, double* nrm2_slot) {
  qq_ctx* c = A.c;
  double* part = c->partial.as<double>();
  double* hscr = A.hscr.as<double>();
  BasisArgs B = A.basis();
  void* w = A.vec(idx);
  int ng = 0;
  for (int pass = 0; pass < 2; ++pass) {
    QQ_CK(launch_multidot(A.pb, B, idx, w, part, &ng, c->st));
    QQ_CK(launch_finalize(part, kRedBlocks, ng * 16, 2 * idx, hscr, 0, c->st));
    QQ_CK(launch_multiaxpy(A.pb, B, idx, hscr, 1.0, w, w, part, c->st));
  }
  QQ_CK(launch_finalize(part, kRedBlocks, 3, 1, nrm2_slot, 0, c->st));
  QQ_CK(launch_normalize(A.pb, A.nel, w, w, nrm2_slot, c->st));
  return QQ_OK;
}

int read_H(Arnoldi& A, int ncols, dense::Mat& Hb) {
  std::vector<double> h(2 * (size_t)(A.m + 1) * A.m);
  QQ_CK(cudaMemcpyAsync(h.data(), A.H.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, A.c->st));
  QQ_CK(cudaStreamSynchronize(A.c->st));
  Hb = dense::Mat(ncols + 1, ncols);
  for (int j = 0; j < ncols; ++j)
    for (int i = 0; i <= ncols; ++i)
      Hb(i, j) = {h[2 * ((size_t)i + (size_t)(A.m + 1) * j)], h[2 * ((size_t)i + (size_t)(A.m + 1) * j) + 1]};
  return QQ_OK;
}

int upload_cvec(qq_ctx* c, const std::vector<dense::cd>& v, double* dev) {
  std::vector<double> h(2 * v.size());
  for (size_t i = 0; i < v.size(); ++i) {
    h[2 * i] = v[i].real();
    h[2 * i + 1] = v[i].imag();
  }
  QQ_CK(cudaMemcpyAsync(dev, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));  // h goes out of scope
  return QQ_OK;
}

int upload_mat(qq_ctx* c, const dense::Mat& M, double* dev, int ld) {
  std::vector<double> h(2 * (size_t)ld * M.n, 0.0);
  for (int j = 0; j < M.n; ++j)
    for (int i = 0; i < M.m; ++i) {
      h[2 * ((size_t)i + (size_t)ld * j)] = M(i, j).real();
      h[2 * ((size_t)i + (size_t)ld * j) + 1] = M(i, j).imag();
    }
  QQ_CK(cudaMemcpyAsync(dev, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

// r = b - A x with ||r||^2 read back
int true_residual(qq_ctx* c, Spinor b, Spinor x, Spinor r, Spinor tmp_odd, const double kappa[2],
                  double* nrm) {
  Tmp h(c, x.prec);
  QQ_TRY(op_dbletm(c, h.sp(), x, tmp_odd, 0, kappa));
  double* s = c->scal.as<double>();
  QQ_TRY(lin(c, r, cimm(1.0), b, cimm(-1.0), h.sp(), cimm(0), Spinor{nullptr, nullptr, P64}, s));
  double n2;
  QQ_TRY(read_scalars(c, s, 1, &n2));
  *nrm = std::sqrt(n2);
  return QQ_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Flexible GMRES(m) with a right preconditioner z = M(v) (Saad 1993): Arnoldi on
// A z_j with z_j = M(v_j), A Z_m = V_{m+1} H_m, update x += Z_m y with y the
// least-squares solution of H_m y = ||r|| e_1.  M may change between applications
// (the network runs in FP32).  FP64 basis; the true residual is checked once per
// cycle against ||phi - A x0||, as GMRES-DR.  *stalled is set when two consecutive
// cycles each reduce the true residual by less than a factor 2.
// ---------------------------------------------------------------------------
int fgmres_fp64(qq_ctx* c, Spinor phi, Spinor x, int m, double resmax, int max_cycles, const double kappa[2],
                const std::function<int(Spinor, Spinor)>& M, SolveStats* st, bool* stalled) {
  if (m < 2 || m > 127) return set_error(QQ_BAD_ARG, "FGMRES(m) out of range");
  *stalled = false;
  Arnoldi A;
  QQ_TRY(A.init(c, P64, m));
  DevBuf Z;
  QQ_CK(Z.alloc((size_t)m * A.nel * 16));
  auto zsp = [&](int j) { return Spinor{static_cast<char*>(Z.p) + (size_t)j * A.nel * 16, nullptr, P64}; };
  Tmp tmp(c, P64), r(c, P64);
  double* nrm2 = c->scal.as<double>() + 8;
  double normnum = 0.0;
  QQ_TRY(true_residual(c, phi, x, r.sp(), tmp.sp(), kappa, &normnum));
  st->mvp += 1;
  if (!std::isfinite(normnum)) return set_error(QQ_NAN, "NaN in initial residual");
  if (!(normnum > 0.0)) {
    st->true_rel = 0.0;
    return QQ_OK;
  }
  double rn = normnum, prev = 1.0;
  int slow = 0;
  for (int cyc = 1; cyc <= max_cycles; ++cyc) {
    QQ_TRY(lin(c, A.sp(0), cimm(1.0 / rn), r.sp()));
    std::vector<dense::cd> cvec(m + 1, 0.0);
    cvec[0] = rn;
    QQ_TRY(A.zeroH());
    for (int j = 0; j < m; ++j) {
      QQ_TRY(M(zsp(j), A.sp(j)));
      QQ_TRY(arnoldi_step_from(A, j, zsp(j), tmp.sp(), kappa, nrm2));
      st->itercount += 1;
      st->mvp += 1;
    }
    dense::Mat Hb;
    QQ_TRY(read_H(A, m, Hb));
    std::vector<dense::cd> y, srv;
    dense::hess_lsq(Hb, cvec, m, y, srv);
    QQ_TRY(upload_cvec(c, y, A.y.as<double>()));
    QQ_CK(launch_basis_accum(P64, BasisArgs{Z.p, A.nel, A.nel}, m, A.y.as<double>(), c->g.vh, x, c->st));
    QQ_TRY(true_residual(c, phi, x, r.sp(), tmp.sp(), kappa, &rn));
    st->mvp += 1;
    const double rel = rn / normnum;
    st->hist.push_back(rel);
    st->hist_mvp.push_back(st->mvp);
    st->true_rel = rel;
    st->ncycles = cyc;
    if (!std::isfinite(rel)) return set_error(QQ_NAN, "NaN residual in flexible GMRES");
    if (rel < resmax) return QQ_OK;
    slow = rel > 0.5 * prev ? slow + 1 : 0;
    prev = rel;
    if (slow >= 2) {
      *stalled = true;
      break;
    }
  }
  return QQ_NOT_CONVERGED;
}

// ---------------------------------------------------------------------------
// Flexible GMRES-DR(m, k): flexible GMRES with Morgan's deflated restarts.  The
// Arnoldi relation A Z_m = V_{m+1} Hbar_m holds with the preconditioned directions
// Z stored in FP64, so x = x0 + Z y is consistent with the FP64 residual however
// M is computed.  At a restart the harmonic Ritz step of GMRES-DR gives P; the bases
// rotate together, V_{k+1} <- V_{m+1} P and Z_k <- Z_m P(0:m, 0:k) (P's first k
// columns vanish in row m + 1), and the next cycle continues from column k, so the
// k smallest harmonic Ritz directions of A M stay in the space.  *stalled is set after
// three consecutive cycles that each gain less than 10% (the first cycles of a
// deflated method near the critical kappa are slow while its eigenvector space forms).
// ---------------------------------------------------------------------------
int fgmresdr_fp64(qq_ctx* c, Spinor phi, Spinor x, int m, int k, double resmax, int max_cycles,
                  const double kappa[2], const std::function<int(Spinor, Spinor)>& M, SolveStats* st,
                  bool* stalled) {
  if (m < 2 || k < 1 || k >= m || m > 127) return set_error(QQ_BAD_ARG, "FGMRES-DR(m,k) out of range");
  *stalled = false;
  Arnoldi A;
  QQ_TRY(A.init(c, P64, m));
  DevBuf Z;
  QQ_CK(Z.alloc((size_t)m * A.nel * 16));
  auto zsp = [&](int j) { return Spinor{static_cast<char*>(Z.p) + (size_t)j * A.nel * 16, nullptr, P64}; };
  Tmp tmp(c, P64), r(c, P64);
  double* nrm2 = c->scal.as<double>() + 8;
  double normnum = 0.0;
  QQ_TRY(true_residual(c, phi, x, r.sp(), tmp.sp(), kappa, &normnum));
  st->mvp += 1;
  if (!std::isfinite(normnum)) return set_error(QQ_NAN, "NaN in initial residual");
  if (!(normnum > 0.0)) {
    st->true_rel = 0.0;
    return QQ_OK;
  }
  QQ_TRY(lin(c, A.sp(0), cimm(1.0 / normnum), r.sp()));
  std::vector<dense::cd> cvec(m + 1, 0.0);
  cvec[0] = normnum;
  QQ_TRY(A.zeroH());
  int j0 = 0, slow = 0;
  double prev = 1.0;
  for (int cyc = 1; cyc <= max_cycles; ++cyc) {
    for (int j = j0; j < m; ++j) {
      QQ_TRY(M(zsp(j), A.sp(j)));
      QQ_TRY(arnoldi_step_from(A, j, zsp(j), tmp.sp(), kappa, nrm2));
      st->itercount += 1;
      st->mvp += 1;
    }
    dense::Mat Hb;
    QQ_TRY(read_H(A, m, Hb));
    std::vector<dense::cd> y, srv;
    dense::hess_lsq(Hb, cvec, m, y, srv);
    QQ_TRY(upload_cvec(c, y, A.y.as<double>()));
    const BasisArgs ZB{Z.p, A.nel, A.nel};
    QQ_CK(launch_basis_accum(P64, ZB, m, A.y.as<double>(), c->g.vh, x, c->st));
    double rn = 0.0;
    QQ_TRY(true_residual(c, phi, x, r.sp(), tmp.sp(), kappa, &rn));
    st->mvp += 1;
    const double rel = rn / normnum;
    st->hist.push_back(rel);
    st->hist_mvp.push_back(st->mvp);
    st->true_rel = rel;
    st->ncycles = cyc;
    if (!std::isfinite(rel)) return set_error(QQ_NAN, "NaN residual in flexible GMRES-DR");
    if (rel < resmax) return QQ_OK;
    slow = rel > 0.9 * prev ? slow + 1 : 0;  // deflation needs a few slow cycles to build up
    prev = rel;
    if (slow >= 3) {
      *stalled = true;
      return QQ_NOT_CONVERGED;
    }
    dense::Mat P, Hk;
    std::vector<dense::cd> cnew, ritz;
    if (!dense::gmresdr_restart(Hb, srv, m, k, P, Hk, cnew, ritz)) {
      *stalled = true;  // no usable harmonic Ritz step: let plain GMRES-DR continue
      return QQ_NOT_CONVERGED;
    }
    st->ritz = ritz;
    QQ_TRY(upload_mat(c, P, A.Pdev.as<double>(), m + 1));
    QQ_CK(launch_rotate(P64, A.basis(), m + 1, k + 1, A.Pdev.as<double>(), m + 1, c->st));
    QQ_CK(launch_rotate(P64, ZB, m, k, A.Pdev.as<double>(), m + 1, c->st));
    QQ_TRY(reorth(A, k, nrm2));
    QQ_TRY(A.zeroH());
    QQ_TRY(upload_mat(c, Hk, A.H.as<double>(), m + 1));
    std::fill(cvec.begin(), cvec.end(), 0.0);
    for (int i = 0; i <= k; ++i) cvec[i] = cnew[i];
    j0 = k;
  }
  return QQ_NOT_CONVERGED;
}

// ---------------------------------------------------------------------------
// GMRES-DR(m, k), FP64, reference semantics: convergence is tested once per cycle with
// the true residual ||phi - A x|| / ||phi - A x0|| < resmax (inverters.f90:3270-3298).
// ---------------------------------------------------------------------------
int gmresdr_fp64(qq_ctx* c, Spinor phi, Spinor x, int m, int k, double resmax, int itermin,
                 const double kappa[2], DeflSpace* defl, SolveStats* st) {
  if (m < 2 || k < 1 || k >= m || m > 127) return set_error(QQ_BAD_ARG, "GMRES(n,k) out of range");
  Arnoldi A;
  QQ_TRY(A.init(c, P64, m));
  Tmp tmp(c, P64), r(c, P64);
  double* nrm2 = c->scal.as<double>() + 8;
  double normnum = 0.0;
  QQ_TRY(true_residual(c, phi, x, r.sp(), tmp.sp(), kappa, &normnum));
  st->mvp = 1;
  if (!(normnum > 0.0) || !std::isfinite(normnum)) {
    st->true_rel = 0.0;
    return std::isfinite(normnum) ? QQ_OK : set_error(QQ_NAN, "NaN in initial residual");
  }
  QQ_TRY(lin(c, A.sp(0), cimm(1.0 / normnum), r.sp()));
  std::vector<dense::cd> cvec(m + 1, 0.0);
  cvec[0] = normnum;
  QQ_TRY(A.zeroH());
  int j0 = 0, icycle = 1, status = QQ_NOT_CONVERGED;
  dense::Mat Hk_last;
  bool restarted = false;
  for (;;) {
    for (int j = j0; j < m; ++j) {
      QQ_TRY(arnoldi_step(A, j, tmp.sp(), kappa, nrm2));
      st->itercount += 1;
      st->mvp += 1;
    }
    dense::Mat Hb;
    QQ_TRY(read_H(A, m, Hb));
    std::vector<dense::cd> y, srv;
    dense::hess_lsq(Hb, cvec, m, y, srv);
    QQ_TRY(upload_cvec(c, y, A.y.as<double>()));
    QQ_CK(launch_basis_accum(P64, A.basis(), m, A.y.as<double>(), c->g.vh, x, c->st));
    double rn = 0.0;
    QQ_TRY(true_residual(c, phi, x, r.sp(), tmp.sp(), kappa, &rn));
    st->mvp += 1;
    const double rel = rn / normnum;
    st->hist.push_back(rel);
    st->hist_mvp.push_back(st->mvp);
    st->true_rel = rel;
    st->ncycles = icycle;
    if (!std::isfinite(rel)) {
      status = set_error(QQ_NAN, "NaN residual in gmresdr");
      break;
    }
    if (rel < resmax && st->itercount >= itermin) {
      status = QQ_OK;
      break;
    }
    if (icycle >= kCycleLimit) break;
    dense::Mat P, Hk;
    std::vector<dense::cd> cnew, ritz;
    if (!dense::gmresdr_restart(Hb, srv, m, k, P, Hk, cnew, ritz)) {
      status = set_error(QQ_SINGULAR, "harmonic Ritz step failed");
      break;
    }
    st->ritz = ritz;
    QQ_TRY(upload_mat(c, P, A.Pdev.as<double>(), m + 1));
    QQ_CK(launch_rotate(P64, A.basis(), m + 1, k + 1, A.Pdev.as<double>(), m + 1, c->st));
    QQ_TRY(reorth(A, k, nrm2));
    QQ_TRY(A.zeroH());
    QQ_TRY(upload_mat(c, Hk, A.H.as<double>(), m + 1));
    std::fill(cvec.begin(), cvec.end(), 0.0);
    for (int i = 0; i <= k; ++i) cvec[i] = cnew[i];
    Hk_last = Hk;
    restarted = true;
    j0 = k;
    icycle += 1;
  }
  if (defl && restarted) {
    defl->k = k;
    defl->pb = P64;
    defl->nel = A.nel;
    QQ_CK(defl->V.alloc((size_t)(k + 1) * A.nel * 16));
    QQ_CK(cudaMemcpyAsync(defl->V.p, A.V.p, (size_t)(k + 1) * A.nel * 16, cudaMemcpyDeviceToDevice, c->st));
    defl->Hk = Hk_last;
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return status;
}

// ---------------------------------------------------------------------------
// Multi-shift GMRES-DR (gmresdrshift, inverters.f90:6041-7179; Darnell, Morgan and
// Wilcox 2008): (A - sigma_s) x_s = b for every shift s, A = gamma5mult.  Arnoldi and
// the deflated restart run on A - sigma_0.  At the end of each cycle the base system
// takes the least-squares solution y, and each further shift solves
//   [Hbar + (sigma_0 - sigma_s) I~ | srv] (d_s, alpha_s) = cmult_s c      (:6576-6747)
// so that its residual stays alpha_s times the base residual; cmult_s <- alpha_s.
// Each x_s += V d_s and r_s -= (A - sigma_s) V d_s (:6816-6830).  Stops when
// ||r_0|| < resmax (absolute, :6865).  Zero initial guess for every shift.
// ---------------------------------------------------------------------------
int gmresdrshift_fp64(qq_ctx* c, Spinor b, const std::vector<Spinor>& xs, const std::vector<Spinor>& rs,
                      const double* sigma, int m, int k, double resmax, int itermin, const double kappa[2],
                      double* resid, SolveStats* st) {
  const int ns = (int)xs.size();
  if (m < 2 || k < 1 || k >= m || m > 127) return set_error(QQ_BAD_ARG, "GMRES(n,k) out of range");
  constexpr int kNormSlot = 32;  // per-shift ||r_s||^2 in c->scal[32 .. 32 + ns)
  if (ns < 1 || ns > kMaxShifts || (int)rs.size() != ns)
    return set_error(QQ_BAD_ARG, "nshifts must be in 1..512");
  Arnoldi A;
  QQ_TRY(A.init(c, P64, m));
  A.g5 = true;
  A.g5shift = sigma[0];
  Tmp tmp(c, P64), xb(c, P64), h(c, P64);
  double* nrm2 = c->scal.as<double>() + 8;
  double* s = c->scal.as<double>();
  double n2 = 0.0;
  QQ_TRY(lin(c, A.sp(0), cimm(1.0), b, cimm(0), Spinor{nullptr, nullptr, P64}, cimm(0),
             Spinor{nullptr, nullptr, P64}, s));
  QQ_TRY(read_scalars(c, s, 1, &n2));
  const double normnum = std::sqrt(n2);
  for (int q = 0; q < ns; ++q) {
    QQ_TRY(zero_field(c, xs[q]));
    QQ_TRY(lin(c, rs[q], cimm(1.0), b));
    resid[q] = normnum;
  }
  if (!std::isfinite(normnum)) return set_error(QQ_NAN, "NaN in the right-hand side");
  if (!(normnum > 0.0)) return QQ_OK;
  QQ_TRY(lin(c, A.sp(0), cimm(1.0 / normnum), A.sp(0)));
  std::vector<dense::cd> cvec(m + 1, 0.0), cmult(ns, 1.0);
  cvec[0] = normnum;
  QQ_TRY(A.zeroH());
  int j0 = 0, icycle = 1, status = QQ_NOT_CONVERGED;
  for (;;) {
    for (int j = j0; j < m; ++j) {
      QQ_TRY(arnoldi_step(A, j, tmp.sp(), kappa, nrm2));
      st->itercount += 1;
      st->mvp += 1;
    }
    dense::Mat Hb;
    QQ_TRY(read_H(A, m, Hb));
    std::vector<dense::cd> y, srv;
    dense::hess_lsq(Hb, cvec, m, y, srv);
    for (int q = 0; q < ns; ++q) {
      std::vector<dense::cd> d;
      if (q == 0) {
        d = y;
      } else {
        dense::Mat M(m + 1, m + 1);
        for (int jj = 0; jj < m; ++jj)
          for (int i = 0; i <= m; ++i) M(i, jj) = Hb(i, jj);
        for (int jj = 0; jj < m; ++jj) M(jj, jj) += sigma[0] - sigma[q];
        for (int i = 0; i <= m; ++i) M(i, m) = srv[i];
        std::vector<dense::cd> rhs(m + 1);
        for (int i = 0; i <= m; ++i) rhs[i] = cmult[q] * cvec[i];
        if (!dense::lu_solve(M, rhs)) return set_error(QQ_SINGULAR, "shifted collinear system singular");
        d.assign(rhs.begin(), rhs.begin() + m);
        cmult[q] = rhs[m];
      }
      QQ_TRY(upload_cvec(c, d, A.y.as<double>()));
      QQ_TRY(zero_field(c, xb.sp()));
      QQ_CK(launch_basis_accum(P64, A.basis(), m, A.y.as<double>(), c->g.vh, xb.sp(), c->st));
      QQ_TRY(lin(c, xs[q], cimm(1.0), xs[q], cimm(1.0), xb.sp()));
      QQ_TRY(op_g5mult(c, h.sp(), xb.sp(), tmp.sp(), 0, kappa, sigma[q]));
      st->mvp += 1;
      QQ_TRY(lin(c, rs[q], cimm(1.0), rs[q], cimm(-1.0), h.sp(), cimm(0), Spinor{nullptr, nullptr, P64},
                 s + kNormSlot + q));
    }
    std::vector<double> r2(ns);
    QQ_TRY(read_scalars(c, s + kNormSlot, ns, r2.data()));
    for (int q = 0; q < ns; ++q) resid[q] = std::sqrt(r2[q]);
    const double rel = resid[0] / normnum;
    st->hist.push_back(rel);
    st->hist_mvp.push_back(st->mvp);
    st->true_rel = rel;
    st->ncycles = icycle;
    if (!std::isfinite(resid[0])) {
      status = set_error(QQ_NAN, "NaN residual in gmresdrshift");
      break;
    }
    if (resid[0] < resmax && st->itercount >= itermin) {
      status = QQ_OK;
      break;
    }
    if (icycle >= kCycleLimit) break;
    dense::Mat P, Hk;
    std::vector<dense::cd> cnew, ritz;
    if (!dense::gmresdr_restart(Hb, srv, m, k, P, Hk, cnew, ritz)) {
      status = set_error(QQ_SINGULAR, "harmonic Ritz step failed");
      break;
    }
    st->ritz = ritz;
    QQ_TRY(upload_mat(c, P, A.Pdev.as<double>(), m + 1));
    QQ_CK(launch_rotate(P64, A.basis(), m + 1, k + 1, A.Pdev.as<double>(), m + 1, c->st));
    QQ_TRY(reorth(A, k, nrm2));
    QQ_TRY(A.zeroH());
    QQ_TRY(upload_mat(c, Hk, A.H.as<double>(), m + 1));
    std::fill(cvec.begin(), cvec.end(), 0.0);
    for (int i = 0; i <= k; ++i) cvec[i] = cnew[i];
    j0 = k;
    icycle += 1;
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return status;
}

// ---------------------------------------------------------------------------
// GMRES-Proj (inverters.f90:7183-8304, sigma = 0): every cycle first minimises the
// residual over the deflation space, then runs GMRES(m).  Zero initial guess;
// stops when ||b - A x|| / ||b|| <= resmax after a GMRES cycle.
// ---------------------------------------------------------------------------
int gmresproj_fp64(qq_ctx* c, Spinor b, Spinor x, int m, int k, double resmax, int itermin,
                   const double kappa[2], const DeflSpace& defl, SolveStats* st) {
  if (defl.k <= 0) return set_error(QQ_BAD_ARG, "empty deflation space");
  if (defl.k != k) return set_error(QQ_BAD_ARG, "deflation space size differs from k");
  if (m < 1 || m > 127) return set_error(QQ_BAD_ARG, "GMRES(n) out of range");
  (void)itermin;
  Arnoldi A;
  QQ_TRY(A.init(c, P64, m));
  Tmp tmp(c, P64), r(c, P64);
  double* nrm2 = c->scal.as<double>() + 8;
  QQ_TRY(zero_field(c, x));
  double rinit = 0.0;
  QQ_TRY(norm2_host(c, b, &rinit));
  rinit = std::sqrt(rinit);
  st->mvp = 2;  // the reference applies the operator twice to the zero start
  if (!(rinit > 0.0)) return QQ_OK;
  QQ_TRY(copy_field(c, r.sp(), b));
  double rn = rinit;
  BasisArgs D{defl.V.p, defl.nel, defl.nel};
  DevBuf cd;
  QQ_CK(cd.alloc(sizeof(double) * 2 * 256));
  int icycle = 1, status = QQ_NOT_CONVERGED;
  for (;;) {
    if (rn / rinit <= resmax) {
      status = QQ_OK;
      break;
    }
    if (icycle > kCycleLimit) break;
    // projection: min || c - Hk y ||, c = Vdefl^H r
    int ng = 0;
    double* part = c->partial.as<double>();
    QQ_CK(launch_multidot(defl.pb, D, k + 1, r.sp().data, part, &ng, c->st));
    QQ_CK(launch_finalize(part, kRedBlocks, ng * 16, 2 * (k + 1), cd.as<double>(), 0, c->st));
    std::vector<double> ch(2 * (k + 1));
    QQ_TRY(read_scalars(c, cd.as<double>(), 2 * (k + 1), ch.data()));
    std::vector<dense::cd> cv(k + 1);
    for (int i = 0; i <= k; ++i) cv[i] = {ch[2 * i], ch[2 * i + 1]};
    std::vector<dense::cd> yp, srvp;
    dense::hess_lsq(defl.Hk, cv, k, yp, srvp);
    QQ_TRY(upload_cvec(c, yp, A.y.as<double>()));
    QQ_CK(launch_basis_accum(defl.pb, D, k, A.y.as<double>(), c->g.vh, x, c->st));
    double beta = 0.0;
    QQ_TRY(true_residual(c, b, x, r.sp(), tmp.sp(), kappa, &beta));
    if (!std::isfinite(beta)) return set_error(QQ_NAN, "NaN residual in gmresproj");
    QQ_TRY(lin(c, A.sp(0), cimm(1.0 / beta), r.sp()));
    std::vector<dense::cd> cvec(m + 1, 0.0);
    cvec[0] = beta;
    QQ_TRY(A.zeroH());
    for (int j = 0; j < m; ++j) {
      QQ_TRY(arnoldi_step(A, j, tmp.sp(), kappa, nrm2));
      st->itercount += 1;
      st->mvp += 1;
    }
    dense::Mat Hb;
    QQ_TRY(read_H(A, m, Hb));
    std::vector<dense::cd> y, srv;
    dense::hess_lsq(Hb, cvec, m, y, srv);
    QQ_TRY(upload_cvec(c, y, A.y.as<double>()));
    QQ_CK(launch_basis_accum(P64, A.basis(), m, A.y.as<double>(), c->g.vh, x, c->st));
    QQ_TRY(true_residual(c, b, x, r.sp(), tmp.sp(), kappa, &rn));
    st->mvp += 1;
    st->hist.push_back(rn / rinit);
    st->hist_mvp.push_back(st->mvp);
    st->true_rel = rn / rinit;
    st->ncycles = icycle;
    if (!std::isfinite(rn)) return set_error(QQ_NAN, "NaN residual in gmresproj");
    // the next projection acts on the least-squares residual V_{m+1} srv
    QQ_TRY(zero_field(c, r.sp()));
    QQ_TRY(upload_cvec(c, srv, A.y.as<double>()));
    QQ_CK(launch_basis_accum(P64, A.basis(), m + 1, A.y.as<double>(), c->g.vh, r.sp(), c->st));
    icycle += 1;
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return status;
}

// ---------------------------------------------------------------------------
// Mixed-precision GMRES-DR(m, k): the Arnoldi process (operator, Krylov basis, Gram-
// Schmidt) runs in FP32 with FP64 reductions; the solution accumulates in FP64 and
// every cycle ends with the FP64 true residual r = b - A x.  The next cycle starts
// from the harmonic-Ritz basis V_{k+1} of the restart with the least-squares
// right-hand side c = V_{k+1}^H r (the projection of the FP64 residual), so rounding
// of the FP32 cycle never accumulates into the answer.  Returns the FP32 deflation
// space (V_{k+1}, Hk) of the last restart for the other right-hand sides.
// ---------------------------------------------------------------------------
int gmresdr_mixed(qq_ctx* c, Spinor b, Spinor x, int m, int k, double tol, int max_cycles,
                  const double kappa[2], DeflSpace* defl, SolveStats* st) {
  if (m < 2 || k < 1 || k >= m || m > 127) return set_error(QQ_BAD_ARG, "GMRES(n,k) out of range");
  Arnoldi A;
  QQ_TRY(A.init(c, P32, m));
  Tmp tmp32(c, P32), tmp64(c, P64), r(c, P64), r32(c, P32);
  double* nrm2 = c->scal.as<double>() + 8;
  double bn = 0.0;
  QQ_TRY(norm2_host(c, b, &bn));
  bn = std::sqrt(bn);
  double rn = 0.0;
  QQ_TRY(true_residual(c, b, x, r.sp(), tmp64.sp(), kappa, &rn));
  st->mvp += 1;
  if (!(bn > 0.0)) return QQ_OK;
  if (!std::isfinite(rn)) return set_error(QQ_NAN, "NaN in initial residual");
  st->true_rel = rn / bn;
  if (rn / bn <= tol) return QQ_OK;
  QQ_TRY(lin(c, A.sp(0), cimm(1.0 / rn), r.sp()));
  std::vector<dense::cd> cvec(m + 1, 0.0);
  cvec[0] = rn;
  QQ_TRY(A.zeroH());
  DevBuf cd, Pd;
  QQ_CK(cd.alloc(sizeof(double) * 2 * 256));
  QQ_CK(Pd.alloc(sizeof(double) * 2 * (size_t)(m + 1) * (k + 1)));
  int j0 = 0, icycle = 1, status = QQ_NOT_CONVERGED;
  dense::Mat Hk_last;
  bool restarted = false;
  for (;;) {
    for (int j = j0; j < m; ++j) {
      QQ_TRY(arnoldi_step(A, j, tmp32.sp(), kappa, nrm2));
      st->itercount += 1;
      st->mvp += 1;
    }
    dense::Mat Hb;
    QQ_TRY(read_H(A, m, Hb));
    std::vector<dense::cd> y, srv;
    dense::hess_lsq(Hb, cvec, m, y, srv);
    QQ_TRY(upload_cvec(c, y, A.y.as<double>()));
    QQ_CK(launch_basis_accum(P32, A.basis(), m, A.y.as<double>(), c->g.vh, x, c->st));
    QQ_TRY(true_residual(c, b, x, r.sp(), tmp64.sp(), kappa, &rn));
    st->mvp += 1;
    st->true_rel = rn / bn;
    st->hist.push_back(rn / bn);
    st->hist_mvp.push_back(st->mvp);
    st->ncycles = icycle;
    if (!std::isfinite(rn)) {
      status = set_error(QQ_NAN, "NaN residual in mixed gmresdr");
      break;
    }
    if (rn / bn <= tol) {
      status = QQ_OK;
      break;
    }
    if (icycle >= max_cycles) break;
    dense::Mat P, Hk;
    std::vector<dense::cd> cnew, ritz;
    if (!dense::gmresdr_restart(Hb, srv, m, k, P, Hk, cnew, ritz)) {
      status = set_error(QQ_SINGULAR, "harmonic Ritz step failed");
      break;
    }
    st->ritz = ritz;
    QQ_TRY(upload_mat(c, P, Pd.as<double>(), m + 1));
    QQ_CK(launch_rotate(P32, A.basis(), m + 1, k + 1, Pd.as<double>(), m + 1, c->st));
    QQ_TRY(reorth(A, k, nrm2));
    QQ_TRY(A.zeroH());
    QQ_TRY(upload_mat(c, Hk, A.H.as<double>(), m + 1));
    // c = V_{k+1}^H r with the FP64 residual rounded to the basis precision
    QQ_TRY(lin(c, r32.sp(), cimm(1.0), r.sp()));
    int ng = 0;
    double* part = c->partial.as<double>();
    QQ_CK(launch_multidot(P32, A.basis(), k + 1, r32.sp().data, part, &ng, c->st));
    QQ_CK(launch_finalize(part, kRedBlocks, ng * 16, 2 * (k + 1), cd.as<double>(), 0, c->st));
    std::vector<double> ch(2 * (k + 1));
    QQ_TRY(read_scalars(c, cd.as<double>(), 2 * (k + 1), ch.data()));
    std::fill(cvec.begin(), cvec.end(), 0.0);
    for (int i = 0; i <= k; ++i) cvec[i] = {ch[2 * i], ch[2 * i + 1]};
    Hk_last = Hk;
    restarted = true;
    j0 = k;
    icycle += 1;
  }
  if (defl && restarted) {
    defl->k = k;
    defl->pb = P32;
    defl->nel = A.nel;
    QQ_CK(defl->V.alloc((size_t)(k + 1) * A.nel * 16));
    QQ_CK(cudaMemcpyAsync(defl->V.p, A.V.p, (size_t)(k + 1) * A.nel * 16, cudaMemcpyDeviceToDevice, c->st));
    defl->Hk = Hk_last;
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return status;
}

// x += V_k y with y = argmin || V_{k+1}^H r - Hk y ||, then r = b - A x (FP64).
// The minimum-residual projection of GMRES-Proj (inverters.f90:7515-7601) onto a
// deflation space of either basis precision.
int defl_project(qq_ctx* c, const DeflSpace& d, Spinor b, Spinor x, Spinor r, const double kappa[2],
                 double* rn) {
  if (d.k <= 0) return QQ_OK;
  Tmp rl(c, d.pb), tmp64(c, P64);
  DevBuf cd, yd;
  QQ_CK(cd.alloc(sizeof(double) * 2 * 256));
  QQ_CK(yd.alloc(sizeof(double) * 2 * 256));
  const void* rv = r.data;
  if (d.pb != P64) {
    QQ_TRY(lin(c, rl.sp(), cimm(1.0), r));
    rv = rl.sp().data;
  }
  BasisArgs D{d.V.p, d.nel, d.nel};
  int ng = 0;
  double* part = c->partial.as<double>();
  QQ_CK(launch_multidot(d.pb, D, d.k + 1, rv, part, &ng, c->st));
  QQ_CK(launch_finalize(part, kRedBlocks, ng * 16, 2 * (d.k + 1), cd.as<double>(), 0, c->st));
  std::vector<double> ch(2 * (d.k + 1));
  QQ_TRY(read_scalars(c, cd.as<double>(), 2 * (d.k + 1), ch.data()));
  std::vector<dense::cd> cv(d.k + 1), y, srv;
  for (int i = 0; i <= d.k; ++i) cv[i] = {ch[2 * i], ch[2 * i + 1]};
  dense::hess_lsq(d.Hk, cv, d.k, y, srv);
  QQ_TRY(upload_cvec(c, y, yd.as<double>()));
  QQ_CK(launch_basis_accum(d.pb, D, d.k, yd.as<double>(), c->g.vh, x, c->st));
  return true_residual(c, b, x, r, tmp64.sp(), kappa, rn);
}

// ---------------------------------------------------------------------------
// BiCGStab (inverters.f90:302-487), FP64.  Stops when ||r|| / ||r0|| < resmax with
// the recursively updated residual, as the reference.
// ---------------------------------------------------------------------------
int bicgstab_fp64(qq_ctx* c, Spinor phi, Spinor x, double resmax, int itermin, int maxiter,
                  const double kappa[2], SolveStats* st) {
  using cdd = std::complex<double>;
  Tmp r(c, P64), p(c, P64), rhat(c, P64), v(c, P64), t(c, P64), tmp(c, P64);
  QQ_TRY(op_dbletm(c, t.sp(), x, tmp.sp(), 0, kappa));
  double r0 = 0.0;
  double* s = c->scal.as<double>();
  QQ_TRY(lin(c, r.sp(), cimm(1.0), phi, cimm(-1.0), t.sp(), cimm(0), Spinor{nullptr, nullptr, P64}, s));
  QQ_TRY(read_scalars(c, s, 1, &r0));
  r0 = std::sqrt(r0);
  st->mvp = 1;
  QQ_TRY(copy_field(c, rhat.sp(), r.sp()));
  QQ_TRY(zero_field(c, v.sp()));
  QQ_TRY(zero_field(c, p.sp()));
  if (!(r0 > 0.0)) return QQ_OK;
  cdd rho = 1.0, alpha = 1.0, omega = 1.0;
  const int limit = maxiter > 0 ? maxiter : 1000000;
  int status = QQ_NOT_CONVERGED;
  for (;;) {
    const cdd oldrho = rho;
    QQ_TRY(dot_host(c, rhat.sp(), r.sp(), &rho, nullptr));
    const cdd betaomega = rho * alpha / oldrho;
    const cdd beta = betaomega / omega;
    // p = r + beta p - betaomega v
    QQ_TRY(lin(c, p.sp(), cimm(1.0), r.sp(), cimm(beta.real(), beta.imag()), p.sp(),
               cimm(-betaomega.real(), -betaomega.imag()), v.sp()));
    QQ_TRY(op_dbletm(c, v.sp(), p.sp(), tmp.sp(), 0, kappa));
    cdd at;
    QQ_TRY(dot_host(c, rhat.sp(), v.sp(), &at, nullptr));
    alpha = rho / at;
    QQ_TRY(lin(c, r.sp(), cimm(1.0), r.sp(), cimm(-alpha.real(), -alpha.imag()), v.sp()));
    QQ_TRY(op_dbletm(c, t.sp(), r.sp(), tmp.sp(), 0, kappa));
    cdd rt;
    double tt = 0.0;
    QQ_TRY(dot_host(c, r.sp(), t.sp(), &rt, &tt));  // <r,t>, |t|^2
    omega = std::conj(rt) / tt;                     // <t,r>/<t,t>
    QQ_TRY(lin(c, x, cimm(1.0), x, cimm(omega.real(), omega.imag()), r.sp(),
               cimm(alpha.real(), alpha.imag()), p.sp()));
    QQ_TRY(lin(c, r.sp(), cimm(1.0), r.sp(), cimm(-omega.real(), -omega.imag()), t.sp(), cimm(0),
               Spinor{nullptr, nullptr, P64}, s));
    double rsq = 0.0;
    QQ_TRY(read_scalars(c, s, 1, &rsq));
    st->itercount += 1;
    st->mvp += 2;
    const double rel = std::sqrt(rsq) / r0;
    st->hist.push_back(rel);
    st->hist_mvp.push_back(st->mvp);
    st->true_rel = rel;
    if (!std::isfinite(rel)) return set_error(QQ_NAN, "NaN residual in bicgstab");
    if (rel < resmax && st->itercount >= itermin) {
      status = QQ_OK;
      break;
    }
    if (st->itercount >= limit) break;
  }
  // report the true residual
  double tr = 0.0;
  QQ_TRY(true_residual(c, phi, x, r.sp(), tmp.sp(), kappa, &tr));
  st->true_rel = tr / r0;
  return status;
}

}  // namespace qq
