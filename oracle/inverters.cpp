// CPU oracle (test infrastructure): restatement of the in-scope Krylov inverters and
// the propagator driver --
//   gmresdr       Q/inverters.f90:2871-3572
//   psc           Q/inverters.f90:4310-4465
//   gmresproject  Q/inverters.f90:7183-8304
//   bicgstab      Q/inverters.f90:302-487
//   fermprop      Q/quark.f90:458-842 (nkappa = -1: Wilson / twisted-mass Wilson)
// Module state of Q/shift.f90 (vtemp, hcnew, beg) lives in an explicit oq_defl handle.
// Parity unpinned against the Fortran (see oracle.h).
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle_impl.h"

namespace {
int kcyclim = 5000;  // U/latdims.f90:70 (lowered only to time a bounded sample)

struct CMat {  // (2, ld, ncol) Fortran-order complex matrix, 1-based access
  std::vector<double> a;
  int ld = 0;
  void init(int ld_, int ncol) {
    ld = ld_;
    a.assign(2 * (size_t)ld_ * ncol, 0.0);
  }
  void zero() { std::fill(a.begin(), a.end(), 0.0); }
  double& r(int i, int j) { return a[2 * ((size_t)(i - 1) + (size_t)ld * (j - 1))]; }
  double& c(int i, int j) { return a[2 * ((size_t)(i - 1) + (size_t)ld * (j - 1)) + 1]; }
  double* data() { return a.data(); }
};
struct CVec {  // (2, n) complex vector, 1-based
  std::vector<double> a;
  void init(int n) { a.assign(2 * (size_t)n, 0.0); }
  double& r(int i) { return a[2 * (i - 1)]; }
  double& c(int i) { return a[2 * (i - 1) + 1]; }
};

// v_dst(icri..) = v_dst - beta*v_src over interior sites (complex axpy in the
// reference's expression order, e.g. inverters.f90:3124-3131).
void caxpy_minus(const oq_geom* g, double* dst, const double* src, const double* beta) {
  OQ_PAR_FOR3
  for (int ibleo = 1; ibleo <= 8; ++ibleo)
    for (int ieo = 1; ieo <= 2; ++ieo)
      for (int id = 1; id <= 4; ++id)
        for (int k = 1; k <= g->nvhalf; ++k) {
          double* D = dst + g->gi(1, k, id, ieo, ibleo);
          const double* S = src + g->gi(1, k, id, ieo, ibleo);
          for (int icri = 0; icri < 6; icri += 2) {
            double re = D[icri] - beta[0] * S[icri] + beta[1] * S[icri + 1];
            double im = D[icri + 1] - beta[1] * S[icri] - beta[0] * S[icri + 1];
            D[icri] = re;
            D[icri + 1] = im;
          }
        }
}

// acc += s*v over interior sites, expression order of inverters.f90:3226-3234.
void caxpy_plus(const oq_geom* g, double* acc, const double* v, double sr, double si) {
  OQ_PAR_FOR3
  for (int ibleo = 1; ibleo <= 8; ++ibleo)
    for (int ieo = 1; ieo <= 2; ++ieo)
      for (int id = 1; id <= 4; ++id)
        for (int i = 1; i <= g->nvhalf; ++i) {
          double* A = acc + g->gi(1, i, id, ieo, ibleo);
          const double* V = v + g->gi(1, i, id, ieo, ibleo);
          for (int icri = 0; icri < 6; icri += 2) {
            double re = A[icri] + sr * V[icri] - si * V[icri + 1];
            double im = A[icri + 1] + si * V[icri] + sr * V[icri + 1];
            A[icri] = re;
            A[icri + 1] = im;
          }
        }
}

void scale_all(const oq_geom* g, double* v, double s) {
  const size_t n = g->vsize();
  OQ_PAR_FOR
  for (size_t k = 0; k < n; ++k) v[k] = s * v[k];
}
void scale_interior(const oq_geom* g, double* v, double s) {
  g->for_interior([&](size_t k) { v[k] = s * v[k]; });
}

// Givens step of inverters.f90:3197-3217 (rotation of rows i, i+1 in column j).
inline void rot_pair(double gcr, double gci, double gsr, double gsi, double& ar, double& ai,
                     double& br, double& bi) {
  double t1r = gcr * ar - gci * ai + gsr * br + gsi * bi;
  double t1i = gcr * ai + gci * ar + gsr * bi - gsi * br;
  double t2r = gcr * br - gci * bi - gsr * ar + gsi * ai;
  double t2i = gcr * bi + gci * br - gsr * ai - gsi * ar;
  ar = t1r; ai = t1i; br = t2r; bi = t2i;
}

// Back substitution of the triangular LS, inverters.f90:3221-3245 (ss = R^-1 c).
void backsub(CMat& hc, CVec& c, CVec& ss, int j) {
  for (int i = 1; i <= j; ++i) {
    ss.r(i) = c.r(i);
    ss.c(i) = c.c(i);
  }
  double con2 = 1.0 / (hc.r(j, j) * hc.r(j, j) + hc.c(j, j) * hc.c(j, j));
  double cst = con2 * (ss.r(j) * hc.r(j, j) + ss.c(j) * hc.c(j, j));
  ss.c(j) = con2 * (ss.c(j) * hc.r(j, j) - ss.r(j) * hc.c(j, j));
  ss.r(j) = cst;
  if (j != 1) {
    for (int i = 1; i <= j - 1; ++i) {
      int ir = j - i + 1, irm1 = ir - 1;
      for (int jj = 1; jj <= irm1; ++jj) {
        cst = ss.r(jj) - ss.r(ir) * hc.r(jj, ir) + ss.c(ir) * hc.c(jj, ir);
        ss.c(jj) = ss.c(jj) - ss.r(ir) * hc.c(jj, ir) - ss.c(ir) * hc.r(jj, ir);
        ss.r(jj) = cst;
      }
      con2 = 1.0 / (hc.r(irm1, irm1) * hc.r(irm1, irm1) + hc.c(irm1, irm1) * hc.c(irm1, irm1));
      cst = con2 * (ss.r(irm1) * hc.r(irm1, irm1) + ss.c(irm1) * hc.c(irm1, irm1));
      ss.c(irm1) = con2 * (ss.c(irm1) * hc.r(irm1, irm1) - ss.r(irm1) * hc.c(irm1, irm1));
      ss.r(irm1) = cst;
    }
  }
}

// New Givens rotation zeroing hc(j+1,j) and its application to c
// (inverters.f90:3187-3218).
void new_rotation(CMat& hc, CVec& c, CVec& gc, CVec& gs, int j) {
  double amags = hc.r(j, j) * hc.r(j, j) + hc.c(j, j) * hc.c(j, j);
  double tv = std::sqrt(amags + hc.r(j + 1, j) * hc.r(j + 1, j) + hc.c(j + 1, j) * hc.c(j + 1, j));
  gc.r(j) = std::sqrt(amags) / tv;
  gc.c(j) = 0.0;
  double con2 = gc.r(j) / amags;
  gs.r(j) = con2 * (hc.r(j + 1, j) * hc.r(j, j) + hc.c(j + 1, j) * hc.c(j, j));
  gs.c(j) = con2 * (hc.c(j + 1, j) * hc.r(j, j) - hc.r(j + 1, j) * hc.c(j, j));
  double hr = gc.r(j) * hc.r(j, j) + gs.r(j) * hc.r(j + 1, j) + gs.c(j) * hc.c(j + 1, j);
  double hi = gc.r(j) * hc.c(j, j) + gs.r(j) * hc.c(j + 1, j) - gs.c(j) * hc.r(j + 1, j);
  hc.r(j, j) = hr;
  hc.c(j, j) = hi;
  hc.r(j + 1, j) = hc.c(j + 1, j) = 0.0;
  double t1r = gc.r(j) * c.r(j) + gs.r(j) * c.r(j + 1) + gs.c(j) * c.c(j + 1);
  double t1i = gc.r(j) * c.c(j) + gs.r(j) * c.c(j + 1) - gs.c(j) * c.r(j + 1);
  double t2r = gc.r(j) * c.r(j + 1) - gs.r(j) * c.r(j) + gs.c(j) * c.c(j);
  double t2i = gc.r(j) * c.c(j + 1) - gs.r(j) * c.c(j) - gs.c(j) * c.r(j);
  c.r(j) = t1r; c.c(j) = t1i; c.r(j + 1) = t2r; c.c(j + 1) = t2i;
}

// Givens triangularisation of a (k+1) x k block with rotation arrays gca/gsa, applied
// to c as well (inverters.f90:3518-3556, :7535-7575).
void block_triangularise(CMat& hc, CVec& c, CMat& gca, CMat& gsa, int k) {
  for (int jj = 1; jj <= k; ++jj)
    for (int i = jj + 1; i <= k + 1; ++i) {
      double amags = hc.r(jj, jj) * hc.r(jj, jj) + hc.c(jj, jj) * hc.c(jj, jj);
      double con2 = 1.0 / amags;
      double tv = std::sqrt(amags + hc.r(i, jj) * hc.r(i, jj) + hc.c(i, jj) * hc.c(i, jj));
      gca.r(i, jj) = std::sqrt(amags) / tv;
      gca.c(i, jj) = 0.0;
      gsa.r(i, jj) = gca.r(i, jj) * con2 * (hc.r(i, jj) * hc.r(jj, jj) + hc.c(i, jj) * hc.c(jj, jj));
      gsa.c(i, jj) = gca.r(i, jj) * con2 * (hc.c(i, jj) * hc.r(jj, jj) - hc.r(i, jj) * hc.c(jj, jj));
      const double ca = gca.r(i, jj), sr = gsa.r(i, jj), si = gsa.c(i, jj);
      for (int j = jj; j <= k; ++j) {
        double t1r = ca * hc.r(jj, j) + sr * hc.r(i, j) + si * hc.c(i, j);
        double t1i = ca * hc.c(jj, j) + sr * hc.c(i, j) - si * hc.r(i, j);
        double t2r = ca * hc.r(i, j) - sr * hc.r(jj, j) + si * hc.c(jj, j);
        double t2i = ca * hc.c(i, j) - sr * hc.c(jj, j) - si * hc.r(jj, j);
        hc.r(jj, j) = t1r; hc.c(jj, j) = t1i; hc.r(i, j) = t2r; hc.c(i, j) = t2i;
      }
      double t1r = ca * c.r(jj) + sr * c.r(i) + si * c.c(i);
      double t1i = ca * c.c(jj) + sr * c.c(i) - si * c.r(i);
      double t2r = ca * c.r(i) - sr * c.r(jj) + si * c.c(jj);
      double t2i = ca * c.c(i) - sr * c.c(jj) - si * c.r(jj);
      c.r(jj) = t1r; c.c(jj) = t1i; c.r(i) = t2r; c.c(i) = t2i;
    }
}

double norm2(const oq_geom* g, const double* a) {
  double adb[2];
  oq_vecdot(g, a, a, adb);
  return adb[0];
}

void log_hist(oq_solve_log* log, int mvp, double rel) {
  if (!log) return;
  if (log->nhist < 4096) {
    log->hist[log->nhist] = rel;
    log->hist_mvp[log->nhist] = mvp;
    log->nhist += 1;
  }
}
}  // namespace

extern "C" void oq_set_kcyclim(int n) { kcyclim = n > 0 ? n : 5000; }

extern "C" oq_defl* oq_defl_create(const oq_geom* g, int nmax, int kmax) {
  auto* d = new oq_defl();
  d->nmax = nmax;
  d->kmax = kmax;
  d->k = 0;
  d->vsize = g->vsize();
  d->vtemp.assign((size_t)(kmax + 1) * d->vsize, 0.0);
  d->hcnew.assign(2 * (size_t)(nmax + 1) * nmax, 0.0);
  d->beg.assign(d->vsize, 0.0);
  return d;
}
extern "C" void oq_defl_destroy(oq_defl* d) { delete d; }
extern "C" void oq_defl_get(const oq_defl* d, int k, double* vtemp, double* hcnew) {
  if (vtemp) std::memcpy(vtemp, d->vtemp.data(), sizeof(double) * (size_t)(k + 1) * d->vsize);
  if (hcnew) {
    const int ld = d->nmax + 1;
    for (int j = 1; j <= k; ++j)
      for (int i = 1; i <= k + 1; ++i) {
        hcnew[2 * ((i - 1) + (size_t)(k + 1) * (j - 1))] = d->hcnew[2 * ((i - 1) + (size_t)ld * (j - 1))];
        hcnew[2 * ((i - 1) + (size_t)(k + 1) * (j - 1)) + 1] = d->hcnew[2 * ((i - 1) + (size_t)ld * (j - 1)) + 1];
      }
  }
}

// ------------------------------------------------------------------------------------
// GMRES-DR(n,k) cycle shared by gmresdr (Q/inverters.f90:2871-3572) and gmresdrshift
// (:6041-7179), which run the same Arnoldi, Givens and harmonic-Ritz restart code.
// ------------------------------------------------------------------------------------
namespace {
struct DR {
  const oq_geom* g;
  int nDR, kDR, nmax, ld;
  size_t nv;
  std::vector<double> v;
  CMat hc, hc2, hc3, hcht, z, ws, gca, gsa;
  CVec c, c2, srv, ss, gc, gs, w, em, tau;
  std::vector<int> ipiv, myselect;
  std::vector<double> mag;
  DR(const oq_geom* g_, int n, int k) : g(g_), nDR(n), kDR(k), nmax(n), ld(n + 1), nv(g_->vsize()) {
    v.assign((size_t)(nDR + 1) * nv, 0.0);
    hc.init(ld, nmax); hc2.init(ld, nmax); hc3.init(ld, nmax); hcht.init(nmax, nmax + 1);
    z.init(ld, nmax + 1); ws.init(ld, kDR); gca.init(kDR + 1, kDR); gsa.init(kDR + 1, kDR);
    c.init(nmax + 1); c2.init(nmax + 1); srv.init(nmax + 1); ss.init(nmax); gc.init(nmax);
    gs.init(nmax); w.init(nmax); em.init(nmax); tau.init(nmax);
    ipiv.assign(nmax, 0);
    myselect.assign(nmax, 0);
    mag.assign(nmax, 0.0);
  }
  double* V(int j) { return v.data() + (size_t)(j - 1) * nv; }

  // Arnoldi step j on V(j+1) = A V(j) (modified Gram-Schmidt, :3099-3155), the diagonal
  // shift hc(j,j) - sigma of gmresdrshift (:6407-6412; gmresdr has sigma = 0), the
  // Givens rotations of the new column (:3157-3218) and the least-squares solution ss
  // (:3221-3245).
  void step(int j, int icycle, double sigma) {
    const int jp1 = j + 1;
    double beta[2];
    for (int i = 1; i <= j; ++i) {
      oq_vecdot(g, V(i), V(jp1), beta);
      hc.r(i, j) = beta[0]; hc.c(i, j) = beta[1];
      hc2.r(i, j) = beta[0]; hc2.c(i, j) = beta[1];
      hc3.r(i, j) = beta[0]; hc3.c(i, j) = beta[1];
      hcht.r(j, i) = hc.r(i, j);
      hcht.c(j, i) = -hc.c(i, j);
      caxpy_minus(g, V(jp1), V(i), beta);
    }
    if (sigma != 0.0) {
      hc.r(j, j) = hc.r(j, j) - sigma;
      hc2.r(j, j) = hc.r(j, j); hc2.c(j, j) = hc.c(j, j);
      hc3.r(j, j) = hc.r(j, j); hc3.c(j, j) = hc.c(j, j);
      hcht.r(j, j) = hc.r(j, j);
      hcht.c(j, j) = -hc.c(j, j);
    }
    oq_vecdot(g, V(jp1), V(jp1), beta);
    hc.r(jp1, j) = std::sqrt(beta[0]); hc.c(jp1, j) = 0.0;
    hc2.r(jp1, j) = hc.r(jp1, j); hc2.c(jp1, j) = 0.0;
    hc3.r(jp1, j) = hc.r(jp1, j); hc3.c(jp1, j) = 0.0;
    hcht.r(j, jp1) = hc.r(jp1, j); hcht.c(j, jp1) = -hc.c(jp1, j);
    scale_all(g, V(jp1), 1.0 / std::sqrt(beta[0]));
    c.r(jp1) = c.c(jp1) = 0.0;
    c2.r(jp1) = c2.c(jp1) = 0.0;

    if (icycle != 1) {
      for (int jj = 1; jj <= kDR; ++jj)
        for (int i = jj + 1; i <= kDR + 1; ++i) {
          const double ar = gca.r(i, jj), ai = gca.c(i, jj), sr = gsa.r(i, jj), si = gsa.c(i, jj);
          double t1r = ar * hc.r(jj, j) - ai * hc.c(jj, j) + sr * hc.r(i, j) + si * hc.c(i, j);
          double t1i = ar * hc.c(jj, j) + ai * hc.r(jj, j) + sr * hc.c(i, j) - si * hc.r(i, j);
          double t2r = ar * hc.r(i, j) - ai * hc.c(i, j) - sr * hc.r(jj, j) + si * hc.c(jj, j);
          double t2i = ar * hc.c(i, j) + ai * hc.r(i, j) - sr * hc.c(jj, j) - si * hc.r(jj, j);
          hc.r(jj, j) = t1r; hc.c(jj, j) = t1i; hc.r(i, j) = t2r; hc.c(i, j) = t2i;
        }
      if (j > kDR + 1)
        for (int i = kDR + 1; i <= j - 1; ++i)
          rot_pair(gc.r(i), gc.c(i), gs.r(i), gs.c(i), hc.r(i, j), hc.c(i, j), hc.r(i + 1, j),
                   hc.c(i + 1, j));
    } else if (j != 1) {
      for (int i = 1; i <= j - 1; ++i)
        rot_pair(gc.r(i), gc.c(i), gs.r(i), gs.c(i), hc.r(i, j), hc.c(i, j), hc.r(i + 1, j),
                 hc.c(i + 1, j));
    }
    new_rotation(hc, c, gc, gs, j);
    backsub(hc, c, ss, j);
  }

  // srv = c2 - hc3 ss, the residual in the basis V_{n+1} (:3257-3268)
  void residual_coords() {
    for (int i = 1; i <= nDR + 1; ++i) {
      srv.r(i) = c2.r(i);
      srv.c(i) = c2.c(i);
    }
    for (int jj = 1; jj <= nDR; ++jj)
      for (int i = 1; i <= nDR + 1; ++i) {
        double a = srv.r(i) - ss.r(jj) * hc3.r(i, jj) + ss.c(jj) * hc3.c(i, jj);
        srv.c(i) = srv.c(i) - ss.r(jj) * hc3.c(i, jj) - ss.c(jj) * hc3.r(i, jj);
        srv.r(i) = a;
      }
  }

  // Harmonic-Ritz restart (:3300-3556): the k smallest harmonic Ritz vectors of
  // H + h_{n+1,n}^2 H^-H e_n e_n^T and the residual give V_{k+1}, hcnew, c; the new
  // (k+1) x k block is triangularised with gca/gsa.
  void restart(oq_defl* defl, oq_solve_log* log) {
    double beta[2];
    for (int i = 1; i <= nDR; ++i) em.r(i) = em.c(i) = 0.0;
    em.r(nDR) = 1.0;
    oq_linearsolver(nDR, 1, hcht.data(), hcht.ld, ipiv.data(), em.a.data(), nDR);
    const double hr = hc2.r(nDR + 1, nDR), hi = hc2.c(nDR + 1, nDR);
    for (int i = 1; i <= nDR; ++i) {
      double a = hc2.r(i, nDR) + em.r(i) * hr * hr - em.r(i) * hi * hi - 2.0 * em.c(i) * hr * hi;
      double b = hc2.c(i, nDR) + em.c(i) * hr * hr + 2.0 * em.r(i) * hi * hr - em.c(i) * hi * hi;
      hc2.r(i, nDR) = a;
      hc2.c(i, nDR) = b;
    }
    oq_hessenberg(hc2.data(), hc2.ld, nDR, 1, nDR, tau.a.data());
    for (int jj = 1; jj <= nDR; ++jj)
      for (int i = jj; i <= nDR; ++i) {
        z.r(i, jj) = hc2.r(i, jj);
        z.c(i, jj) = hc2.c(i, jj);
      }
    oq_qgenerator(nDR, 1, nDR, z.data(), z.ld, tau.a.data());
    oq_evalues(1, nDR, 1, nDR, hc2.data(), hc2.ld, w.a.data(), z.data(), z.ld);
    mag[0] = std::sqrt(w.r(1) * w.r(1) + w.c(1) * w.c(1));
    for (int i = 2; i <= nDR; ++i) {
      mag[i - 1] = std::sqrt(w.r(i) * w.r(i) + w.c(i) * w.c(i));
      int is = 0;
      for (;;) {
        is += 1;
        if (is > i - 1) break;
        if (mag[i - 1] < mag[is - 1]) {
          double tval = mag[i - 1];
          for (int ivb = i - 1; ivb >= is; --ivb) mag[ivb] = mag[ivb - 1];
          mag[is - 1] = tval;
          break;
        }
      }
    }
    for (int i = 1; i <= nDR; ++i)
      myselect[i - 1] = std::sqrt(w.r(i) * w.r(i) + w.c(i) * w.c(i)) <= mag[kDR - 1] ? 1 : 0;
    int idis = 0;
    oq_orgschur(myselect.data(), nDR, hc2.data(), hc2.ld, z.data(), z.ld, w.a.data(), &idis);
    if (log) {
      log->nritz = nDR < 512 ? nDR : 512;
      for (int i = 0; i < log->nritz; ++i) {
        log->ritz[2 * i] = w.r(i + 1);
        log->ritz[2 * i + 1] = w.c(i + 1);
      }
    }
    for (int i = 1; i <= kDR; ++i) z.r(nDR + 1, i) = z.c(nDR + 1, i) = 0.0;
    for (int i = 1; i <= nDR + 1; ++i) {
      z.r(i, kDR + 1) = srv.r(i);
      z.c(i, kDR + 1) = srv.c(i);
    }
    for (int jj = 1; jj <= kDR; ++jj) {
      double tv0 = 0.0, tv1 = 0.0;
      for (int i = 1; i <= nDR + 1; ++i) {
        tv0 = tv0 + z.r(i, jj) * z.r(i, kDR + 1) + z.c(i, jj) * z.c(i, kDR + 1);
        tv1 = tv1 + z.r(i, jj) * z.c(i, kDR + 1) - z.c(i, jj) * z.r(i, kDR + 1);
      }
      for (int i = 1; i <= nDR + 1; ++i) {
        double a = z.r(i, kDR + 1) - tv0 * z.r(i, jj) + tv1 * z.c(i, jj);
        double b = z.c(i, kDR + 1) - tv0 * z.c(i, jj) - tv1 * z.r(i, jj);
        z.r(i, kDR + 1) = a;
        z.c(i, kDR + 1) = b;
      }
    }
    double rv = 1.0 / oq::twonorm_c(&z.r(1, kDR + 1), nDR + 1);
    for (int i = 1; i <= nDR + 1; ++i) {
      z.r(i, kDR + 1) *= rv;
      z.c(i, kDR + 1) *= rv;
    }
    for (int jj = 1; jj <= kDR; ++jj) {
      for (int ii = 1; ii <= nDR + 1; ++ii) ws.r(ii, jj) = ws.c(ii, jj) = 0.0;
      for (int ii = 1; ii <= nDR; ++ii)
        for (int i = 1; i <= nDR + 1; ++i) {
          double a = ws.r(i, jj) + z.r(ii, jj) * hc3.r(i, ii) - z.c(ii, jj) * hc3.c(i, ii);
          double b = ws.c(i, jj) + z.r(ii, jj) * hc3.c(i, ii) + z.c(ii, jj) * hc3.r(i, ii);
          ws.r(i, jj) = a;
          ws.c(i, jj) = b;
        }
    }
    CMat hcnew;
    hcnew.init(ld, nmax);
    for (int jj = 1; jj <= kDR; ++jj)
      for (int ii = 1; ii <= kDR + 1; ++ii) {
        double a = 0.0, b = 0.0;
        for (int i = 1; i <= nDR + 1; ++i) {
          a = a + z.r(i, ii) * ws.r(i, jj) + z.c(i, ii) * ws.c(i, jj);
          b = b + z.r(i, ii) * ws.c(i, jj) - z.c(i, ii) * ws.r(i, jj);
        }
        hcnew.r(ii, jj) = a;
        hcnew.c(ii, jj) = b;
      }
    for (int jj = 1; jj <= nDR; ++jj)
      for (int ii = 1; ii <= nDR; ++ii) {
        hcht.r(ii, jj) = hcht.c(ii, jj) = 0.0;
        hc2.r(ii, jj) = hc2.c(ii, jj) = 0.0;
      }
    for (int jj = 1; jj <= kDR; ++jj) {
      for (int ii = 1; ii <= kDR + 1; ++ii) {
        hc.r(ii, jj) = hc2.r(ii, jj) = hc3.r(ii, jj) = hcnew.r(ii, jj);
        hc.c(ii, jj) = hc2.c(ii, jj) = hc3.c(ii, jj) = hcnew.c(ii, jj);
      }
      for (int ii = 1; ii <= kDR + 1; ++ii) {
        hcht.r(jj, ii) = hcnew.r(ii, jj);
        hcht.c(jj, ii) = -hcnew.c(ii, jj);
      }
    }
    for (int ii = 1; ii <= kDR + 1; ++ii) {
      double a = 0.0, b = 0.0;
      for (int i = 1; i <= nDR + 1; ++i) {
        a = a + z.r(i, ii) * srv.r(i) + z.c(i, ii) * srv.c(i);
        b = b + z.r(i, ii) * srv.c(i) - z.c(i, ii) * srv.r(i);
      }
      c.r(ii) = a; c.c(ii) = b;
      c2.r(ii) = a; c2.c(ii) = b;
    }
    // V_{k+1} <- V_{m+1} Z, site by site (inverters.f90:3461-3485).
    std::vector<double> vt(6 * (size_t)(kDR + 1));
    for (int ibleo = 1; ibleo <= 8; ++ibleo)
      for (int ieo = 1; ieo <= 2; ++ieo)
        for (int id = 1; id <= 4; ++id)
          for (int i = 1; i <= g->nvhalf; ++i) {
            const size_t off = g->gi(1, i, id, ieo, ibleo);
            for (int jj = 1; jj <= kDR + 1; ++jj) {
              double* VT = vt.data() + 6 * (jj - 1);
              for (int q = 0; q < 6; ++q) VT[q] = 0.0;
              for (int k = 1; k <= nDR + 1; ++k) {
                const double* Vk = V(k) + off;
                for (int icri = 0; icri < 6; icri += 2) {
                  double a = VT[icri] + z.r(k, jj) * Vk[icri] - z.c(k, jj) * Vk[icri + 1];
                  double b = VT[icri + 1] + z.c(k, jj) * Vk[icri] + z.r(k, jj) * Vk[icri + 1];
                  VT[icri] = a;
                  VT[icri + 1] = b;
                }
              }
            }
            for (int jj = 1; jj <= kDR + 1; ++jj)
              for (int q = 0; q < 6; ++q) V(jj)[off + q] = vt[6 * (jj - 1) + q];
          }
    for (int jj = 1; jj <= kDR; ++jj) {
      oq_vecdot(g, V(jj), V(kDR + 1), beta);
      caxpy_minus(g, V(kDR + 1), V(jj), beta);
    }
    oq_vecdot(g, V(kDR + 1), V(kDR + 1), beta);
    scale_interior(g, V(kDR + 1), 1.0 / std::sqrt(beta[0]));
    if (defl) {  // module shift: vtemp(:, 1..k+1), hcnew
      defl->k = kDR;
      if ((int)defl->vtemp.size() < (int)((kDR + 1) * nv)) defl->vtemp.resize((kDR + 1) * nv);
      std::fill(defl->vtemp.begin(), defl->vtemp.end(), 0.0);
      for (int jj = 1; jj <= kDR + 1; ++jj)
        g->for_interior([&](size_t k) { defl->vtemp[(size_t)(jj - 1) * nv + k] = V(jj)[k]; });
      defl->nmax = nmax;
      defl->hcnew.assign(hcnew.a.begin(), hcnew.a.end());
    }
    block_triangularise(hc, c, gca, gsa, kDR);
  }
};
}  // namespace

// ------------------------------------------------------------------------------------
// GMRES-DR(n,k): Q/inverters.f90:2871-3572
// ------------------------------------------------------------------------------------
extern "C" int oq_gmresdr(const oq_geom* g, const double* phi, double* x, const int GMRES[2],
                          double resmax, int itermin, const double* u, const double kappa[2],
                          oq_defl* defl, oq_solve_log* log) {
  const int nDR = GMRES[0], kDR = GMRES[1];
  const size_t nv = g->vsize();
  if (log) std::memset(log, 0, sizeof(*log));
  DR D(g, nDR, kDR);
  std::vector<double> r(nv, 0.0), h(nv, 0.0), xt(nv, 0.0), xb(nv, 0.0);
  int icycle = 1, mvp = 0;
  double beta[2];

  // MORGAN'S STEP 1.
  oq::hdbletm(g, h.data(), u, x, 0, kappa);
  mvp += 1;
  g->for_interior([&](size_t k) {
    r[k] = phi[k] - h[k];
    D.V(1)[k] = r[k];
    xt[k] = x[k];
  });
  oq_vecdot(g, D.V(1), D.V(1), beta);
  beta[0] = std::sqrt(beta[0]);
  const double normnum = beta[0];
  scale_all(g, D.V(1), 1.0 / beta[0]);
  D.c.r(1) = beta[0];
  D.c.c(1) = 0.0;
  D.c2.r(1) = D.c.r(1);
  D.c2.c(1) = D.c.c(1);

  int itercount = 0, j = 0, status = 1;
  for (;;) {
    if (icycle > kcyclim) break;
    j += 1;
    itercount += 1;
    oq::hdbletm(g, D.V(j + 1), u, D.V(j), 0, kappa);
    mvp += 1;
    D.step(j, icycle, 0.0);

    std::fill(xb.begin(), xb.end(), 0.0);
    for (int jj = 1; jj <= j; ++jj) caxpy_plus(g, xb.data(), D.V(jj), D.ss.r(jj), D.ss.c(jj));
    g->for_interior([&](size_t k) { x[k] = xt[k] + xb[k]; });
    D.residual_coords();

    if (j >= nDR) {
      oq::hdbletm(g, h.data(), u, x, 0, kappa);
      mvp += 1;
      g->for_interior([&](size_t k) { r[k] = phi[k] - h[k]; });
      oq_vecdot(g, r.data(), r.data(), beta);
      beta[0] = std::sqrt(beta[0]);
      log_hist(log, mvp, beta[0] / normnum);
      if (beta[0] / normnum < resmax && itercount >= itermin) {
        status = 0;
        break;
      }
      g->for_interior([&](size_t k) { xt[k] = x[k]; });
      D.restart(defl, log);
      j = kDR;
      icycle += 1;
    }
  }
  if (log) {
    oq::hdbletm(g, h.data(), u, x, 0, kappa);
    g->for_interior([&](size_t k) { r[k] = phi[k] - h[k]; });
    log->itercount = itercount;
    log->mvp = mvp;
    log->ncycles = icycle;
    log->final_rel = std::sqrt(norm2(g, r.data())) / std::sqrt(norm2(g, phi));
  }
  return status;
}

// ------------------------------------------------------------------------------------
// gmresdrshift: Q/inverters.f90:6041-7179.  GMRES-DR(n,k) on A - sigma_1, A the
// operator of gamma5mult (Q/diracops.f90:1750-1860), and for every further shift s the
// solution of (A - sigma_s) x_s = b whose residual stays collinear with the base
// residual (Frommer-Glaessner; Darnell, Morgan and Wilcox 2008):
//   [Hbar + (sigma_1 - sigma_s) I~ | srv] (d_s, alpha_s) = cmult_s c2      (:6576-6747)
// solved here with linearsolver on the square (j+1) system instead of zgeqrf/zungqr
// (the same unique solution).  Where the reference cannot run as written, the
// evident intent is kept and stated:
//   * sigma is an argument (the reference's local sigma is never assigned);
//   * the shifted solutions are formed at the end of every cycle (the reference tests
//     j >= nmaxGMRES at :6754, which GMRES-DR(n < nmaxGMRES) never reaches before restarting);
//   * the initial guess is zero for every shift, so the initial residuals are b and
//     collinear (the reference copies b - A x_1 to every shift, :6297-6315).
// Each shift's residual is updated recursively, r_s -= (A - sigma_s) xb_s (:6816-6830),
// and the iteration stops when ||r_1|| < resmax (absolute, as :6865).
// ------------------------------------------------------------------------------------
extern "C" int oq_gmresdrshift(const oq_geom* g, const double* b, double* xshift, int nshifts,
                               const double* sigma, const int GMRES[2], double resmax,
                               int itermin, const double* u, const double kappa[2],
                               double* resid, oq_solve_log* log) {
  const int nDR = GMRES[0], kDR = GMRES[1];
  const size_t nv = g->vsize();
  if (log) std::memset(log, 0, sizeof(*log));
  DR D(g, nDR, kDR);
  std::vector<double> h(nv, 0.0), xb(nv, 0.0), rshift((size_t)nshifts * nv, 0.0);
  auto X = [&](int s) { return xshift + (size_t)(s - 1) * nv; };
  auto R = [&](int s) { return rshift.data() + (size_t)(s - 1) * nv; };
  std::vector<double> cmr(nshifts + 1, 1.0), cmi(nshifts + 1, 0.0);  // cmult
  std::vector<double> dr((size_t)(nDR + 1) * (nshifts + 1)), di(dr.size());
  int icycle = 1, mvp = 0;
  double beta[2];

  std::fill(xshift, xshift + (size_t)nshifts * nv, 0.0);
  g->for_interior([&](size_t k) {
    D.V(1)[k] = b[k];
    for (int s = 1; s <= nshifts; ++s) R(s)[k] = b[k];
  });
  oq_vecdot(g, D.V(1), D.V(1), beta);
  beta[0] = std::sqrt(beta[0]);
  const double normnum = beta[0];
  for (int s = 1; s <= nshifts; ++s) resid[s - 1] = normnum;
  if (!(normnum > 0.0)) return 0;
  scale_all(g, D.V(1), 1.0 / beta[0]);
  D.c.r(1) = beta[0];
  D.c.c(1) = 0.0;
  D.c2.r(1) = D.c.r(1);
  D.c2.c(1) = D.c.c(1);

  int itercount = 0, j = 0, status = 1;
  for (;;) {
    if (icycle > kcyclim) break;
    j += 1;
    itercount += 1;
    oq::gamma5mult(g, D.V(j + 1), u, D.V(j), 0, kappa);
    mvp += 1;
    D.step(j, icycle, sigma[0]);
    D.residual_coords();
    if (j < nDR) continue;

    // base shift: d = ss; further shifts: the collinear solve with the base srv
    for (int i = 1; i <= j; ++i) {
      dr[i] = D.ss.r(i);
      di[i] = D.ss.c(i);
    }
    for (int s = 2; s <= nshifts; ++s) {
      const int n1 = j + 1;
      std::vector<double> a(2 * (size_t)n1 * n1, 0.0), rhs(2 * (size_t)n1, 0.0);
      std::vector<int> piv(n1);
      for (int jj = 1; jj <= j; ++jj)
        for (int ii = 1; ii <= n1; ++ii) {
          a[2 * ((ii - 1) + (size_t)n1 * (jj - 1))] = D.hc2.r(ii, jj);
          a[2 * ((ii - 1) + (size_t)n1 * (jj - 1)) + 1] = D.hc2.c(ii, jj);
        }
      for (int jj = 1; jj <= j; ++jj)
        a[2 * ((jj - 1) + (size_t)n1 * (jj - 1))] += sigma[0] - sigma[s - 1];
      for (int ii = 1; ii <= n1; ++ii) {
        a[2 * ((ii - 1) + (size_t)n1 * j)] = D.srv.r(ii);
        a[2 * ((ii - 1) + (size_t)n1 * j) + 1] = D.srv.c(ii);
        rhs[2 * (ii - 1)] = cmr[s] * D.c2.r(ii) - cmi[s] * D.c2.c(ii);
        rhs[2 * (ii - 1) + 1] = cmr[s] * D.c2.c(ii) + cmi[s] * D.c2.r(ii);
      }
      oq_linearsolver(n1, 1, a.data(), n1, piv.data(), rhs.data(), n1);
      for (int i = 1; i <= j; ++i) {
        dr[(size_t)(s - 1) * (nDR + 1) + i] = rhs[2 * (i - 1)];
        di[(size_t)(s - 1) * (nDR + 1) + i] = rhs[2 * (i - 1) + 1];
      }
      cmr[s] = rhs[2 * j];
      cmi[s] = rhs[2 * j + 1];
    }
    for (int s = 1; s <= nshifts; ++s) {
      std::fill(xb.begin(), xb.end(), 0.0);
      for (int jj = 1; jj <= j; ++jj)
        caxpy_plus(g, xb.data(), D.V(jj), dr[(size_t)(s - 1) * (nDR + 1) + jj],
                   di[(size_t)(s - 1) * (nDR + 1) + jj]);
      g->for_interior([&](size_t k) { X(s)[k] = X(s)[k] + xb[k]; });
      oq::gamma5mult(g, h.data(), u, xb.data(), 0, kappa);
      mvp += 1;
      const double sg = sigma[s - 1];
      g->for_interior([&](size_t k) { R(s)[k] = R(s)[k] - h[k] + sg * xb[k]; });
      oq_vecdot(g, R(s), R(s), beta);
      resid[s - 1] = std::sqrt(beta[0]);
    }
    log_hist(log, mvp, resid[0] / normnum);
    if (resid[0] < resmax && itercount >= itermin) {
      status = 0;
      break;
    }
    D.restart(nullptr, log);
    j = kDR;
    icycle += 1;
  }
  if (log) {
    log->itercount = itercount;
    log->mvp = mvp;
    log->ncycles = icycle;
    log->final_rel = resid[0] / normnum;
  }
  return status;
}

// ------------------------------------------------------------------------------------
// GMRES-Proj: Q/inverters.f90:7183-8304 (sigma = 0; single shift)
// ------------------------------------------------------------------------------------
extern "C" int oq_gmresproject(const oq_geom* g, const double* b, double* xshift,
                               const int GMRES[2], double resmax, int itermin,
                               const double* u, const double kappa[2], int isignal,
                               oq_defl* defl, oq_solve_log* log) {
  const int nDR = GMRES[0], kDR = GMRES[1];
  const size_t nv = g->vsize();
  if (log) std::memset(log, 0, sizeof(*log));
  const int nmax = nDR > kDR ? nDR : kDR + 1, ld = nmax + 1;
  std::vector<double> v((size_t)(nDR + 1) * nv, 0.0);
  auto V = [&](int j) { return v.data() + (size_t)(j - 1) * nv; };
  auto VT = [&](int j) { return defl->vtemp.data() + (size_t)(j - 1) * nv; };
  std::vector<double> r(nv, 0.0), h(nv, 0.0), rshift(nv, 0.0), xb(nv, 0.0);
  CMat hc, hc2, hc3, gca, gsa;
  hc.init(ld, nmax); hc2.init(ld, nmax); hc3.init(ld, nmax);
  gca.init(kDR + 1, kDR); gsa.init(kDR + 1, kDR);
  CVec c, c2, ss, gc, gs, srv, st;
  c.init(nmax + 1); c2.init(nmax + 1); ss.init(nmax); gc.init(nmax); gs.init(nmax);
  srv.init(nmax + 1); st.init(nmax + 1);
  const double sigma = 0.0;
  std::fill(xshift, xshift + nv, 0.0);
  int icycle = 1, mvp = 0, itercount = 0;
  double beta[2];
  oq_vecdot(g, b, b, beta);
  oq::hdbletm(g, h.data(), u, xshift, 0, kappa);
  mvp += 1;
  g->for_interior([&](size_t k) { rshift[k] = b[k] - h[k] + sigma * xshift[k]; });
  if (isignal == 1) {
    rshift = defl->beg;
  } else {
    defl->beg = rshift;
  }
  oq_vecdot(g, rshift.data(), rshift.data(), beta);
  const double rinit = std::sqrt(beta[0]);
  double rn = rinit;
  oq::hdbletm(g, h.data(), u, xshift, 0, kappa);
  mvp += 1;
  g->for_interior([&](size_t k) { r[k] = defl->beg[k] - h[k] + sigma * xshift[k]; });
  rshift = r;
  std::fill(xshift, xshift + nv, 0.0);
  const int k = kDR;
  const int ldh = defl->nmax + 1;
  int status = 1;
  for (;;) {
    if (rn / rinit <= resmax) {
      status = 0;
      break;
    }
    if (icycle > kcyclim) break;
    // Projection over the deflation space (inverters.f90:7515-7601).
    for (int i = 1; i <= k + 1; ++i) {
      oq_vecdot(g, VT(i), rshift.data(), beta);
      c.r(i) = beta[0]; c.c(i) = beta[1];
      c2.r(i) = beta[0]; c2.c(i) = beta[1];
    }
    for (int ii = 1; ii <= k + 1; ++ii)
      for (int jj = 1; jj <= k; ++jj) {
        hc2.r(ii, jj) = defl->hcnew[2 * ((ii - 1) + (size_t)ldh * (jj - 1))];
        hc2.c(ii, jj) = defl->hcnew[2 * ((ii - 1) + (size_t)ldh * (jj - 1)) + 1];
      }
    for (int jj = 1; jj <= k; ++jj) hc2.r(jj, jj) = hc2.r(jj, jj) - sigma;
    block_triangularise(hc2, c, gca, gsa, k);
    backsub(hc2, c, ss, k);
    std::fill(xb.begin(), xb.end(), 0.0);
    for (int jj = 1; jj <= k; ++jj) caxpy_plus(g, xb.data(), VT(jj), ss.r(jj), ss.c(jj));
    g->for_interior([&](size_t q) { xshift[q] = xshift[q] + xb[q]; });
    oq::hdbletm(g, h.data(), u, xshift, 0, kappa);
    g->for_interior([&](size_t q) { rshift[q] = defl->beg[q] - h[q] + sigma * xshift[q]; });

    oq_vecdot(g, rshift.data(), rshift.data(), beta);
    double betashift = beta[0];
    {
      const double cst = 1.0 / std::sqrt(betashift);
      g->for_interior([&](size_t q) { V(1)[q] = cst * rshift[q]; });
    }
    c.r(1) = std::sqrt(betashift);
    c.c(1) = 0.0;
    c2.r(1) = c.r(1);
    c2.c(1) = c.c(1);
    for (int j = 1; j <= nDR; ++j) {
      const int jp1 = j + 1;
      itercount += 1;
      oq::hdbletm(g, V(jp1), u, V(j), 0, kappa);
      mvp += 1;
      for (int i = 1; i <= j; ++i) {
        oq_vecdot(g, V(i), V(jp1), beta);
        hc.r(i, j) = beta[0]; hc.c(i, j) = beta[1];
        hc2.r(i, j) = beta[0]; hc2.c(i, j) = beta[1];
        hc3.r(i, j) = beta[0]; hc3.c(i, j) = beta[1];
        caxpy_minus(g, V(jp1), V(i), beta);
      }
      hc.r(j, j) = hc.r(j, j) - sigma;
      hc2.r(j, j) = hc.r(j, j); hc2.c(j, j) = hc.c(j, j);
      hc3.r(j, j) = hc.r(j, j); hc3.c(j, j) = hc.c(j, j);
      oq_vecdot(g, V(jp1), V(jp1), beta);
      hc.r(jp1, j) = std::sqrt(beta[0]); hc.c(jp1, j) = 0.0;
      hc2.r(jp1, j) = hc.r(jp1, j); hc2.c(jp1, j) = 0.0;
      hc3.r(jp1, j) = hc.r(jp1, j); hc3.c(jp1, j) = 0.0;
      {
        const double cst = 1.0 / std::sqrt(beta[0]);
        g->for_interior([&](size_t q) { V(jp1)[q] = cst * V(jp1)[q]; });
      }
      c.r(jp1) = c.c(jp1) = 0.0;
      c2.r(jp1) = c2.c(jp1) = 0.0;
      if (j != 1)
        for (int i = 1; i <= j - 1; ++i)
          rot_pair(gc.r(i), gc.c(i), gs.r(i), gs.c(i), hc.r(i, j), hc.c(i, j), hc.r(i + 1, j),
                   hc.c(i + 1, j));
      new_rotation(hc, c, gc, gs, j);
      backsub(hc, c, ss, j);
      for (int i = 1; i <= jp1; ++i) st.r(i) = st.c(i) = 0.0;
      for (int ii = 1; ii <= jp1; ++ii) {
        for (int jj = 1; jj <= j; ++jj) {
          double a = st.r(ii) + hc2.r(ii, jj) * ss.r(jj) - hc2.c(ii, jj) * ss.c(jj);
          double bb = st.c(ii) + hc2.r(ii, jj) * ss.c(jj) + hc2.c(ii, jj) * ss.r(jj);
          st.r(ii) = a;
          st.c(ii) = bb;
        }
        srv.r(ii) = c2.r(ii) - st.r(ii);
        srv.c(ii) = c2.c(ii) - st.c(ii);
      }
      if (j >= nDR) {
        std::fill(xb.begin(), xb.end(), 0.0);
        for (int jj = 1; jj <= j; ++jj) caxpy_plus(g, xb.data(), V(jj), ss.r(jj), ss.c(jj));
        g->for_interior([&](size_t q) { xshift[q] = xshift[q] + xb[q]; });
        oq::hdbletm(g, h.data(), u, xshift, 0, kappa);
        mvp += 1;
        g->for_interior([&](size_t q) { rshift[q] = defl->beg[q] - h[q] + sigma * xshift[q]; });
        oq_vecdot(g, rshift.data(), rshift.data(), beta);
        betashift = std::sqrt(beta[0]);
        rn = betashift;
        log_hist(log, mvp, rn / rinit);
        std::fill(rshift.begin(), rshift.end(), 0.0);
        for (int ii = 1; ii <= nDR + 1; ++ii) {
          const double* Vi = V(ii);
          const double sr = srv.r(ii), si = srv.c(ii);
          for (int ibleo = 1; ibleo <= 8; ++ibleo)
            for (int ieo = 1; ieo <= 2; ++ieo)
              for (int id = 1; id <= 4; ++id)
                for (int jj = 1; jj <= g->nvhalf; ++jj) {
                  const size_t off = g->gi(1, jj, id, ieo, ibleo);
                  for (int icri = 0; icri < 6; icri += 2) {
                    double a = rshift[off + icri] + Vi[off + icri] * sr - Vi[off + icri + 1] * si;
                    double bb = rshift[off + icri + 1] + Vi[off + icri] * si + Vi[off + icri + 1] * sr;
                    rshift[off + icri] = a;
                    rshift[off + icri + 1] = bb;
                  }
                }
        }
        const double cst = 1.0 / betashift;
        g->for_interior([&](size_t q) { V(1)[q] = cst * rshift[q]; });
        icycle += 1;
      }
    }
  }
  (void)itermin;
  if (log) {
    oq::hdbletm(g, h.data(), u, xshift, 0, kappa);
    g->for_interior([&](size_t q) { r[q] = b[q] - h[q]; });
    log->itercount = itercount;
    log->mvp = mvp;
    log->ncycles = icycle;
    log->final_rel = std::sqrt(norm2(g, r.data())) / std::sqrt(norm2(g, b));
  }
  return status;
}

// psc Q/inverters.f90:4310-4465
extern "C" int oq_psc(const oq_geom* g, const double* b, double* x, const int GMRES[2],
                      double resmax, int itermin, const double* u, const double kappa[2],
                      int isignal, oq_defl* defl, oq_solve_log* log) {
  const size_t nv = g->vsize();
  const int kDR = GMRES[1];
  if (isignal == 1) {
    std::vector<double> xs(x, x + nv);
    int st = oq_gmresdr(g, b, xs.data(), GMRES, resmax, itermin, u, kappa, defl, log);
    defl->beg.assign(nv, 0.0);
    g->for_interior([&](size_t k) { defl->beg[k] = defl->vtemp[(size_t)kDR * nv + k]; });
    std::memcpy(x, xs.data(), sizeof(double) * nv);
    return st;
  }
  const double projresmax = 1.0e-8;  // hard-coded at inverters.f90:4442
  int GMRESproj[2] = {GMRES[0] - GMRES[1], GMRES[1]};
  std::vector<double> xs(nv, 0.0);
  int st = oq_gmresproject(g, b, xs.data(), GMRESproj, projresmax, itermin, u, kappa, isignal,
                           defl, log);
  std::memcpy(x, xs.data(), sizeof(double) * nv);
  (void)resmax;
  return st;
}

// ------------------------------------------------------------------------------------
// BiCGStab: Q/inverters.f90:302-487
// ------------------------------------------------------------------------------------
extern "C" int oq_bicgstab(const oq_geom* g, const double* phi, double* x, double resmax,
                           int itermin, const double* u, const double kappa[2],
                           oq_solve_log* log, int maxiter) {
  const size_t nv = g->vsize();
  if (log) std::memset(log, 0, sizeof(*log));
  std::vector<double> r(nv, 0.0), p(nv, 0.0), rhat(nv, 0.0), v(nv, 0.0), t(nv, 0.0);
  int itercount = 0;
  oq::hdbletm(g, t.data(), u, x, 0, kappa);
  g->for_interior([&](size_t k) { r[k] = phi[k] - t[k]; });
  g->for_interior([&](size_t k) { rhat[k] = r[k]; });
  double r0srt[2];
  oq_vecdot(g, r.data(), r.data(), r0srt);
  r0srt[0] = std::sqrt(r0srt[0]);
  double rho[2] = {1.0, 0.0}, oldrho[2], alpha[2] = {1.0, 0.0}, omega[2] = {1.0, 0.0};
  double betaomega[2], beta[2], alphatmp[2], top[2], bottom[2], rsq[2];
  int status = 1;
  for (;;) {
    oldrho[0] = rho[0];
    oldrho[1] = rho[1];
    oq_vecdot(g, rhat.data(), r.data(), rho);
    double bob = 1.0 / (oldrho[0] * oldrho[0] + oldrho[1] * oldrho[1]);
    betaomega[0] = bob * (rho[0] * oldrho[0] * alpha[0] + rho[0] * oldrho[1] * alpha[1] -
                          rho[1] * oldrho[0] * alpha[1] + rho[1] * oldrho[1] * alpha[0]);
    betaomega[1] = bob * (rho[1] * oldrho[0] * alpha[0] - rho[0] * oldrho[1] * alpha[0] +
                          rho[0] * oldrho[0] * alpha[1] + rho[1] * oldrho[1] * alpha[1]);
    double bb = 1.0 / (omega[0] * omega[0] + omega[1] * omega[1]);
    beta[0] = bb * (betaomega[0] * omega[0] + betaomega[1] * omega[1]);
    beta[1] = bb * (betaomega[1] * omega[0] - betaomega[0] * omega[1]);
    g->for_interior([&](size_t k) { t[k] = p[k]; });
    g->for_spin_range(
        [&](size_t s1, size_t s2, size_t s3, size_t s4) {
          for (size_t s : {s1, s2, s3, s4}) {
            double pr = r[s] + beta[0] * t[s] - betaomega[0] * v[s] - beta[1] * t[s + 1] +
                        betaomega[1] * v[s + 1];
            double pi = r[s + 1] + beta[0] * t[s + 1] - betaomega[0] * v[s + 1] + beta[1] * t[s] -
                        betaomega[1] * v[s];
            p[s] = pr;
            p[s + 1] = pi;
          }
        },
        g->nvhalf, true);
    oq::hdbletm(g, v.data(), u, p.data(), 0, kappa);
    oq_vecdot(g, rhat.data(), v.data(), alphatmp);
    double ab = 1.0 / (alphatmp[0] * alphatmp[0] + alphatmp[1] * alphatmp[1]);
    alpha[0] = ab * (rho[0] * alphatmp[0] + rho[1] * alphatmp[1]);
    alpha[1] = ab * (rho[1] * alphatmp[0] - rho[0] * alphatmp[1]);
    g->for_spin_range(
        [&](size_t s1, size_t s2, size_t s3, size_t s4) {
          for (size_t s : {s1, s2, s3, s4}) {
            double a = r[s] - alpha[0] * v[s] + alpha[1] * v[s + 1];
            double b2 = r[s + 1] - alpha[0] * v[s + 1] - alpha[1] * v[s];
            r[s] = a;
            r[s + 1] = b2;
          }
        },
        g->nvhalf, true);
    oq::hdbletm(g, t.data(), u, r.data(), 0, kappa);
    oq_vecdot(g, t.data(), r.data(), top);
    oq_vecdot(g, t.data(), t.data(), bottom);
    double ob = 1.0 / (bottom[0] * bottom[0] + bottom[1] * bottom[1]);
    omega[0] = ob * (top[0] * bottom[0] + top[1] * bottom[1]);
    omega[1] = ob * (top[1] * bottom[0] - top[0] * bottom[1]);
    g->for_spin_range(
        [&](size_t s1, size_t s2, size_t s3, size_t s4) {
          for (size_t s : {s1, s2, s3, s4}) {
            double a = x[s] + omega[0] * r[s] + alpha[0] * p[s] - omega[1] * r[s + 1] -
                       alpha[1] * p[s + 1];
            double b2 = x[s + 1] + omega[0] * r[s + 1] + alpha[0] * p[s + 1] + omega[1] * r[s] +
                        alpha[1] * p[s];
            x[s] = a;
            x[s + 1] = b2;
          }
        },
        g->nvhalf, true);
    g->for_spin_range(
        [&](size_t s1, size_t s2, size_t s3, size_t s4) {
          for (size_t s : {s1, s2, s3, s4}) {
            double a = r[s] - omega[0] * t[s] + omega[1] * t[s + 1];
            double b2 = r[s + 1] - omega[0] * t[s + 1] - omega[1] * t[s];
            r[s] = a;
            r[s + 1] = b2;
          }
        },
        g->nvhalf, true);
    itercount += 1;
    oq_vecdot(g, r.data(), r.data(), rsq);
    double exitnorm = std::sqrt(rsq[0]) / r0srt[0];
    log_hist(log, 2 * itercount, exitnorm);
    if (exitnorm < resmax && itercount >= itermin) {
      status = 0;
      break;
    }
    if (maxiter > 0 && itercount >= maxiter) break;
  }
  if (log) {
    log->itercount = itercount;
    log->mvp = 2 * itercount + 1;
    oq::hdbletm(g, t.data(), u, x, 0, kappa);
    g->for_interior([&](size_t k) { r[k] = phi[k] - t[k]; });
    log->final_rel = std::sqrt(norm2(g, r.data())) / std::sqrt(norm2(g, phi));
  }
  return status;
}

// ------------------------------------------------------------------------------------
// fermprop, nkappa = -1 (Wilson / twisted-mass Wilson): Q/quark.f90:458-842.
// inverter: 0 = bicgstab, 5 = gmresdr, 6 = psc.  xe, xo are single propagator halves.
// ------------------------------------------------------------------------------------
extern "C" int oq_fermprop(const oq_geom* g, const double* be, double* bo,
                           const double kappa[2], int inverter, double resmax, int itermin,
                           const int nGMRES[2], const double* u, double* xe, double* xo,
                           int ntmqcd, int isignal, oq_defl* defl, oq_solve_log* log) {
  const size_t nv = g->vsize();
  std::vector<double> vecsrc(nv, 0.0);
  double fac1 = 2.0 * kappa[0] * kappa[1];
  g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
    vecsrc[s1] = bo[s1] - fac1 * bo[s3];
    vecsrc[s2] = bo[s2] - fac1 * bo[s4];
    vecsrc[s3] = bo[s3] + fac1 * bo[s1];
    vecsrc[s4] = bo[s4] + fac1 * bo[s2];
  });
  oq::hsingle(g, xo, u, vecsrc.data(), 0, 1);
  fac1 = 1.0 / (kappa[0] * kappa[0]);
  const double tk = 2.0 * kappa[0] * kappa[1];
  const double fac2 = 1.0 / (kappa[0] * (1.0 + tk * tk));
  g->for_interior([&](size_t k) { vecsrc[k] = fac1 * be[k] + fac2 * xo[k]; });
  if (inverter > 3) std::fill(xe, xe + nv, 0.0);
  int st = 1;
  if (inverter == 0) {
    st = oq_bicgstab(g, vecsrc.data(), xe, resmax, itermin, u, kappa, log, 0);
  } else if (inverter == 5) {
    st = oq_gmresdr(g, vecsrc.data(), xe, nGMRES, resmax, itermin, u, kappa, defl, log);
  } else if (inverter == 6) {
    st = oq_psc(g, vecsrc.data(), xe, nGMRES, resmax, itermin, u, kappa, isignal, defl, log);
  } else {
    return -1;
  }
  oq::hsingle(g, xo, u, xe, 0, 2);
  g->for_interior([&](size_t k) { xo[k] = bo[k] + kappa[0] * xo[k]; });
  fac1 = 1.0 / (1.0 + tk * tk);
  g->for_interior([&](size_t k) { vecsrc[k] = fac1 * xo[k]; });
  fac1 = 2.0 * kappa[0] * kappa[1];
  g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
    xo[s1] = vecsrc[s1] - fac1 * vecsrc[s3];
    xo[s2] = vecsrc[s2] - fac1 * vecsrc[s4];
    xo[s3] = vecsrc[s3] + fac1 * vecsrc[s1];
    xo[s4] = vecsrc[s4] + fac1 * vecsrc[s2];
  });
  if (ntmqcd != 0 && std::fabs(kappa[1]) > 0.0001) {
    oq_gamma5vector(g, xo, ntmqcd);
    oq_gamma5vector(g, xe, ntmqcd);
  }
  return st;
}
