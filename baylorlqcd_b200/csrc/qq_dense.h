// Small dense FP64 complex linear algebra for the Krylov solvers: the (m+1) x m
// Hessenberg least-squares problem, the harmonic-Ritz eigenproblem of GMRES-DR
// (Morgan, SIAM J. Sci. Comput. 24 (2002) 20) and the deflation projections.
// Written for matrices of order <= a few hundred; column-major, 0-based.
//
// Algorithms (textbook forms, Golub & Van Loan, Matrix Computations, 4th ed.):
//   * LU with partial pivoting (Alg. 3.4.1) for H^{-dagger} e_m;
//   * Householder reduction to upper Hessenberg form with accumulated Q (Alg. 7.4.2);
//   * complex single-shift implicit QR with Wilkinson shift and deflation
//     (Alg. 7.5.1 adapted to complex arithmetic), accumulating Schur vectors;
//   * reordering of the complex Schur form by adjacent Givens swaps (Sec. 7.6.2);
//   * Householder QR of a tall matrix for least squares.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace qq {
namespace dense {

using cd = std::complex<double>;

struct Mat {
  int m = 0, n = 0;
  std::vector<cd> a;
  Mat() = default;
  Mat(int m_, int n_) : m(m_), n(n_), a((size_t)m_ * n_, cd(0, 0)) {}
  cd& operator()(int i, int j) { return a[(size_t)i + (size_t)m * j]; }
  const cd& operator()(int i, int j) const { return a[(size_t)i + (size_t)m * j]; }
};

inline Mat identity(int n) {
  Mat I(n, n);
  for (int i = 0; i < n; ++i) I(i, i) = 1.0;
  return I;
}

// Solve A x = b (A n x n, overwritten), partial pivoting.  Returns false if singular.
inline bool lu_solve(Mat A, std::vector<cd>& b) {
  const int n = A.n;
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::abs(A(k, k));
    for (int i = k + 1; i < n; ++i)
      if (std::abs(A(i, k)) > best) {
        best = std::abs(A(i, k));
        p = i;
      }
    if (best == 0.0) return false;
    piv[k] = p;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(A(k, j), A(p, j));
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < n; ++i) {
      const cd l = A(i, k) / A(k, k);
      A(i, k) = l;
      for (int j = k + 1; j < n; ++j) A(i, j) -= l * A(k, j);
      b[i] -= l * b[k];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    cd s = b[i];
    for (int j = i + 1; j < n; ++j) s -= A(i, j) * b[j];
    b[i] = s / A(i, i);
  }
  return true;
}

// Givens rotation G = [c s; -conj(s) c] (c real) with G [a; b] = [r; 0].
inline void givens(cd a, cd b, double& c, cd& s, cd& r) {
  const double ab = std::abs(b);
  if (ab == 0.0) {
    c = 1.0;
    s = 0.0;
    r = a;
    return;
  }
  const double aa = std::abs(a);
  if (aa == 0.0) {
    c = 0.0;
    s = std::conj(b) / ab;
    r = ab;
    return;
  }
  const double nrm = std::hypot(aa, ab);
  c = aa / nrm;
  const cd phase = a / aa;
  s = phase * std::conj(b) / nrm;
  r = phase * nrm;
}

// Apply G (acting on rows i, i+1) from the left to columns [j0, j1) of A.
inline void rot_rows(Mat& A, int i, double c, cd s, int j0, int j1) {
  for (int j = j0; j < j1; ++j) {
    const cd x = A(i, j), y = A(i + 1, j);
    A(i, j) = c * x + s * y;
    A(i + 1, j) = -std::conj(s) * x + c * y;
  }
}
// Apply G^dagger (acting on columns i, i+1) from the right to rows [r0, r1) of A.
inline void rot_cols(Mat& A, int i, double c, cd s, int r0, int r1) {
  for (int r = r0; r < r1; ++r) {
    const cd x = A(r, i), y = A(r, i + 1);
    A(r, i) = c * x + std::conj(s) * y;
    A(r, i + 1) = -s * x + c * y;
  }
}

// Householder reduction H = Q^dagger A Q to upper Hessenberg form; Q accumulated.
inline void hessenberg(Mat& A, Mat& Q) {
  const int n = A.n;
  Q = identity(n);
  std::vector<cd> v(n);
  for (int k = 0; k < n - 2; ++k) {
    double xnorm = 0.0;
    for (int i = k + 1; i < n; ++i) xnorm += std::norm(A(i, k));
    xnorm = std::sqrt(xnorm);
    if (xnorm == 0.0) continue;
    const cd x0 = A(k + 1, k);
    const cd alpha = (std::abs(x0) == 0.0 ? cd(1, 0) : x0 / std::abs(x0)) * (-xnorm);
    for (int i = 0; i < n; ++i) v[i] = 0.0;
    v[k + 1] = x0 - alpha;
    for (int i = k + 2; i < n; ++i) v[i] = A(i, k);
    double vn = 0.0;
    for (int i = k + 1; i < n; ++i) vn += std::norm(v[i]);
    if (vn == 0.0) continue;
    const double tau = 2.0 / vn;
    // A <- (I - tau v v^H) A
    for (int j = 0; j < n; ++j) {
      cd s = 0.0;
      for (int i = k + 1; i < n; ++i) s += std::conj(v[i]) * A(i, j);
      s *= tau;
      for (int i = k + 1; i < n; ++i) A(i, j) -= v[i] * s;
    }
    // A <- A (I - tau v v^H); Q <- Q (I - tau v v^H)
    for (int i = 0; i < n; ++i) {
      cd s = 0.0, t = 0.0;
      for (int j = k + 1; j < n; ++j) {
        s += A(i, j) * v[j];
        t += Q(i, j) * v[j];
      }
      s *= tau;
      t *= tau;
      for (int j = k + 1; j < n; ++j) {
        A(i, j) -= s * std::conj(v[j]);
        Q(i, j) -= t * std::conj(v[j]);
      }
    }
    for (int i = k + 2; i < n; ++i) A(i, k) = 0.0;
  }
}

// Complex Schur form T = Z^dagger H Z of an upper Hessenberg H (in place: H -> T),
// Z updated as Z <- Z * Q.  Returns false if the iteration count is exceeded.
inline bool schur(Mat& H, Mat& Z) {
  const int n = H.n;
  const double eps = 2.220446049250313e-16;
  int hi = n - 1;
  int iter = 0, total = 0;
  while (hi > 0) {
    // find the active block [lo, hi]
    int lo = hi;
    while (lo > 0) {
      const double s = std::abs(H(lo, lo)) + std::abs(H(lo - 1, lo - 1));
      if (std::abs(H(lo, lo - 1)) <= eps * (s == 0.0 ? 1.0 : s)) {
        H(lo, lo - 1) = 0.0;
        break;
      }
      --lo;
    }
    if (lo == hi) {
      --hi;
      iter = 0;
      continue;
    }
    if (++total > 60 * n) return false;
    ++iter;
    // Wilkinson shift from the trailing 2x2 block
    cd mu;
    if (iter % 11 == 10) {
      mu = H(hi, hi) + 0.75 * std::abs(H(hi, hi - 1));  // exceptional shift
    } else {
      const cd a = H(hi - 1, hi - 1), b = H(hi - 1, hi), c = H(hi, hi - 1), d = H(hi, hi);
      const cd tr = a + d, det = a * d - b * c;
      const cd disc = std::sqrt(tr * tr * 0.25 - det);
      const cd l1 = tr * 0.5 + disc, l2 = tr * 0.5 - disc;
      mu = std::abs(l1 - d) < std::abs(l2 - d) ? l1 : l2;
    }
    // implicit single-shift QR sweep on rows/cols lo..hi (bulge chase)
    cd x = H(lo, lo) - mu, y = H(lo + 1, lo);
    for (int k = lo; k < hi; ++k) {
      double c;
      cd s, r;
      givens(x, y, c, s, r);
      rot_rows(H, k, c, s, k > lo ? k - 1 : lo, n);
      rot_cols(H, k, c, s, 0, std::min(k + 3, hi + 1));
      rot_cols(Z, k, c, s, 0, Z.m);
      if (k > lo) H(k + 1, k - 1) = 0.0;
      if (k < hi - 1) {
        x = H(k + 1, k);
        y = H(k + 2, k);
      }
    }
  }
  for (int j = 0; j < n; ++j)
    for (int i = j + 1; i < n; ++i) H(i, j) = 0.0;
  return true;
}

// Swap the adjacent diagonal entries k, k+1 of an upper triangular T (Schur form),
// updating Z so that A = Z T Z^dagger still holds.
inline void schur_swap(Mat& T, Mat& Z, int k) {
  const int n = T.n;
  const cd t11 = T(k, k), t22 = T(k + 1, k + 1);
  // rotation G with G^H [T(k,k+1); t22 - t11] ~ e1 direction: (ZTREXC's choice)
  double c;
  cd s, r;
  givens(T(k, k + 1), t22 - t11, c, s, r);
  rot_rows(T, k, c, s, k, n);
  rot_cols(T, k, c, s, 0, k + 2);
  rot_cols(Z, k, c, s, 0, Z.m);
  T(k, k) = t22;
  T(k + 1, k + 1) = t11;
  T(k + 1, k) = 0.0;
}

// Reorder the Schur form so that the entries with sel[i] move (stably) to the top.
inline void schur_reorder(Mat& T, Mat& Z, std::vector<int> sel) {
  const int n = T.n;
  int ks = 0;
  for (int k = 0; k < n; ++k) {
    if (!sel[k]) continue;
    for (int j = k - 1; j >= ks; --j) {
      schur_swap(T, Z, j);
      std::swap(sel[j], sel[j + 1]);
    }
    ++ks;
  }
}

// Least squares min || c - Hb y || for an (m+1) x m upper Hessenberg Hb by Givens;
// returns y and the residual vector srv = c - Hb y (length m+1).
inline void hess_lsq(const Mat& Hb, const std::vector<cd>& c, int m, std::vector<cd>& y,
                     std::vector<cd>& srv) {
  Mat R(m + 1, m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i <= m; ++i) R(i, j) = Hb(i, j);
  std::vector<cd> g(c.begin(), c.begin() + m + 1);
  // general (k+1) x k dense leading block is handled by rotating every subdiagonal
  for (int j = 0; j < m; ++j)
    for (int i = m; i > j; --i) {
      if (std::abs(R(i, j)) == 0.0) continue;
      double cc;
      cd s, r;
      givens(R(i - 1, j), R(i, j), cc, s, r);
      rot_rows(R, i - 1, cc, s, j, m);
      const cd a = g[i - 1], b = g[i];
      g[i - 1] = cc * a + s * b;
      g[i] = -std::conj(s) * a + cc * b;
      R(i, j) = 0.0;
    }
  y.assign(m, 0.0);
  for (int i = m - 1; i >= 0; --i) {
    cd s = g[i];
    for (int j = i + 1; j < m; ++j) s -= R(i, j) * y[j];
    y[i] = s / R(i, i);
  }
  srv.assign(m + 1, 0.0);
  for (int i = 0; i <= m; ++i) {
    cd s = c[i];
    for (int j = 0; j < m; ++j) s -= Hb(i, j) * y[j];
    srv[i] = s;
  }
}

// Eigenvalues w and right eigenvectors (columns of V) of a general complex n x n A:
// Hessenberg reduction, complex Schur form T = Z^H A Z, then for each j the solution of
// (T - T_jj) y = 0 with y_j = 1 by back substitution (Golub & Van Loan Sec. 7.6.4; a
// denominator smaller than eps |T_jj| is replaced by that bound), and v_j = Z y.  Each
// column has unit 2-norm and its largest-modulus entry (the first on ties) real and
// positive, the normalisation of LAPACK's ZGEEV.  Returns false if QR did not converge.
inline bool eig_vectors(const Mat& A, std::vector<cd>& w, Mat& V) {
  const int n = A.n;
  Mat T = A, Z;
  hessenberg(T, Z);
  if (!schur(T, Z)) return false;
  const double eps = 2.220446049250313e-16, tiny = 1e-300;
  w.resize(n);
  for (int j = 0; j < n; ++j) w[j] = T(j, j);
  V = Mat(n, n);
  std::vector<cd> y(n);
  for (int j = 0; j < n; ++j) {
    const cd lam = T(j, j);
    const double smin = std::max(eps * std::abs(lam), tiny);
    std::fill(y.begin(), y.end(), cd(0, 0));
    y[j] = 1.0;
    for (int i = j - 1; i >= 0; --i) {
      cd s = 0.0;
      for (int l = i + 1; l <= j; ++l) s += T(i, l) * y[l];
      cd d = T(i, i) - lam;
      if (std::abs(d) < smin) d = smin;
      y[i] = -s / d;
    }
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) {
      cd s = 0.0;
      for (int l = 0; l <= j; ++l) s += Z(i, l) * y[l];
      V(i, j) = s;
      nrm += std::norm(s);
    }
    nrm = std::sqrt(nrm);
    int kmax = 0;
    double best = -1.0;
    for (int i = 0; i < n; ++i) {
      V(i, j) /= nrm;
      if (std::norm(V(i, j)) > best) {
        best = std::norm(V(i, j));
        kmax = i;
      }
    }
    const cd ph = std::conj(V(kmax, j)) / std::abs(V(kmax, j));
    for (int i = 0; i < n; ++i) V(i, j) *= ph;
    V(kmax, j) = cd(V(kmax, j).real(), 0.0);
  }
  return true;
}

// Householder QR of a tall m x n matrix A (m >= n): Q (m x n) with orthonormal columns
// and A = Q R, R upper triangular with a real positive diagonal (Householder
// reflectors, Golub & Van Loan Alg. 5.2.1, Q accumulated backwards as ZUNGQR does).
inline void house_q(const Mat& A, Mat& Q) {
  const int m = A.m, n = A.n;
  Mat R = A;
  std::vector<std::vector<cd>> vs(n);
  std::vector<double> taus(n, 0.0);
  for (int k = 0; k < n; ++k) {
    double xn = 0.0;
    for (int i = k; i < m; ++i) xn += std::norm(R(i, k));
    xn = std::sqrt(xn);
    std::vector<cd> v(m, 0.0);
    if (xn == 0.0) {
      vs[k] = v;
      continue;
    }
    const cd x0 = R(k, k);
    const cd alpha = (std::abs(x0) == 0.0 ? cd(1, 0) : x0 / std::abs(x0)) * (-xn);
    v[k] = x0 - alpha;
    for (int i = k + 1; i < m; ++i) v[i] = R(i, k);
    double vn = 0.0;
    for (int i = k; i < m; ++i) vn += std::norm(v[i]);
    const double tau = vn == 0.0 ? 0.0 : 2.0 / vn;
    for (int j = k; j < n; ++j) {
      cd s = 0.0;
      for (int i = k; i < m; ++i) s += std::conj(v[i]) * R(i, j);
      s *= tau;
      for (int i = k; i < m; ++i) R(i, j) -= v[i] * s;
    }
    vs[k] = v;
    taus[k] = tau;
  }
  // Q = H_0 H_1 ... H_{n-1} applied to the first n columns of the identity; each
  // column is then rotated so that R's diagonal is real and positive.
  Q = Mat(m, n);
  for (int j = 0; j < n; ++j) Q(j, j) = 1.0;
  for (int k = n - 1; k >= 0; --k) {
    const std::vector<cd>& v = vs[k];
    for (int j = 0; j < n; ++j) {
      cd s = 0.0;
      for (int i = k; i < m; ++i) s += std::conj(v[i]) * Q(i, j);
      s *= taus[k];
      for (int i = k; i < m; ++i) Q(i, j) -= v[i] * s;
    }
  }
  for (int j = 0; j < n; ++j) {
    const cd d = R(j, j);
    if (std::abs(d) == 0.0) continue;
    const cd ph = d / std::abs(d);
    for (int i = 0; i < m; ++i) Q(i, j) *= ph;
  }
}

// One GMRES-DR restart (Morgan 2002, steps 5-8): given Hb ((m+1) x m, the Arnoldi
// relation A V_m = V_{m+1} Hb) and the least-squares residual srv (length m+1),
// build P ((m+1) x (k+1), orthonormal columns), the new Hb_k = P^H Hb P_k
// ((k+1) x k), the new right-hand side cnew = P^H srv, and the harmonic Ritz values.
inline bool gmresdr_restart(const Mat& Hb, const std::vector<cd>& srv, int m, int k, Mat& P,
                            Mat& Hk, std::vector<cd>& cnew, std::vector<cd>& ritz) {
  // harmonic Ritz: eig(H_m + h^2 f e_m^T), f = H_m^{-dagger} e_m
  Mat Hm(m, m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) Hm(i, j) = Hb(i, j);
  Mat HmH(m, m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) HmH(i, j) = std::conj(Hm(j, i));
  std::vector<cd> f(m, 0.0);
  f[m - 1] = 1.0;
  if (!lu_solve(HmH, f)) return false;
  const cd h = Hb(m, m - 1);
  Mat A = Hm;
  for (int i = 0; i < m; ++i) A(i, m - 1) += h * h * f[i];
  Mat Q;
  hessenberg(A, Q);
  if (!schur(A, Q)) return false;
  ritz.resize(m);
  std::vector<double> mag(m);
  for (int i = 0; i < m; ++i) {
    ritz[i] = A(i, i);
    mag[i] = std::abs(ritz[i]);
  }
  std::vector<double> sorted = mag;
  std::sort(sorted.begin(), sorted.end());
  const double thr = sorted[k - 1];
  std::vector<int> sel(m);
  int nsel = 0;
  for (int i = 0; i < m; ++i) {
    sel[i] = (mag[i] <= thr && nsel < k) ? 1 : 0;
    nsel += sel[i];
  }
  schur_reorder(A, Q, sel);
  for (int i = 0; i < m; ++i) ritz[i] = A(i, i);
  // P = [ [Q_k; 0], srv orthogonalised ]  (twice, for safety)
  P = Mat(m + 1, k + 1);
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < m; ++i) P(i, j) = Q(i, j);
  std::vector<cd> p(srv);
  for (int pass = 0; pass < 2; ++pass)
    for (int j = 0; j < k; ++j) {
      cd d = 0.0;
      for (int i = 0; i <= m; ++i) d += std::conj(P(i, j)) * p[i];
      for (int i = 0; i <= m; ++i) p[i] -= d * P(i, j);
    }
  double nrm = 0.0;
  for (int i = 0; i <= m; ++i) nrm += std::norm(p[i]);
  nrm = std::sqrt(nrm);
  if (nrm == 0.0) return false;
  for (int i = 0; i <= m; ++i) P(i, k) = p[i] / nrm;
  // Hk = P^H Hb P_k
  Mat W(m + 1, k);
  for (int j = 0; j < k; ++j)
    for (int i = 0; i <= m; ++i) {
      cd s = 0.0;
      for (int l = 0; l < m; ++l) s += Hb(i, l) * P(l, j);
      W(i, j) = s;
    }
  Hk = Mat(k + 1, k);
  for (int j = 0; j < k; ++j)
    for (int i = 0; i <= k; ++i) {
      cd s = 0.0;
      for (int l = 0; l <= m; ++l) s += std::conj(P(l, i)) * W(l, j);
      Hk(i, j) = s;
    }
  cnew.assign(k + 1, 0.0);
  for (int i = 0; i <= k; ++i) {
    cd s = 0.0;
    for (int l = 0; l <= m; ++l) s += std::conj(P(l, i)) * srv[l];
    cnew[i] = s;
  }
  return true;
}

}  // namespace dense
}  // namespace qq
