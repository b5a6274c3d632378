// CPU oracle (test infrastructure): restatement of the pseudolapack routines that
// GMRES-DR uses -- Q/pseudolapack.f90 linearsolver :45-75, orgschur :252-305,
// LUfactor :309-385, schurswap :389-463, hessenberg :700-770, qgenerator :774-864,
// evalues :868-1211 (the nh < maxb branch, which calls QRdouble), QRdouble :2196-2504,
// makereflector :2508-2603, multreflector :2607-2652, mvutil1 :2656-2734,
// mvutil2 :2738-2766, mvutil5 :3005-3033, mvutil6 :3037-3078, mmutil2 :3169-3257,
// rowswap :3261-3318, rotatecomp :3609-3720, twonorm, compdiv, pythag2/3, safesqrt.
// Constants dlamchs/dlamche/dlamchp/dlamch1 are the module parameters at :25-29.
// Parity unpinned against the Fortran (see oracle.h); checked against scipy LAPACK.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {
constexpr double dlamchs = 2.3e-308, dlamche = 1.2e-16, dlamchp = 2.3e-16,
                 dlamch1 = 2.0e-146;

// Column-major complex matrix view, 1-based (i,j).
struct CM {
  double* p;
  int ld;
  double& r(int i, int j) const { return p[2 * ((size_t)(i - 1) + (size_t)ld * (j - 1))]; }
  double& c(int i, int j) const { return p[2 * ((size_t)(i - 1) + (size_t)ld * (j - 1)) + 1]; }
  double* at(int i, int j) const { return p + 2 * ((size_t)(i - 1) + (size_t)ld * (j - 1)); }
  CM sub(int i, int j) const { return CM{at(i, j), ld}; }
};
// Complex vector view, 1-based.
struct CV {
  double* p;
  double& r(int i) const { return p[2 * (i - 1)]; }
  double& c(int i) const { return p[2 * (i - 1) + 1]; }
};

inline double fsign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }

double twonorm(const double* x, int n) {
  if (n < 1) return 0.0;
  double bigscale = 0.0, ssq = 1.0;
  for (int ix = 0; ix < n; ++ix)
    for (int part = 0; part < 2; ++part) {
      const double v = x[2 * ix + part];
      if (v != 0.0) {
        const double temp = std::fabs(v);
        if (bigscale < temp) {
          ssq = 1.0 + ssq * (bigscale / temp) * (bigscale / temp);
          bigscale = temp;
        } else {
          ssq = ssq + (temp / bigscale) * (temp / bigscale);
        }
      }
    }
  return bigscale * std::sqrt(ssq);
}

void compdiv(const double* a, const double* b, double* p) {
  double c, d, p0, p1;
  if (std::fabs(b[1]) < std::fabs(b[0])) {
    c = b[1] / b[0];
    d = b[0] + b[1] * c;
    p0 = (a[0] + a[1] * c) / d;
    p1 = (a[1] - a[0] * c) / d;
  } else {
    c = b[0] / b[1];
    d = b[1] + b[0] * c;
    p0 = (a[1] + a[0] * c) / d;
    p1 = (-a[0] + a[1] * c) / d;
  }
  p[0] = p0;
  p[1] = p1;
}

double pythag2(double x, double y) {
  double xabs = std::fabs(x), yabs = std::fabs(y);
  double w = std::fmax(xabs, yabs), z = std::fmin(xabs, yabs);
  if (z == 0.0) return w;
  return w * std::sqrt(1.0 + (z / w) * (z / w));
}

double pythag3(double x, double y, double z) {
  double xabs = std::fabs(x), yabs = std::fabs(y), zabs = std::fabs(z);
  double w = std::fmax(xabs, std::fmax(yabs, zabs));
  if (w == 0.0) return 0.0;
  return w * std::sqrt((xabs / w) * (xabs / w) + (yabs / w) * (yabs / w) + (zabs / w) * (zabs / w));
}

void safesqrt(const double* x, double* y) {
  y[0] = std::sqrt(0.5 * (std::sqrt(x[0] * x[0] + x[1] * x[1]) + x[0]));
  if (y[0] != 0.0) {
    y[1] = 0.5 * x[1] / y[0];
  } else {
    y[1] = std::sqrt(0.5 * (std::sqrt(x[0] * x[0] + x[1] * x[1]) - x[0]));
    if (y[1] != 0.0) {
      y[0] = 0.5 * x[1] / y[1];
    } else {
      y[0] = y[1] = 0.0;
    }
  }
}

// x has n-1 complex entries (contiguous).
void makereflector(int n, double* alpha, double* x, double* tau) {
  const double safmin = dlamchs / dlamche;
  if (n < 1) {
    tau[0] = tau[1] = 0.0;
    return;
  }
  double xnorm = twonorm(x, n - 1);
  if (xnorm == 0.0 && alpha[1] == 0.0) {
    tau[0] = tau[1] = 0.0;
    return;
  }
  double beta = -fsign(pythag3(alpha[0], alpha[1], xnorm), alpha[0]);
  const double rsafmn = 1.0 / safmin;
  int knt = 0;
  if (std::fabs(beta) < safmin) {
    for (;;) {
      knt += 1;
      for (int i = 0; i < n - 1; ++i) {
        x[2 * i] *= rsafmn;
        x[2 * i + 1] *= rsafmn;
      }
      beta = rsafmn * beta;
      alpha[0] = rsafmn * alpha[0];
      alpha[1] = rsafmn * alpha[1];
      if (std::fabs(beta) >= safmin) break;
    }
    xnorm = twonorm(x, n - 1);
    beta = -fsign(pythag3(alpha[0], alpha[1], xnorm), alpha[0]);
  }
  tau[0] = (beta - alpha[0]) / beta;
  tau[1] = -alpha[1] / beta;
  double a[2] = {1.0, 0.0};
  double b[2] = {alpha[0] - beta, alpha[1]};
  compdiv(a, b, alpha);
  for (int i = 0; i < n - 1; ++i) {
    double xRe = alpha[0] * x[2 * i] - alpha[1] * x[2 * i + 1];
    x[2 * i + 1] = alpha[0] * x[2 * i + 1] + alpha[1] * x[2 * i];
    x[2 * i] = xRe;
  }
  alpha[0] = beta;
  alpha[1] = 0.0;
  for (int i = 0; i < knt; ++i) {
    alpha[0] *= safmin;
    alpha[1] *= safmin;
  }
}

// y = alpha*op(a)*x + beta*y ; op = a (dagger=0, a is m x n) or a^dagger (dagger=1)
void mvutil1(int dagger, int m, int n, const double* alpha, CM a, const double* x,
             const double* beta, double* y) {
  if (!(m > 0 && n > 0 &&
        (alpha[0] != 0.0 || alpha[1] != 0.0 || beta[0] != 1.0 || beta[1] != 0.0)))
    return;
  int leny = dagger == 0 ? m : n;
  if (beta[0] != 1.0 || beta[1] != 0.0) {
    if (beta[0] == 0.0 && beta[1] == 0.0) {
      for (int i = 0; i < leny; ++i) y[2 * i] = y[2 * i + 1] = 0.0;
    } else {
      for (int i = 0; i < leny; ++i) {
        double yRe = beta[0] * y[2 * i] - beta[1] * y[2 * i + 1];
        y[2 * i + 1] = beta[0] * y[2 * i + 1] + beta[1] * y[2 * i];
        y[2 * i] = yRe;
      }
    }
  }
  if (alpha[0] == 0.0 && alpha[1] == 0.0) return;
  if (dagger == 0) {
    for (int j = 1; j <= n; ++j) {
      const double xr = x[2 * (j - 1)], xi = x[2 * (j - 1) + 1];
      if (xr != 0.0 || xi != 0.0) {
        double t0 = alpha[0] * xr - alpha[1] * xi;
        double t1 = alpha[0] * xi + alpha[1] * xr;
        for (int i = 1; i <= m; ++i) {
          y[2 * (i - 1)] = y[2 * (i - 1)] + t0 * a.r(i, j) - t1 * a.c(i, j);
          y[2 * (i - 1) + 1] = y[2 * (i - 1) + 1] + t0 * a.c(i, j) + t1 * a.r(i, j);
        }
      }
    }
  } else {
    for (int j = 1; j <= n; ++j) {
      double t0 = 0.0, t1 = 0.0;
      for (int i = 1; i <= m; ++i) {
        t0 = t0 + a.r(i, j) * x[2 * (i - 1)] + a.c(i, j) * x[2 * (i - 1) + 1];
        t1 = t1 + a.r(i, j) * x[2 * (i - 1) + 1] - a.c(i, j) * x[2 * (i - 1)];
      }
      y[2 * (j - 1)] = y[2 * (j - 1)] + alpha[0] * t0 - alpha[1] * t1;
      y[2 * (j - 1) + 1] = y[2 * (j - 1) + 1] + alpha[0] * t1 + alpha[1] * t0;
    }
  }
}

// a += alpha * x * y^dagger   (m x n)
void mvutil2(int m, int n, const double* alpha, const double* x, const double* y, CM a) {
  if (!(m != 0 && n != 0 && (alpha[0] != 0.0 || alpha[1] != 0.0))) return;
  for (int j = 1; j <= n; ++j) {
    const double yr = y[2 * (j - 1)], yi = y[2 * (j - 1) + 1];
    if (yr != 0.0 || yi != 0.0) {
      double t0 = alpha[0] * yr + alpha[1] * yi;
      double t1 = alpha[1] * yr - alpha[0] * yi;
      for (int i = 1; i <= m; ++i) {
        const double xr = x[2 * (i - 1)], xi = x[2 * (i - 1) + 1];
        a.r(i, j) = a.r(i, j) + xr * t0 - xi * t1;
        a.c(i, j) = a.c(i, j) + xr * t1 + xi * t0;
      }
    }
  }
}

// a += alpha * x * y^T  (x stride-1 column, y with stride ldy complex entries)
void mvutil5(int m, int n, const double* alpha, const double* x, const double* y, int ldy,
             CM a) {
  if (!(m != 0 && n != 0 && (alpha[0] != 0.0 || alpha[1] != 0.0))) return;
  for (int j = 1; j <= n; ++j) {
    const double yr = y[2 * (size_t)ldy * (j - 1)], yi = y[2 * (size_t)ldy * (j - 1) + 1];
    if (yr != 0.0 || yi != 0.0) {
      double t0 = alpha[0] * yr - alpha[1] * yi;
      double t1 = alpha[1] * yr + alpha[0] * yi;
      for (int i = 1; i <= m; ++i) {
        const double xr = x[2 * (i - 1)], xi = x[2 * (i - 1) + 1];
        a.r(i, j) = a.r(i, j) + xr * t0 - xi * t1;
        a.c(i, j) = a.c(i, j) + xr * t1 + xi * t0;
      }
    }
  }
}

void LUfactor(int m, int n, CM a, int* ipiv) {
  const double minusone[2] = {-1.0, 0.0};
  const int mn = m < n ? m : n;
  for (int j = 1; j <= mn; ++j) {
    int jp = j;
    if (m > j) {
      double smax = std::fabs(a.r(j, j)) + std::fabs(a.c(j, j));
      for (int i = j + 1; i <= m; ++i) {
        double stry = std::fabs(a.r(i, j)) + std::fabs(a.c(i, j));
        if (stry > smax) {
          jp = i;
          smax = stry;
        }
      }
    }
    ipiv[j - 1] = jp;
    if (a.r(jp, j) != 0.0 || a.c(jp, j) != 0.0) {
      if (jp != j) {
        for (int i = 1; i <= n; ++i) {
          double t0 = a.r(j, i), t1 = a.c(j, i);
          a.r(j, i) = a.r(jp, i);
          a.c(j, i) = a.c(jp, i);
          a.r(jp, i) = t0;
          a.c(jp, i) = t1;
        }
      }
      if (j < m) {
        const double den = a.r(j, j) * a.r(j, j) + a.c(j, j) * a.c(j, j);
        const double at0 = a.r(j, j) / den;
        const double at1 = -a.c(j, j) / den;
        for (int i = j + 1; i <= m; ++i) {
          double stry = at0 * a.r(i, j) - at1 * a.c(i, j);
          a.c(i, j) = at0 * a.c(i, j) + at1 * a.r(i, j);
          a.r(i, j) = stry;
        }
      }
    } else {
      // The reference writes PSEUDOLAPACK.ERROR and stops; the oracle records the
      // singularity by leaving a zero pivot (callers check ipiv[j-1] < 0).
      ipiv[j - 1] = -j;
      return;
    }
    int row = m - j, col = n - j;
    if (j < mn) mvutil5(row, col, minusone, a.at(j + 1, j), a.at(j, j + 1), a.ld, a.sub(j + 1, j + 1));
  }
}

void mmutil2(bool upper, int m, int n, CM a, CM b) {
  // alpha = (1,0) at every call site: the scaling branches are no-ops.
  if (upper) {
    for (int j = 1; j <= n; ++j)
      for (int k = m; k >= 1; --k) {
        if (b.r(k, j) != 0.0 || b.c(k, j) != 0.0) {
          double denom = 1.0 / (a.r(k, k) * a.r(k, k) + a.c(k, k) * a.c(k, k));
          double temp = denom * (b.r(k, j) * a.r(k, k) + b.c(k, j) * a.c(k, k));
          b.c(k, j) = denom * (b.c(k, j) * a.r(k, k) - b.r(k, j) * a.c(k, k));
          b.r(k, j) = temp;
          for (int i = 1; i <= k - 1; ++i) {
            temp = b.r(i, j) - b.r(k, j) * a.r(i, k) + b.c(k, j) * a.c(i, k);
            b.c(i, j) = b.c(i, j) - b.r(k, j) * a.c(i, k) - b.c(k, j) * a.r(i, k);
            b.r(i, j) = temp;
          }
        }
      }
  } else {
    for (int j = 1; j <= n; ++j)
      for (int k = 1; k <= m; ++k) {
        if (b.r(k, j) != 0.0 || b.c(k, j) != 0.0) {
          for (int i = k + 1; i <= m; ++i) {
            double temp = b.r(i, j) - b.r(k, j) * a.r(i, k) + b.c(k, j) * a.c(i, k);
            b.c(i, j) = b.c(i, j) - b.r(k, j) * a.c(i, k) - b.c(k, j) * a.r(i, k);
            b.r(i, j) = temp;
          }
        }
      }
  }
}

void rowswap(int n, CM a, int k1, int k2, const int* ipiv) {
  // The reference blocks the columns by 32; the swap sequence per column is identical.
  for (int k = 1; k <= n; ++k) {
    int ix = k1;
    for (int i = k1; i <= k2; ++i) {
      int ip = ipiv[ix - 1];
      if (ip != i) {
        double t0 = a.r(i, k), t1 = a.c(i, k);
        a.r(i, k) = a.r(ip, k);
        a.c(i, k) = a.c(ip, k);
        a.r(ip, k) = t0;
        a.c(ip, k) = t1;
      }
      ix += 1;
    }
  }
}

void multreflector(bool left, int m, int n, const double* v, const double* tau, CM c,
                   double* work) {
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  if (tau[0] != 0.0 || tau[1] != 0.0) {
    const double mtau[2] = {-tau[0], -tau[1]};
    if (left) {
      mvutil1(1, m, n, one, c, v, zero, work);
      mvutil2(m, n, mtau, v, work, c);
    } else {
      mvutil1(0, m, n, one, c, v, zero, work);
      mvutil2(m, n, mtau, work, v, c);
    }
  }
}

void rotatecomp(const double* f, const double* g, double* cs, double* sn, double* r) {
  int iflag = 0;
  const double safmin = dlamchs;
  const double safmn2 = dlamch1;
  const double safmx2 = 1.0 / safmn2;
  double myscale = std::fmax(std::fmax(std::fabs(f[0]), std::fabs(f[1])),
                             std::fmax(std::fabs(g[0]), std::fabs(g[1])));
  double fs[2] = {f[0], f[1]}, gs[2] = {g[0], g[1]};
  int icount = 0;
  if (myscale >= safmx2) {
    for (;;) {
      icount += 1;
      fs[0] *= safmn2; fs[1] *= safmn2;
      gs[0] *= safmn2; gs[1] *= safmn2;
      myscale *= safmn2;
      if (myscale < safmx2) break;
    }
  } else if (myscale <= safmn2) {
    if (g[0] == 0.0 && g[1] == 0.0) {
      *cs = 1.0;
      sn[0] = sn[1] = 0.0;
      r[0] = f[0];
      r[1] = f[1];
      iflag = 1;
    }
    if (iflag == 0) {
      for (;;) {
        icount -= 1;
        fs[0] *= safmx2; fs[1] *= safmx2;
        gs[0] *= safmx2; gs[1] *= safmx2;
        myscale *= safmx2;
        if (myscale > safmn2) break;
      }
    }
  }
  if (iflag != 0) return;
  double f2 = fs[0] * fs[0] + fs[1] * fs[1];
  double g2 = gs[0] * gs[0] + gs[1] * gs[1];
  if (f2 <= std::fmax(g2, 1.0) * safmin) {
    if (f[0] == 0.0 && f[1] == 0.0) {
      *cs = 0.0;
      r[0] = pythag2(g[0], g[1]);
      r[1] = 0.0;  // r is declared complex; the reference assigns a real to both parts
      double d = pythag2(gs[0], gs[1]);
      sn[0] = gs[0] / d;
      sn[1] = -gs[1] / d;
      return;
    }
    double f2s = pythag2(fs[0], fs[1]);
    double g2s = std::sqrt(g2);
    *cs = f2s / g2s;
    double ff[2];
    if (std::fmax(std::fabs(f[0]), std::fabs(f[1])) > 1.0) {
      double d = pythag2(f[0], f[1]);
      ff[0] = f[0] / d;
      ff[1] = f[1] / d;
    } else {
      double dr = safmx2 * f[0], di = safmx2 * f[1];
      double d = pythag2(dr, di);
      ff[0] = dr / d;
      ff[1] = di / d;
    }
    sn[0] = (ff[0] * gs[0] + ff[1] * gs[1]) / g2s;
    sn[1] = (ff[1] * gs[0] - ff[0] * gs[1]) / g2s;
    r[0] = *cs * f[0] + sn[0] * g[0] - sn[1] * g[1];
    r[1] = *cs * f[1] + sn[0] * g[1] + sn[1] * g[0];
  } else {
    double f2s = std::sqrt(1.0 + g2 / f2);
    r[0] = f2s * fs[0];
    r[1] = f2s * fs[1];
    *cs = 1.0 / f2s;
    double d = f2 + g2;
    sn[0] = r[0] / d;
    sn[1] = r[1] / d;
    double temp = sn[0] * gs[0] + sn[1] * gs[1];
    sn[1] = sn[1] * gs[0] - sn[0] * gs[1];
    sn[0] = temp;
    if (icount > 0) {
      for (int i = 0; i < icount; ++i) { r[0] *= safmx2; r[1] *= safmx2; }
    } else if (icount < 0) {
      for (int i = 0; i < -icount; ++i) { r[0] *= safmn2; r[1] *= safmn2; }
    }
  }
}

void schurswap(int n, CM t, CM q, int ifst, int ilst) {
  if (!(n > 1 && ifst != ilst)) return;
  int m1, m2, m3;
  if (ifst < ilst) {
    m1 = 0; m2 = -1; m3 = 1;
  } else {
    m1 = -1; m2 = 0; m3 = -1;
  }
  for (int k = ifst + m1; m3 > 0 ? k <= ilst + m2 : k >= ilst + m2; k += m3) {
    double t11[2] = {t.r(k, k), t.c(k, k)};
    double t22[2] = {t.r(k + 1, k + 1), t.c(k + 1, k + 1)};
    double temp[2] = {t22[0] - t11[0], t22[1] - t11[1]};
    double cs, sn[2], rr[2];
    double fk[2] = {t.r(k, k + 1), t.c(k, k + 1)};
    rotatecomp(fk, temp, &cs, sn, rr);
    if (k + 2 <= n) {
      for (int i = k + 2; i <= n; ++i) {
        double a0 = cs * t.r(k, i) + sn[0] * t.r(k + 1, i) - sn[1] * t.c(k + 1, i);
        double a1 = cs * t.c(k, i) + sn[0] * t.c(k + 1, i) + sn[1] * t.r(k + 1, i);
        double b0 = cs * t.r(k + 1, i) - sn[0] * t.r(k, i) - sn[1] * t.c(k, i);
        double b1 = cs * t.c(k + 1, i) - sn[0] * t.c(k, i) + sn[1] * t.r(k, i);
        t.r(k + 1, i) = b0;
        t.c(k + 1, i) = b1;
        t.r(k, i) = a0;
        t.c(k, i) = a1;
      }
    }
    for (int i = 1; i <= k - 1; ++i) {
      double a0 = cs * t.r(i, k) + sn[0] * t.r(i, k + 1) + sn[1] * t.c(i, k + 1);
      double a1 = cs * t.c(i, k) + sn[0] * t.c(i, k + 1) - sn[1] * t.r(i, k + 1);
      double b0 = cs * t.r(i, k + 1) - sn[0] * t.r(i, k) + sn[1] * t.c(i, k);
      double b1 = cs * t.c(i, k + 1) - sn[0] * t.c(i, k) - sn[1] * t.r(i, k);
      t.r(i, k + 1) = b0;
      t.c(i, k + 1) = b1;
      t.r(i, k) = a0;
      t.c(i, k) = a1;
    }
    t.r(k, k) = t22[0];
    t.c(k, k) = t22[1];
    t.r(k + 1, k + 1) = t11[0];
    t.c(k + 1, k + 1) = t11[1];
    for (int i = 1; i <= n; ++i) {
      double a0 = cs * q.r(i, k) + sn[0] * q.r(i, k + 1) + sn[1] * q.c(i, k + 1);
      double a1 = cs * q.c(i, k) + sn[0] * q.c(i, k + 1) - sn[1] * q.r(i, k + 1);
      double b0 = cs * q.r(i, k + 1) - sn[0] * q.r(i, k) + sn[1] * q.c(i, k);
      double b1 = cs * q.c(i, k + 1) - sn[0] * q.c(i, k) - sn[1] * q.r(i, k);
      q.r(i, k + 1) = b0;
      q.c(i, k + 1) = b1;
      q.r(i, k) = a0;
      q.c(i, k) = a1;
    }
  }
}

// Returns 0 on success, 1 if the iteration limit was hit (the reference stops).
int QRdouble(int ischur, int n, int ilo, int ihi, CM h, double* w, int iloz, int ihiz, CM z) {
  if (n == 0) return 0;
  if (ilo == ihi) {
    w[2 * (ilo - 1)] = h.r(ilo, ilo);
    w[2 * (ilo - 1) + 1] = h.c(ilo, ilo);
    return 0;
  }
  const double ulp = dlamchp;
  const double smlnum = dlamchs / ulp;
  int i1 = 0, i2 = 0;
  if (ischur == 1) {
    i1 = 1;
    i2 = n;
  }
  int itn = 30 * (ihi - ilo + 1);
  int i = ihi;
  while (i >= ilo) {
    int l = ilo;
    int its = -1;
    int iflag = 0;
    for (;;) {
      its += 1;
      if (its > itn) break;
      int k = i + 1;
      for (;;) {
        k -= 1;
        if (k < l + 1) break;
        double tst1 = std::fabs(h.r(k - 1, k - 1)) + std::fabs(h.c(k - 1, k - 1)) +
                      std::fabs(h.r(k, k)) + std::fabs(h.c(k, k));
        if (tst1 == 0.0 && i + 1 != l) {
          for (int j = l; j <= i; ++j) {
            double myrsum = 0.0;
            for (int ii = l; ii <= std::min(i, j + 1); ++ii)
              myrsum = myrsum + std::sqrt(h.r(ii, j) * h.r(ii, j) + h.c(ii, j) * h.c(ii, j));
            tst1 = std::fmax(tst1, myrsum);
          }
        }
        if (std::fabs(h.r(k, k - 1)) <= std::fmax(ulp * tst1, smlnum)) break;
      }
      l = k;
      if (l > ilo) {
        h.r(l, l - 1) = 0.0;
        h.c(l, l - 1) = 0.0;
      }
      if (l < i) {
        iflag = 0;
      } else {
        iflag = 1;
        break;
      }
      if (ischur == 0) {
        i1 = l;
        i2 = i;
      }
      double t[2];
      if (its == 10 || its == 20) {
        double s = 0.75 * std::fabs(h.r(i, i - 1));
        t[0] = s + h.r(i, i);
        t[1] = h.c(i, i);
      } else {
        t[0] = h.r(i, i);
        t[1] = h.c(i, i);
        double u[2] = {h.r(i - 1, i) * h.r(i, i - 1), h.c(i - 1, i) * h.r(i, i - 1)};
        if (u[0] != 0.0 || u[1] != 0.0) {
          double x[2] = {0.5 * (h.r(i - 1, i - 1) - t[0]), 0.5 * (h.c(i - 1, i - 1) - t[1])};
          double ytemp[2] = {x[0] * x[0] - x[1] * x[1] + u[0], 2.0 * x[0] * x[1] + u[1]};
          double y[2];
          safesqrt(ytemp, y);
          if (x[0] * y[0] + x[1] * y[1] < 0.0) {
            y[0] = -y[0];
            y[1] = -y[1];
          }
          double xy[2] = {x[0] + y[0], x[1] + y[1]};
          double tbit[2];
          compdiv(u, xy, tbit);
          t[0] = t[0] - tbit[0];
          t[1] = t[1] - tbit[1];
        }
      }
      int jflag = 0;
      int m = i;
      double v[4];  // v(:,1), v(:,2)
      for (;;) {
        m -= 1;
        if (m < l + 1) break;
        double h11[2] = {h.r(m, m), h.c(m, m)};
        double h22[2] = {h.r(m + 1, m + 1), h.c(m + 1, m + 1)};
        double h11s[2] = {h11[0] - t[0], h11[1] - t[1]};
        double h21[2] = {h.r(m + 1, m), h.c(m + 1, m)};
        double s = std::fabs(h11s[0]) + std::fabs(h11s[1]) + std::sqrt(h21[0] * h21[0] + h21[1] * h21[1]);
        h11s[0] /= s; h11s[1] /= s;
        h21[0] /= s; h21[1] /= s;
        v[0] = h11s[0]; v[1] = h11s[1]; v[2] = h21[0]; v[3] = h21[1];
        double h10[2] = {h.r(m, m - 1), h.c(m, m - 1)};
        double tst1 = (std::fabs(h11s[0]) + std::fabs(h11s[1])) *
                      (std::fabs(h11[0]) + std::fabs(h11[1]) + std::fabs(h22[0]) + std::fabs(h22[1]));
        double a = h10[0] * h21[0] - h10[1] * h21[1];
        double b = h10[0] * h21[1] + h10[1] * h21[0];
        double myrsum = std::sqrt(a * a + b * b);
        if (myrsum <= ulp * tst1) {
          jflag = 1;
          break;
        }
      }
      if (jflag == 0) {
        double h11[2] = {h.r(l, l), h.c(l, l)};
        double h11s[2] = {h11[0] - t[0], h11[1] - t[1]};
        double h21[2] = {h.r(l + 1, l), h.c(l + 1, l)};
        double s = std::fabs(h11s[0]) + std::fabs(h11s[1]) + std::sqrt(h21[0] * h21[0] + h21[1] * h21[1]);
        h11s[0] /= s; h11s[1] /= s;
        h21[0] /= s; h21[1] /= s;
        v[0] = h11s[0]; v[1] = h11s[1]; v[2] = h21[0]; v[3] = h21[1];
      }
      for (int k2 = m; k2 <= i - 1; ++k2) {
        if (k2 > m) {
          v[0] = h.r(k2, k2 - 1); v[1] = h.c(k2, k2 - 1);
          v[2] = h.r(k2 + 1, k2 - 1); v[3] = h.c(k2 + 1, k2 - 1);
        }
        double t1[2];
        makereflector(2, v, v + 2, t1);
        if (k2 > m) {
          h.r(k2, k2 - 1) = v[0]; h.c(k2, k2 - 1) = v[1];
          h.r(k2 + 1, k2 - 1) = 0.0; h.c(k2 + 1, k2 - 1) = 0.0;
        }
        double t2 = t1[0] * v[2] - t1[1] * v[3];
        for (int j = k2; j <= i2; ++j) {
          double s0 = t1[0] * h.r(k2, j) + t1[1] * h.c(k2, j) + t2 * h.r(k2 + 1, j);
          double s1 = t1[0] * h.c(k2, j) - t1[1] * h.r(k2, j) + t2 * h.c(k2 + 1, j);
          h.r(k2, j) = h.r(k2, j) - s0;
          h.c(k2, j) = h.c(k2, j) - s1;
          h.r(k2 + 1, j) = h.r(k2 + 1, j) - s0 * v[2] + s1 * v[3];
          h.c(k2 + 1, j) = h.c(k2 + 1, j) - s0 * v[3] - s1 * v[2];
        }
        for (int j = i1; j <= std::min(k2 + 2, i); ++j) {
          double s0 = t1[0] * h.r(j, k2) - t1[1] * h.c(j, k2) + t2 * h.r(j, k2 + 1);
          double s1 = t1[0] * h.c(j, k2) + t1[1] * h.r(j, k2) + t2 * h.c(j, k2 + 1);
          h.r(j, k2) = h.r(j, k2) - s0;
          h.c(j, k2) = h.c(j, k2) - s1;
          h.r(j, k2 + 1) = h.r(j, k2 + 1) - s0 * v[2] - s1 * v[3];
          h.c(j, k2 + 1) = h.c(j, k2 + 1) - s1 * v[2] + s0 * v[3];
        }
        if (ischur == 1) {
          for (int j = iloz; j <= ihiz; ++j) {
            double s0 = t1[0] * z.r(j, k2) - t1[1] * z.c(j, k2) + t2 * z.r(j, k2 + 1);
            double s1 = t1[0] * z.c(j, k2) + t1[1] * z.r(j, k2) + t2 * z.c(j, k2 + 1);
            z.r(j, k2) = z.r(j, k2) - s0;
            z.c(j, k2) = z.c(j, k2) - s1;
            z.r(j, k2 + 1) = z.r(j, k2 + 1) - s0 * v[2] - s1 * v[3];
            z.c(j, k2 + 1) = z.c(j, k2 + 1) - s1 * v[2] + s0 * v[3];
          }
        }
        if (k2 == m && m > l) {
          double temp[2] = {1.0 - t1[0], 0.0 - t1[1]};
          double myrsum = std::sqrt(temp[0] * temp[0] + temp[1] * temp[1]);
          temp[0] /= myrsum;
          temp[1] /= myrsum;
          double hRe = h.r(m + 1, m) * temp[0] + h.c(m + 1, m) * temp[1];
          h.c(m + 1, m) = h.c(m + 1, m) * temp[0] - h.r(m + 1, m) * temp[1];
          h.r(m + 1, m) = hRe;
          if (m + 2 <= i) {
            hRe = h.r(m + 2, m + 1) * temp[0] - h.c(m + 2, m + 1) * temp[1];
            h.c(m + 2, m + 1) = h.c(m + 2, m + 1) * temp[0] + h.r(m + 2, m + 1) * temp[1];
            h.r(m + 2, m + 1) = hRe;
          }
          for (int j = m; j <= i; ++j) {
            if (j != m + 1) {
              if (i2 > j) {
                for (int ii = j + 1; ii <= i2; ++ii) {
                  hRe = temp[0] * h.r(j, ii) - temp[1] * h.c(j, ii);
                  h.c(j, ii) = temp[0] * h.c(j, ii) + temp[1] * h.r(j, ii);
                  h.r(j, ii) = hRe;
                }
              }
              for (int ii = i1; ii <= j - 1; ++ii) {
                hRe = temp[0] * h.r(ii, j) + temp[1] * h.c(ii, j);
                h.c(ii, j) = temp[0] * h.c(ii, j) - temp[1] * h.r(ii, j);
                h.r(ii, j) = hRe;
              }
              if (ischur == 1) {
                for (int ii = iloz; ii <= ihiz; ++ii) {
                  hRe = temp[0] * z.r(ii, j) + temp[1] * z.c(ii, j);
                  z.c(ii, j) = temp[0] * z.c(ii, j) - temp[1] * z.r(ii, j);
                  z.r(ii, j) = hRe;
                }
              }
            }
          }
        }
      }
      double temp[2] = {h.r(i, i - 1), h.c(i, i - 1)};
      if (temp[1] != 0.0) {
        double rtemp = std::sqrt(temp[0] * temp[0] + temp[1] * temp[1]);
        h.r(i, i - 1) = rtemp;
        h.c(i, i - 1) = 0.0;
        temp[0] /= rtemp;
        temp[1] /= rtemp;
        if (i2 > i) {
          for (int ii = i + 1; ii <= i2; ++ii) {
            double hRe = temp[0] * h.r(i, ii) + temp[1] * h.c(i, ii);
            h.c(i, ii) = temp[0] * h.c(i, ii) - temp[1] * h.r(i, ii);
            h.r(i, ii) = hRe;
          }
        }
        for (int ii = i1; ii <= i - 1; ++ii) {
          double hRe = temp[0] * h.r(ii, i) - temp[1] * h.c(ii, i);
          h.c(ii, i) = temp[0] * h.c(ii, i) + temp[1] * h.r(ii, i);
          h.r(ii, i) = hRe;
        }
        if (ischur == 1) {
          for (int ii = iloz; ii <= ihiz; ++ii) {
            double hRe = temp[0] * z.r(ii, i) - temp[1] * z.c(ii, i);
            z.c(ii, i) = temp[0] * z.c(ii, i) + temp[1] * z.r(ii, i);
            z.r(ii, i) = hRe;
          }
        }
      }
    }
    if (iflag == 0) return 1;  // "Failed to converge in QRdouble."
    w[2 * (i - 1)] = h.r(i, i);
    w[2 * (i - 1) + 1] = h.c(i, i);
    itn = itn - its;
    i = l - 1;
  }
  return 0;
}
}  // namespace

extern "C" void oq_linearsolver(int n, int nrhs, double* a, int lda, int* ipiv, double* b,
                                int ldb) {
  CM A{a, lda}, B{b, ldb};
  LUfactor(n, n, A, ipiv);
  if (n > 0 && ipiv[n - 1] < 0) return;
  for (int j = 0; j < n; ++j)
    if (ipiv[j] < 0) return;
  rowswap(nrhs, B, 1, n, ipiv);
  mmutil2(false, n, nrhs, A, B);
  mmutil2(true, n, nrhs, A, B);
}

extern "C" void oq_hessenberg(double* a, int lda, int n, int ilo, int ihi, double* tau) {
  CM A{a, lda};
  std::vector<double> work(2 * (size_t)(n + 2), 0.0);
  for (int i = 0; i < 2 * n; ++i) tau[i] = 0.0;
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  for (int i = ilo; i <= ihi - 1; ++i) {
    double alpha[2] = {A.r(i + 1, i), A.c(i + 1, i)};
    int myn = ihi - i;
    makereflector(myn, alpha, A.at(std::min(i + 2, n), i), tau + 2 * (i - 1));
    A.r(i + 1, i) = 1.0;
    A.c(i + 1, i) = 0.0;
    const double* ti = tau + 2 * (i - 1);
    if (ti[0] != 0.0 || ti[1] != 0.0) {
      int row = ihi, col = ihi - i;
      mvutil1(0, row, col, one, A.sub(1, i + 1), A.at(i + 1, i), zero, work.data());
      double tt[2] = {-ti[0], -ti[1]};
      mvutil2(row, col, tt, work.data(), A.at(i + 1, i), A.sub(1, i + 1));
    }
    if (ti[0] != 0.0 || ti[1] != 0.0) {
      int row = ihi - i, col = n - i;
      mvutil1(1, row, col, one, A.sub(i + 1, i + 1), A.at(i + 1, i), zero, work.data());
      double tt[2] = {-ti[0], ti[1]};
      mvutil2(row, col, tt, A.at(i + 1, i), work.data(), A.sub(i + 1, i + 1));
    }
    A.r(i + 1, i) = alpha[0];
    A.c(i + 1, i) = alpha[1];
  }
}

extern "C" void oq_qgenerator(int n, int ilo, int ihi, double* a, int lda, const double* tau) {
  CM A{a, lda};
  std::vector<double> work(2 * (size_t)(n + 2), 0.0);
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  const int nh = ihi - ilo;
  if (n == 0) return;
  for (int j = ihi; j >= ilo + 1; --j) {
    for (int i = 1; i <= j - 1; ++i) A.r(i, j) = A.c(i, j) = 0.0;
    for (int i = j + 1; i <= ihi; ++i) {
      A.r(i, j) = A.r(i, j - 1);
      A.c(i, j) = A.c(i, j - 1);
    }
    for (int i = ihi + 1; i <= n; ++i) A.r(i, j) = A.c(i, j) = 0.0;
  }
  for (int j = 1; j <= ilo; ++j) {
    for (int i = 1; i <= n; ++i) A.r(i, j) = A.c(i, j) = 0.0;
    A.r(j, j) = 1.0;
  }
  for (int j = ihi + 1; j <= n; ++j) {
    for (int i = 1; i <= n; ++i) A.r(i, j) = A.c(i, j) = 0.0;
    A.r(j, j) = 1.0;
  }
  if (nh > 0) {
    for (int i = ihi; i >= ilo + 1; --i) {
      const double* t = tau + 2 * (i - 2);
      if (i < ihi) {
        A.r(i, i) = 1.0;
        A.c(i, i) = 0.0;
        if (t[0] != 0.0 || t[1] != 0.0) {
          int row = ihi - i + 1, col = ihi - i;
          mvutil1(1, row, col, one, A.sub(i, i + 1), A.at(i, i), zero, work.data());
          double tt[2] = {-t[0], -t[1]};
          mvutil2(row, col, tt, A.at(i, i), work.data(), A.sub(i, i + 1));
        }
        for (int j = i + 1; j <= ihi; ++j) {
          double aRe = -t[0] * A.r(j, i) + t[1] * A.c(j, i);
          A.c(j, i) = -t[0] * A.c(j, i) - t[1] * A.r(j, i);
          A.r(j, i) = aRe;
        }
      }
      A.r(i, i) = 1.0 - t[0];
      A.c(i, i) = 0.0 - t[1];
      for (int j = ilo + 1; j <= i - 1; ++j) A.r(j, i) = A.c(j, i) = 0.0;
    }
  }
}

extern "C" void oq_evalues(int ischur, int n, int ilo, int ihi, double* h, int ldh,
                           double* w, double* z, int ldz) {
  CM H{h, ldh}, Z{z, ldz};
  for (int i = 1; i <= ilo - 1; ++i) {
    w[2 * (i - 1)] = H.r(i, i);
    w[2 * (i - 1) + 1] = H.c(i, i);
  }
  for (int i = ihi + 1; i <= n; ++i) {
    w[2 * (i - 1)] = H.r(i, i);
    w[2 * (i - 1) + 1] = H.c(i, i);
  }
  if (n == 0) return;
  if (ilo == ihi) {
    w[2 * (ilo - 1)] = H.r(ilo, ilo);
    w[2 * (ilo - 1) + 1] = H.c(ilo, ilo);
    return;
  }
  for (int j = ilo; j <= ihi - 2; ++j)
    for (int i = j + 2; i <= n; ++i) H.r(i, j) = H.c(i, j) = 0.0;
  int i1, i2;
  if (ischur == 1) {
    i1 = 1;
    i2 = n;
  } else {
    i1 = ilo;
    i2 = ihi;
  }
  for (int i = ilo + 1; i <= ihi; ++i) {
    double temp[2] = {H.r(i, i - 1), H.c(i, i - 1)};
    if (temp[1] != 0.0) {
      double rtemp = pythag2(temp[0], temp[1]);
      H.r(i, i - 1) = rtemp;
      H.c(i, i - 1) = 0.0;
      temp[0] /= rtemp;
      temp[1] /= rtemp;
      if (i2 > i) {
        for (int j = i + 1; j <= i2; ++j) {
          double hRe = temp[0] * H.r(i, j) + temp[1] * H.c(i, j);
          H.c(i, j) = temp[0] * H.c(i, j) - temp[1] * H.r(i, j);
          H.r(i, j) = hRe;
        }
      }
      for (int j = i1; j <= i - 1; ++j) {
        double hRe = temp[0] * H.r(j, i) - temp[1] * H.c(j, i);
        H.c(j, i) = temp[0] * H.c(j, i) + temp[1] * H.r(j, i);
        H.r(j, i) = hRe;
      }
      if (i < ihi) {
        double hRe = temp[0] * H.r(i + 1, i) - temp[1] * H.c(i + 1, i);
        H.c(i + 1, i) = temp[0] * H.c(i + 1, i) + temp[1] * H.r(i + 1, i);
        H.r(i + 1, i) = hRe;
      }
      if (ischur == 1) {
        for (int j = ilo; j <= ihi; ++j) {
          double hRe = temp[0] * Z.r(j, i) - temp[1] * Z.c(j, i);
          Z.c(j, i) = temp[0] * Z.c(j, i) + temp[1] * Z.r(j, i);
          Z.r(j, i) = hRe;
        }
      }
    }
  }
  // maxb = 900 (evalues :987-991): every in-scope problem takes the QRdouble branch.
  QRdouble(ischur, n, ilo, ihi, H, w, ilo, ihi, Z);
}

extern "C" void oq_orgschur(const int* select, int n, double* t, int ldt, double* q,
                            int ldq, double* w, int* mout) {
  CM T{t, ldt}, Q{q, ldq};
  int m = 0;
  for (int k = 0; k < n; ++k)
    if (select[k]) m += 1;
  if (m != n && m != 0) {
    int ks = 0;
    for (int k = 1; k <= n; ++k) {
      if (select[k - 1]) {
        ks += 1;
        if (k != ks) schurswap(n, T, Q, k, ks);
      }
    }
  }
  for (int k = 1; k <= n; ++k) {
    w[2 * (k - 1)] = T.r(k, k);
    w[2 * (k - 1) + 1] = T.c(k, k);
  }
  *mout = m;
}

namespace oq {
double twonorm_c(const double* x, int n) { return twonorm(x, n); }
}  // namespace oq
