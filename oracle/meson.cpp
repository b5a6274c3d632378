// CPU oracle (test infrastructure): sink smearing and the correlators of mesoncorr.
//   * smear, Q/diracops.f90:712-858: nsmear sweeps of
//       h <- (1 - 6 a) h + a sum_{mu=1..3} [ U_mu(x) h(x+mu) + U_mu(x-mu)^+ h(x-mu) ]
//     with bc(mu) on hops across the lattice edge, both halves from the previous sweep
//     (the reference's setmvf / mdv / slidevector block machinery evaluates this sum; it is
//     written here per lexicographic site);
//   * mesoncorr, Q/quark.f90:1297-2137, the correlator loop :1806-1961: the reference's
//     site loop (itbit, izbit, iybit, ixbit, ibl, ieo with ix(ieo1) = ixbit3 - 2,
//     ix(ieo2) = ixbit3), per (id, jd, ii) the colour sum of q(jc, jd; ic, jd2(iop, id))
//     conj(qbar(jc, jd2(jop, jd); ic, id)), the sign and rootm1 rule, and the momentum sum
//     with the cos / sin products of :1925-1955 (lessnoise = 0, as lessnoiseoverride = 1
//     forces).  The propagator value at a loop site is read from the reference-layout
//     column through the site map (the reference reads the same values from its FPwrite
//     files in that loop order).  channels = 0: only the pairs the reference evaluates
//     (jop, iop <= 2 without S->S); channels = 1: all 28.
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "oracle_impl.h"

namespace {

using C = std::complex<double>;

const int kRootm1[16] = {-1, 1, -1, 1, -1, -1, 1, -1, 1, 1, 1, -1, 1, -1, 1, -1};
const int kJd2[16][4] = {{3, 4, 1, 2}, {1, 2, 3, 4}, {2, 1, 4, 3}, {2, 1, 4, 3}, {1, 2, 3, 4}, {3, 4, 1, 2},
                         {4, 3, 2, 1}, {4, 3, 2, 1}, {3, 4, 1, 2}, {1, 2, 3, 4}, {3, 4, 1, 2}, {4, 3, 2, 1},
                         {4, 3, 2, 1}, {2, 1, 4, 3}, {2, 1, 4, 3}, {1, 2, 3, 4}};
const double kSgni[16][4] = {{-1, -1, 1, 1}, {1, 1, 1, 1},   {-1, -1, 1, 1}, {1, -1, -1, 1},
                             {-1, 1, 1, -1}, {1, 1, 1, 1},   {-1, -1, -1, -1}, {1, -1, 1, -1},
                             {-1, 1, -1, 1}, {-1, -1, 1, 1}, {1, -1, -1, 1}, {-1, 1, 1, -1},
                             {1, 1, -1, -1}, {1, 1, 1, 1},   {-1, 1, -1, 1}, {1, -1, 1, -1}};
const double kSgnj[16][4] = {{1, 1, -1, -1}, {1, 1, 1, 1},   {1, 1, -1, -1}, {-1, 1, 1, -1},
                             {1, -1, -1, 1}, {1, 1, 1, 1},   {1, 1, 1, 1},   {-1, 1, -1, 1},
                             {1, -1, 1, -1}, {-1, -1, 1, 1}, {-1, 1, 1, -1}, {1, -1, -1, 1},
                             {-1, -1, 1, 1}, {1, 1, 1, 1},   {-1, 1, -1, 1}, {1, -1, 1, -1}};
// jop, iop of ii = 1..28 with corrsp = .true. (:1575-1634)
const int kJop[28] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 6, 2, 3, 4, 5, 7, 8, 9};
const int kIop[28] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 2, 6, 7, 8, 9, 10, 3, 4, 5, 6, 2, 1, 14, 15, 16, 14, 15, 16};

}  // namespace

extern "C" void oq_smear(const oq_geom* g, const double* u, double* he, double* ho, const double* ge,
                         const double* go, double asmear, int nsmear) {
  const size_t vs = g->vsize();
  const int n[4] = {g->n[0], g->n[1], g->n[2], g->n[3]};
  const int V = n[0] * n[1] * n[2] * n[3];
  std::vector<double> a(2 * vs, 0.0), b(2 * vs, 0.0);
  std::memcpy(a.data(), ge, sizeof(double) * vs);
  std::memcpy(a.data() + vs, go, sizeof(double) * vs);
  auto site = [&](const int x[4], int* isite, int* ieo, int* ibl, int* gbl, int* ibleo) {
    oq_site_of_coords(g, x, isite, ieo, ibl, gbl, ibleo);
  };
  const double bs = 1.0 - 6.0 * asmear;
  for (int it = 0; it < nsmear; ++it) {
    for (int L = 0; L < V; ++L) {
      const int x[4] = {L % n[0], (L / n[0]) % n[1], (L / (n[0] * n[1])) % n[2], L / (n[0] * n[1] * n[2])};
      int isite, ieo, ibl, gbl, ibleo;
      site(x, &isite, &ieo, &ibl, &gbl, &ibleo);
      C acc[4][3] = {};
      for (int mu = 0; mu < 3; ++mu)
        for (int dir = 0; dir < 2; ++dir) {
          int y[4] = {x[0], x[1], x[2], x[3]};
          double f = 1.0;
          y[mu] += dir == 0 ? 1 : -1;
          if (y[mu] < 0 || y[mu] >= n[mu]) {
            f = g->bc[mu];
            y[mu] = (y[mu] + n[mu]) % n[mu];
          }
          int js, je, jb, jg, jbe;
          site(y, &js, &je, &jb, &jg, &jbe);
          // the link U_mu at x (forward) or at y = x - mu (backward)
          const int ls = dir == 0 ? isite : js, le = dir == 0 ? ieo : je, lb = dir == 0 ? ibl : jb;
          C U[3][3];
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
              U[r][c] = C(u[g->ui(2 * (3 * r + c) + 1, ls, mu + 1, le, lb)], u[g->ui(2 * (3 * r + c) + 2, ls, mu + 1, le, lb)]);
          const double* h = a.data() + (jg == 1 ? 0 : vs);
          for (int d = 0; d < 4; ++d) {
            C v[3];
            for (int c = 0; c < 3; ++c)
              v[c] = f * C(h[g->gi(2 * c + 1, js, d + 1, je, jbe)], h[g->gi(2 * c + 2, js, d + 1, je, jbe)]);
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) acc[d][r] += dir == 0 ? U[r][c] * v[c] : std::conj(U[c][r]) * v[c];
          }
        }
      const double* h = a.data() + (gbl == 1 ? 0 : vs);
      double* o = b.data() + (gbl == 1 ? 0 : vs);
      for (int d = 0; d < 4; ++d)
        for (int c = 0; c < 3; ++c) {
          const size_t k = g->gi(2 * c + 1, isite, d + 1, ieo, ibleo);
          o[k] = bs * h[k] + asmear * acc[d][c].real();
          o[k + 1] = bs * h[k + 1] + asmear * acc[d][c].imag();
        }
    }
    std::swap(a, b);
  }
  std::memcpy(he, a.data(), sizeof(double) * vs);
  std::memcpy(ho, a.data() + vs, sizeof(double) * vs);
}

// corrRe, corrIm(nt, -4:4, -4:4, -4:4, 28)
extern "C" void oq_mesoncorr(const oq_geom* g, const double* q, const double* qbar, const int src[4], int channels,
                             double* corrRe, double* corrIm) {
  const size_t vs = g->vsize();
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2], nt = g->n[3];
  const double twoPi = 6.283185307179586;
  const size_t ncorr = (size_t)nt * 729 * 28;
  std::memset(corrRe, 0, sizeof(double) * ncorr);
  std::memset(corrIm, 0, sizeof(double) * ncorr);
  if (!qbar) qbar = q;
  auto CR = [&](int it, int px, int py, int pz, int ii) -> size_t {
    return (size_t)(it - 1) + (size_t)nt * ((px + 4) + 9 * ((py + 4) + 9 * ((pz + 4) + 9 * (size_t)(ii - 1))));
  };
  // the propagator component (source jc, jd; sink ic, id) at global site (ix, iy, iz, it)
  auto prop = [&](const double* col0, int jc, int jd, int ic, int id, const int x1[4]) {
    const int x[4] = {x1[0] - 1, x1[1] - 1, x1[2] - 1, x1[3] - 1};
    int isite, ieo, ibl, gbl, ibleo;
    oq_site_of_coords(g, x, &isite, &ieo, &ibl, &gbl, &ibleo);
    const double* col = col0 + ((size_t)((jc - 1) * 4 + (jd - 1)) * 2 + (gbl - 1)) * vs;
    const size_t k = g->gi(2 * ic - 1, isite, id, ieo, ibleo);
    return C(col[k], col[k + 1]);
  };
  int ieo1 = 2, ieo2 = 1, ix[3];
  double mycos[3][9], mysin[3][9];
  for (int itbit = 2; itbit <= nt; itbit += 2) {
    ieo1 = 3 - ieo1;
    ieo2 = 3 - ieo2;
    for (int izbit = 2; izbit <= nz; izbit += 2) {
      ieo1 = 3 - ieo1;
      ieo2 = 3 - ieo2;
      for (int iybit = 2; iybit <= ny; iybit += 2) {
        ieo1 = 3 - ieo1;
        ieo2 = 3 - ieo2;
        for (int ixbit = 4; ixbit <= nx; ixbit += 4) {
          for (int ibl = 1; ibl <= 16; ++ibl) {
            const int it = ibl > 8 ? itbit : itbit - 1;
            int iblbit = 1 + (ibl - 1) % 8;
            const int iz = iblbit > 4 ? izbit : izbit - 1;
            iblbit = 1 + (iblbit - 1) % 4;
            const int iy = iblbit > 2 ? iybit : iybit - 1;
            const int ixbit3 = ibl % 2 == 1 ? ixbit - 1 : ixbit;
            ix[ieo1] = ixbit3 - 2;
            ix[ieo2] = ixbit3;
            for (int ieo = 1; ieo <= 2; ++ieo) {
              const int x1[4] = {ix[ieo], iy, iz, it};
              for (int m = -4; m <= 4; ++m) {
                mycos[0][m + 4] = std::cos(twoPi * (double)(m * (ix[ieo] - src[0])) / (double)nx);
                mysin[0][m + 4] = std::sin(twoPi * (double)(m * (ix[ieo] - src[0])) / (double)nx);
                mycos[1][m + 4] = std::cos(twoPi * (double)(m * (iy - src[1])) / (double)ny);
                mysin[1][m + 4] = std::sin(twoPi * (double)(m * (iy - src[1])) / (double)ny);
                mycos[2][m + 4] = std::cos(twoPi * (double)(m * (iz - src[2])) / (double)nz);
                mysin[2][m + 4] = std::sin(twoPi * (double)(m * (iz - src[2])) / (double)nz);
              }
              for (int id = 1; id <= 4; ++id)
                for (int jd = 1; jd <= 4; ++jd)
                  for (int ii = 1; ii <= 28; ++ii) {
                    const int jop = kJop[ii - 1], iop = kIop[ii - 1];
                    if (channels == 0 && !(jop <= 2 && iop <= 2 && (jop != 1 || iop != 1))) continue;
                    double bitRe = 0.0, bitIm = 0.0;
                    for (int ic = 1; ic <= 3; ++ic)
                      for (int jc = 1; jc <= 3; ++jc) {
                        const C a = prop(q, jc, jd, ic, kJd2[iop - 1][id - 1], x1);
                        const C b = prop(qbar, jc, kJd2[jop - 1][jd - 1], ic, id, x1);
                        bitRe += a.real() * b.real() + a.imag() * b.imag();
                        bitIm += a.imag() * b.real() - a.real() * b.imag();
                      }
                    const double s = kSgnj[jop - 1][jd - 1] * kSgni[iop - 1][id - 1];
                    if (kRootm1[jop - 1] == 1 && kRootm1[iop - 1] == 1) {
                      bitRe = bitRe * s;
                      bitIm = bitIm * s;
                    } else if (kRootm1[jop - 1] == -1 && kRootm1[iop - 1] == -1) {
                      bitRe = -bitRe * s;
                      bitIm = -bitIm * s;
                    } else {
                      const double t = bitIm * s;
                      bitIm = bitRe * s;
                      bitRe = t;
                    }
                    for (int pz = 0; pz < 9; ++pz)
                      for (int py = 0; py < 9; ++py)
                        for (int px = 0; px < 9; ++px) {
                          const double c1 = mycos[0][px], c2 = mycos[1][py], c3 = mycos[2][pz];
                          const double s1 = mysin[0][px], s2 = mysin[1][py], s3 = mysin[2][pz];
                          const size_t o = CR(it, px - 4, py - 4, pz - 4, ii);
                          corrRe[o] = corrRe[o] + bitRe * c1 * c2 * c3;
                          corrIm[o] = corrIm[o] + bitIm * c1 * c2 * c3;
                          corrRe[o] = corrRe[o] - bitIm * (c1 * c2 * s3 + c1 * s2 * c3 + s1 * c2 * c3) -
                                      bitRe * (s1 * s2 * c3 + s1 * c2 * s3 + c1 * s2 * s3) + bitIm * s1 * s2 * s3;
                          corrIm[o] = corrIm[o] + bitRe * (c1 * c2 * s3 + c1 * s2 * c3 + s1 * c2 * c3) -
                                      bitIm * (s1 * s2 * c3 + s1 * c2 * s3 + c1 * s2 * s3) - bitRe * s1 * s2 * s3;
                        }
                  }
            }
          }
        }
      }
    }
  }
}
