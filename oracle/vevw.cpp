// CPU oracle (test infrastructure): the Wilson loop driver's perturbative vacuum values,
// a literal restatement of vev, Q/disconloops.f90:4653-5339, for one process
// (npx = npy = npz = npt = 1, so itmin = 1 and the coordinates are global).
//
// The loops run in the reference's order: mu = 1..4, ieo = 1..2, ibl = 1..16, the planes
// nu = 2..5-mu with muvec(nu) = 1 + modulo(mu+nu-2, 4) (:4752-4765), then the sites of
// the block in the reference's enumeration (itbit, izbit, iybit, ixbit, :4781-4822),
// which also gives each site's coordinates.  Per site:
//   * the plaquette as the reference multiplies it (:4766-4776): staptemp = U_nu(x)
//     U_mu(x+nu) (setmmf, iflg 1), staple = staptemp U_nu(x+mu)^+ (setmmf, iflg 2),
//     elemloop = U_mu(x) staple^+ (mmd), and its trace's real and imaginary parts;
//     the links are found by their coordinates (periodic), and the enumeration is
//     checked against the pointsource site map (Q/quark.f90:70-105): a mismatch makes
//     the routine return -1;
//   * the phase factors cos/sin(twoPi (x - io) / n) and of 2 (x - io) with the default-
//     kind twoPi literal (:4700), at the site and at the vertices shifted along mu
//     (ipp = 1), along muvec(nu) (ipp = 2) and along both (ipp = 3) (:4823-4945);
//   * the sums tsum, ssum, mtsum, mssum, j4sum, j1t..j3t, j12t..j32t, j12s..j32s with
//     the reference's expressions (:4947-5199), per time slice
//     it = itmin + 2 ((i-1)/itstep) + (ibl-1)/8.
// Then the normalisations with factor = 8 kappa^4, the average plaquette and psi, the
// assembly of Jvev(2, nt, 5, 5) and its sign (:5201-5310).
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle_impl.h"

namespace {

// c = a b for 3x3 complex matrices stored as 18 reals, row-major (re, im) pairs
// (G/gaugetools.f90 mm :741-).
void su3_mm(const double* a, const double* b, double* c) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double re = 0.0, im = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double ar = a[2 * (3 * i + k)], ai = a[2 * (3 * i + k) + 1];
        const double br = b[2 * (3 * k + j)], bi = b[2 * (3 * k + j) + 1];
        re += ar * br - ai * bi;
        im += ar * bi + ai * br;
      }
      c[2 * (3 * i + j)] = re;
      c[2 * (3 * i + j) + 1] = im;
    }
}

// c = a b^+ (G/gaugetools.f90 mmd :908-984).
void su3_mmd(const double* a, const double* b, double* c) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double re = 0.0, im = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double ar = a[2 * (3 * i + k)], ai = a[2 * (3 * i + k) + 1];
        const double br = b[2 * (3 * j + k)], bi = -b[2 * (3 * j + k) + 1];
        re += ar * br - ai * bi;
        im += ar * bi + ai * br;
      }
      c[2 * (3 * i + j)] = re;
      c[2 * (3 * i + j) + 1] = im;
    }
}

// The link U_mu (1-based mu) at 0-based coordinates x, wrapped periodically.
const double* link(const oq_geom* g, const double* u, const int* x0, int mu) {
  int x[4];
  for (int a = 0; a < 4; ++a) x[a] = ((x0[a] % g->n[a]) + g->n[a]) % g->n[a];
  int isite, ieo, ibl, gblclr, ibleo;
  oq_site_of_coords(g, x, &isite, &ieo, &ibl, &gblclr, &ibleo);
  return u + g->ui(1, isite, mu, ieo, ibl);
}

}  // namespace

extern "C" int oq_vevw(const oq_geom* g, const double* u, const int io[3], double kappa, double* Jvev,
                       double* plaq_out, double* psi_out) {
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2], nt = g->n[3];
  const int nvhalf = g->nvhalf;
  const int nxyzt = nx * ny * nz * nt;
  const int itstep = 2 * nvhalf / nt;  // :4680 with npt = 1
  const int itmin = 1;
  const double twoPi = (double)6.283185307179586f;  // :4700, a default-kind literal
  std::vector<double> tsum(nt + 1, 0.0), ssum(nt + 1, 0.0), j1t(nt + 1, 0.0), j2t(nt + 1, 0.0),
      j3t(nt + 1, 0.0);
  // (4, nt) arrays, 1-based: A[imom][it]
  typedef std::vector<std::vector<double>> A4;
  auto mk = [&]() { return A4(5, std::vector<double>(nt + 1, 0.0)); };
  A4 mtsum = mk(), mssum = mk(), j4sum = mk(), j12s = mk(), j13s = mk(), j21s = mk(), j23s = mk(),
     j31s = mk(), j32s = mk(), j12t = mk(), j13t = mk(), j21t = mk(), j23t = mk(), j31t = mk(), j32t = mk();
  std::vector<double> el1(nvhalf + 1), el2(nvhalf + 1);
  // per-site trig: index [ipp] with ipp 0 = the site itself (cosx(i) ...), 1..3 = pcos(ipp)
  struct Tr {
    double cx, cy, cz, c2x, c2y, c2z, sx, sy, sz, s2x, s2y, s2z;
  };
  std::vector<Tr> tr((size_t)4 * (nvhalf + 1));
  auto T = [&](int ipp, int i) -> Tr& { return tr[(size_t)ipp * (nvhalf + 1) + i]; };
  int muvec[5];
  for (int mu = 1; mu <= 4; ++mu) {
    for (int i = 1; i <= 4; ++i) muvec[i] = 1 + (((mu + i - 2) % 4) + 4) % 4;
    for (int ieo = 1; ieo <= 2; ++ieo) {
      for (int ibl = 1; ibl <= 16; ++ibl) {
        for (int nu = 2; nu <= 5 - mu; ++nu) {
          const int mv = muvec[nu];
          // the reference's site enumeration and coordinates (:4781-4822)
          int isite = 0, ieo1 = 2, ieo2 = 1;
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
                  isite += 1;
                  const int it = ibl > 8 ? itbit : itbit - 1;
                  int iblbit = 1 + (ibl - 1) % 8;
                  const int iz = iblbit > 4 ? izbit : izbit - 1;
                  iblbit = 1 + (iblbit - 1) % 4;
                  const int iy = iblbit > 2 ? iybit : iybit - 1;
                  const int ixbit3 = ibl % 2 == 1 ? ixbit - 1 : ixbit;
                  int ix[3];
                  ix[ieo1] = ixbit3 - 2;
                  ix[ieo2] = ixbit3;
                  const int X = ix[ieo];
                  // the site map agrees with the one the links are stored by
                  const int x0[4] = {X - 1, iy - 1, iz - 1, it - 1};
                  {
                    int s2, e2, b2, gc, be2;
                    oq_site_of_coords(g, x0, &s2, &e2, &b2, &gc, &be2);
                    if (s2 != isite || e2 != ieo || b2 != ibl) return -1;
                  }
                  // the plaquette (:4766-4778)
                  int xn[4] = {x0[0], x0[1], x0[2], x0[3]}, xm[4] = {x0[0], x0[1], x0[2], x0[3]};
                  xn[mv - 1] += 1;
                  xm[mu - 1] += 1;
                  double staptemp[18], staple[18], elem[18];
                  su3_mm(link(g, u, x0, mv), link(g, u, xn, mu), staptemp);
                  su3_mmd(staptemp, link(g, u, xm, mv), staple);
                  su3_mmd(link(g, u, x0, mu), staple, elem);
                  el1[isite] = elem[0] + elem[8] + elem[16];
                  el2[isite] = elem[1] + elem[9] + elem[17];
                  // phase factors (:4823-4945)
                  auto cs = [&](double num, double n) { return twoPi * num / n; };
                  Tr& t0 = T(0, isite);
                  t0.cx = std::cos(cs((double)(X - io[0]), nx));
                  t0.sx = std::sin(cs((double)(X - io[0]), nx));
                  t0.c2x = std::cos(cs((double)(2 * (X - io[0])), nx));
                  t0.s2x = std::sin(cs((double)(2 * (X - io[0])), nx));
                  t0.cy = std::cos(cs((double)(iy - io[1]), ny));
                  t0.sy = std::sin(cs((double)(iy - io[1]), ny));
                  t0.c2y = std::cos(cs((double)(2 * (iy - io[1])), ny));
                  t0.s2y = std::sin(cs((double)(2 * (iy - io[1])), ny));
                  t0.cz = std::cos(cs((double)(iz - io[2]), nz));
                  t0.sz = std::sin(cs((double)(iz - io[2]), nz));
                  t0.c2z = std::cos(cs((double)(2 * (iz - io[2])), nz));
                  t0.s2z = std::sin(cs((double)(2 * (iz - io[2])), nz));
                  for (int ipp = 1; ipp <= 3; ++ipp) T(ipp, isite) = t0;
                  // the vertex shifted along direction d goes into ipp = which and 3
                  auto shift = [&](int d, int which) {
                    Tr& p = T(which, isite);
                    if (d == 1) {
                      p.cx = std::cos(cs((double)(1 + X - io[0]), nx));
                      p.sx = std::sin(cs((double)(1 + X - io[0]), nx));
                      p.c2x = std::cos(cs((double)(2 * (1 + X - io[0])), nx));
                      p.s2x = std::sin(cs((double)(2 * (1 + X - io[0])), nx));
                      T(3, isite).cx = p.cx;
                      T(3, isite).sx = p.sx;
                      T(3, isite).c2x = p.c2x;
                      T(3, isite).s2x = p.s2x;
                    } else if (d == 2) {
                      p.cy = std::cos(cs((double)(1 + iy - io[1]), ny));
                      p.sy = std::sin(cs((double)(1 + iy - io[1]), ny));
                      p.c2y = std::cos(cs((double)(2 * (1 + iy - io[1])), ny));
                      p.s2y = std::sin(cs((double)(2 * (1 + iy - io[1])), ny));
                      T(3, isite).cy = p.cy;
                      T(3, isite).sy = p.sy;
                      T(3, isite).c2y = p.c2y;
                      T(3, isite).s2y = p.s2y;
                    } else if (d == 3) {
                      p.cz = std::cos(cs((double)(1 + iz - io[2]), nz));
                      p.sz = std::sin(cs((double)(1 + iz - io[2]), nz));
                      p.c2z = std::cos(cs((double)(2 * (1 + iz - io[2])), nz));
                      p.s2z = std::sin(cs((double)(2 * (1 + iz - io[2])), nz));
                      T(3, isite).cz = p.cz;
                      T(3, isite).sz = p.sz;
                      T(3, isite).c2z = p.c2z;
                      T(3, isite).s2z = p.s2z;
                    }
                  };
                  shift(mu, 1);
                  shift(mv, 2);
                }
              }
            }
          }
          // the sums (:4947-5199), site by site in the block's order
          for (int i = 1; i <= nvhalf; ++i) {
            const int it = itmin + 2 * ((i - 1) / itstep) + (ibl - 1) / 8;
            const double e1 = el1[i], e2 = el2[i];
            const Tr& c = T(0, i);
            const Tr& p1 = T(1, i);
            const Tr& p2 = T(2, i);
            const Tr& p3 = T(3, i);
            if (mv == 4 || mu == 4)
              tsum[it] += e1;
            else
              ssum[it] += e1;
            {
              const double fac1 = (c.cx + c.cy + c.cz + p1.cx + p1.cy + p1.cz + p2.cx + p2.cy + p2.cz + p3.cx +
                                   p3.cy + p3.cz) /
                                  3.0;
              const double fac2 = (c.cx * c.cy + c.cx * c.cz + c.cy * c.cz + p1.cx * p1.cy + p1.cx * p1.cz +
                                   p1.cy * p1.cz + p2.cx * p2.cy + p2.cx * p2.cz + p2.cy * p2.cz + p3.cx * p3.cy +
                                   p3.cx * p3.cz + p3.cy * p3.cz) /
                                  3.0;
              const double fac3 =
                  c.cx * c.cy * c.cz + p1.cx * p1.cy * p1.cz + p2.cx * p2.cy * p2.cz + p3.cx * p3.cy * p3.cz;
              const double fac4 = (c.c2x + c.c2y + c.c2z + p1.c2x + p1.c2y + p1.c2z + p2.c2x + p2.c2y + p2.c2z +
                                   p3.c2x + p3.c2y + p3.c2z) /
                                  3.0;
              A4& m = mv == 4 ? mtsum : mssum;
              m[1][it] += fac1 * e1;
              m[2][it] += fac2 * e1;
              m[3][it] += fac3 * e1;
              m[4][it] += fac4 * e1;
            }
            if (mv == 4) {  // J_4 (:5005-5029)
              const double fac1 = (c.cx + c.cy + c.cz - p1.cx - p1.cy - p1.cz) / 3.0;
              const double fac2 =
                  (c.cx * c.cy + c.cx * c.cz + c.cy * c.cz - p1.cx * p1.cy - p1.cx * p1.cz - p1.cy * p1.cz) / 3.0;
              const double fac3 = c.cx * c.cy * c.cz - p1.cx * p1.cy * p1.cz;
              const double fac4 = (c.c2x + c.c2y + c.c2z - p1.c2x - p1.c2y - p1.c2z) / 3.0;
              j4sum[1][it] -= fac1 * e2;
              j4sum[2][it] -= fac2 * e2;
              j4sum[3][it] -= fac3 * e2;
              j4sum[4][it] -= fac4 * e2;
            }
            // sine weights: (s, s (c_b + c_c)/2, s c_b c_c, s2) of one axis at one vertex
            auto add = [&](A4& J, double f1, double f2, double f3, double f4, double w) {
              J[1][it] += f1 * w;
              J[2][it] += f2 * w;
              J[3][it] += f3 * w;
              J[4][it] += f4 * w;
            };
            auto sub = [&](A4& J, double f1, double f2, double f3, double f4, double w) {
              J[1][it] -= f1 * w;
              J[2][it] -= f2 * w;
              J[3][it] -= f3 * w;
              J[4][it] -= f4 * w;
            };
            if (mu == 1 && mv == 4) {  // :5030-5053
              j1t[it] += e2;
              add(j13t, c.sz, c.sz * (c.cx + c.cy) / 2.0, c.sz * c.cx * c.cy, c.s2z, e2);
              add(j12t, c.sy, c.sy * (c.cx + c.cz) / 2.0, c.sy * c.cx * c.cz, c.s2y, e2);
            }
            if (mu == 2 && mv == 4) {  // :5054-5077
              j2t[it] += e2;
              add(j21t, c.sx, c.sx * (c.cy + c.cz) / 2.0, c.sx * c.cy * c.cz, c.s2x, e2);
              add(j23t, c.sz, c.sz * (c.cx + c.cy) / 2.0, c.sz * c.cx * c.cy, c.s2z, e2);
            }
            if (mu == 3 && mv == 4) {  // :5078-5101
              j3t[it] += e2;
              add(j32t, c.sy, c.sy * (c.cx + c.cz) / 2.0, c.sy * c.cx * c.cz, c.s2y, e2);
              add(j31t, c.sx, c.sx * (c.cy + c.cz) / 2.0, c.sx * c.cy * c.cz, c.s2x, e2);
            }
            if (mu == 1 && mv != 4) {  // :5102-5126
              add(j13s, c.sz - p2.sz, c.sz * (c.cx + c.cy) / 2.0 - p2.sz * (p2.cx + p2.cy) / 2.0,
                  c.sz * c.cx * c.cy - p2.sz * p2.cx * p2.cy, c.s2z - p2.s2z, e2);
              add(j12s, c.sy - p2.sy, c.sy * (c.cx + c.cz) / 2.0 - p2.sy * (p2.cx + p2.cz) / 2.0,
                  c.sy * c.cx * c.cz - p2.sy * p2.cx * p2.cz, c.s2y - p2.s2y, e2);
            }
            if (mu == 2 && mv == 3) {  // :5127-5148
              add(j21s, c.sx - p2.sx, c.sx * (c.cy + c.cz) / 2.0 - p2.sx * (p2.cy + p2.cz) / 2.0,
                  c.sx * c.cy * c.cz - p2.sx * p2.cy * p2.cz, c.s2x - p2.s2x, e2);
              add(j23s, c.sz - p2.sz, c.sz * (c.cx + c.cy) / 2.0 - p2.sz * (p2.cx + p2.cy) / 2.0,
                  c.sz * c.cx * c.cy - p2.sz * p2.cx * p2.cy, c.s2z - p2.s2z, e2);
            } else if (mu == 1 && mv == 2) {  // :5149-5173
              sub(j21s, c.sx - p1.sx, c.sx * (c.cy + c.cz) / 2.0 - p1.sx * (p1.cy + p1.cz) / 2.0,
                  c.sx * c.cy * c.cz - p1.sx * p1.cy * p1.cz, c.s2x - p1.s2x, e2);
              sub(j23s, c.sz - p1.sz, c.sz * (c.cx + c.cy) / 2.0 - p1.sz * (p1.cx + p1.cy) / 2.0,
                  c.sz * c.cx * c.cy - p1.sz * p1.cx * p1.cy, c.s2z - p1.s2z, e2);
            }
            if (mv == 3) {  // :5174-5197
              sub(j32s, c.sy - p1.sy, c.sy * (c.cx + c.cz) / 2.0 - p1.sy * (p1.cx + p1.cz) / 2.0,
                  c.sy * c.cx * c.cz - p1.sy * p1.cx * p1.cz, c.s2y - p1.s2y, e2);
              sub(j31s, c.sx - p1.sx, c.sx * (c.cy + c.cz) / 2.0 - p1.sx * (p1.cy + p1.cz) / 2.0,
                  c.sx * c.cy * c.cz - p1.sx * p1.cy * p1.cz, c.s2x - p1.s2x, e2);
            }
          }
        }
      }
    }
  }
  // normalisations (:5201-5240)
  const double factor = 8.0 * kappa * kappa * kappa * kappa;
  double plaq = 0.0;
  for (int it = 1; it <= nt; ++it) plaq = plaq + tsum[it] + ssum[it];
  plaq = plaq / (double)(18 * nxyzt);
  for (int it = 1; it <= nt; ++it) {
    tsum[it] *= 4.0 * factor;
    ssum[it] *= 8.0 * factor;
    j1t[it] *= 2.0 * factor;
    j2t[it] *= 2.0 * factor;
    j3t[it] *= 2.0 * factor;
    for (int im = 1; im <= 4; ++im) {
      mtsum[im][it] *= factor;
      mssum[im][it] *= 2.0 * factor;
      for (A4* J : {&j4sum, &j12s, &j13s, &j21s, &j23s, &j31s, &j32s, &j12t, &j13t, &j21t, &j23t, &j31t, &j32t})
        (*J)[im][it] *= 2.0 * factor;
    }
  }
  double psi = ssum[1] + tsum[1];
  for (int it = 2; it <= nt; ++it) psi = psi + ssum[it] + tsum[it] + tsum[it - 1];
  psi = psi / (double)nxyzt;
  // Jvev(2, nt, 5, 5), Fortran order (:5259-5310)
  auto J = [&](int ri, int it, int im, int op) -> double& {
    return Jvev[(size_t)(ri - 1) + 2 * ((size_t)(it - 1) + (size_t)nt * ((im - 1) + 5 * (size_t)(op - 1)))];
  };
  std::memset(Jvev, 0, sizeof(double) * 2 * nt * 25);
  J(1, 1, 1, 5) = ssum[1] + tsum[1];
  for (int it = 2; it <= nt; ++it) J(1, it, 1, 5) = ssum[it] + tsum[it] + tsum[it - 1];
  for (int im = 1; im <= 4; ++im) {
    J(1, 1, im + 1, 5) = mssum[im][1] + mtsum[im][1];
    for (int it = 2; it <= nt; ++it) J(1, it, im + 1, 5) = mssum[im][it] + mtsum[im][it] + mtsum[im][it - 1];
  }
  for (int im = 1; im <= 4; ++im)
    for (int it = 1; it <= nt; ++it) J(2, it, im + 1, 4) = j4sum[im][it];
  J(2, 1, 1, 1) = j1t[1];
  J(2, 1, 1, 2) = j2t[1];
  J(2, 1, 1, 3) = j3t[1];
  for (int it = 2; it <= nt; ++it) {
    J(2, it, 1, 1) = j1t[it] - j1t[it - 1];
    J(2, it, 1, 2) = j2t[it] - j2t[it - 1];
    J(2, it, 1, 3) = j3t[it] - j3t[it - 1];
  }
  for (int im = 1; im <= 4; ++im) {
    J(1, 1, im + 1, 1) = j13s[im][1] + j13t[im][1];
    J(2, 1, im + 1, 1) = j21s[im][1] + j21t[im][1];
    J(1, 1, im + 1, 2) = j32s[im][1] + j32t[im][1];
    J(2, 1, im + 1, 2) = j12s[im][1] + j12t[im][1];
    J(1, 1, im + 1, 3) = j23s[im][1] + j23t[im][1];
    J(2, 1, im + 1, 3) = j31s[im][1] + j31t[im][1];
    for (int it = 2; it <= nt; ++it) {
      J(1, it, im + 1, 1) = j13s[im][it] - j13t[im][it - 1] + j13t[im][it];
      J(2, it, im + 1, 1) = j21s[im][it] - j21t[im][it - 1] + j21t[im][it];
      J(1, it, im + 1, 2) = j32s[im][it] - j32t[im][it - 1] + j32t[im][it];
      J(2, it, im + 1, 2) = j12s[im][it] - j12t[im][it - 1] + j12t[im][it];
      J(1, it, im + 1, 3) = j23s[im][it] - j23t[im][it - 1] + j23t[im][it];
      J(2, it, im + 1, 3) = j31s[im][it] - j31t[im][it - 1] + j31t[im][it];
    }
  }
  for (int k = 0; k < 2 * nt * 25; ++k) Jvev[k] = -Jvev[k];  // :5312
  if (plaq_out) *plaq_out = plaq;
  if (psi_out) *psi_out = psi;
  return 0;
}
