// CPU oracle (test infrastructure): the reference's pseudo-heatbath for the Wilson
// plaquette action, restating
//   * sweep, C/cfgsprops.f90:1973-2001: for ieo = 1,2, ibl = 1..16, mu = 1..4, the
//     staples of the links u(:, 1..nvhalf, mu, ieo, ibl), then phbup on them;
//   * staple, G/gaugetools.f90:39-345, nearest-neighbour (gaction = 1) part:
//     c = sum_{nu /= mu} coact(1,mu,nu) [U_nu(x) U_mu(x+nu) U_nu(x+mu)^+
//                                        + U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu)],
//     coact(1,mu,nu) = beta on an isotropic lattice without tadpole factors
//     (G/lattice.f90:396-422), links periodic;
//   * phbup, G/heatbath.f90:33-76: the three SU(2) subgroups (rows 1,2 / 2,3 / 1,3) in
//     turn, each projected from u c^+ (phbsub1..3, :80-235), updated by su2up and
//     multiplied into u (sprd1, :327-467);
//   * su2up, :239-323: Kennedy-Pendleton with the lagged-Fibonacci stream rnds in the
//     reference's order (4 numbers per link still to update per round, rounds until all
//     links accept, then 2 per link for the hypersphere).  As in the reference: twoPi is
//     a default-kind (single precision) constant, and the accepted flags id() are not
//     reset between hits, so nhit > 1 adds nothing after the first.
// The site order of a sublattice is isite = 1..nvhalf of the reference layout.  The
// 3x3 products of the staples and the subgroup projections are written here in complex
// form; the reference's hand-expanded real arithmetic may round differently, which after
// many sweeps gives a different (equally distributed) configuration: the oracle's
// plaquette is reproducible for this restatement, not the reference's own number.
#include <cmath>
#include <complex>
#include <vector>

#include "oracle_impl.h"

namespace {

using C = std::complex<double>;
struct M3 {
  C e[3][3];
};

M3 mul(const M3& a, const M3& b) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      C s = 0.0;
      for (int k = 0; k < 3; ++k) s += a.e[i][k] * b.e[k][j];
      r.e[i][j] = s;
    }
  return r;
}
M3 dag(const M3& a) {
  M3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.e[i][j] = std::conj(a.e[j][i]);
  return r;
}

struct HbLattice {
  const oq_geom* g;
  int n[4];
  std::vector<int> isite, ieo, ibl;  // per lexicographic site
  std::vector<int> lex;              // [(ibl-1)*2 + (ieo-1)][isite-1] -> lexicographic site
  explicit HbLattice(const oq_geom* geo) : g(geo) {
    for (int d = 0; d < 4; ++d) n[d] = g->n[d];
    const int V = n[0] * n[1] * n[2] * n[3];
    isite.resize(V);
    ieo.resize(V);
    ibl.resize(V);
    lex.assign((size_t)32 * g->nvhalf, -1);
    for (int t = 0; t < n[3]; ++t)
      for (int z = 0; z < n[2]; ++z)
        for (int y = 0; y < n[1]; ++y)
          for (int x = 0; x < n[0]; ++x) {
            const int xc[4] = {x, y, z, t};
            int is, ie, ib, gblclr, ibleo;
            oq_site_of_coords(g, xc, &is, &ie, &ib, &gblclr, &ibleo);
            const int L = x + n[0] * (y + n[1] * (z + n[2] * t));
            isite[L] = is;
            ieo[L] = ie;
            ibl[L] = ib;
            lex[((size_t)(ib - 1) * 2 + (ie - 1)) * g->nvhalf + (is - 1)] = L;
          }
  }
  int shift(int L, int mu, int s) const {
    int c[4] = {L % n[0], (L / n[0]) % n[1], (L / (n[0] * n[1])) % n[2], L / (n[0] * n[1] * n[2])};
    c[mu] = (c[mu] + s + n[mu]) % n[mu];
    return c[0] + n[0] * (c[1] + n[1] * (c[2] + n[2] * c[3]));
  }
  M3 link(const double* u, int L, int mu) const {
    M3 m;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        m.e[a][b] = C(u[g->ui(2 * (3 * a + b) + 1, isite[L], mu + 1, ieo[L], ibl[L])],
                      u[g->ui(2 * (3 * a + b) + 2, isite[L], mu + 1, ieo[L], ibl[L])]);
    return m;
  }
  void set(double* u, int L, int mu, const M3& m) const {
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        u[g->ui(2 * (3 * a + b) + 1, isite[L], mu + 1, ieo[L], ibl[L])] = m.e[a][b].real();
        u[g->ui(2 * (3 * a + b) + 2, isite[L], mu + 1, ieo[L], ibl[L])] = m.e[a][b].imag();
      }
  }
};

// staple (nearest-neighbour part), G/gaugetools.f90:39-345
M3 staple(const HbLattice& H, const double* u, int L, int mu, double beta) {
  M3 c{};
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == mu) continue;
    const int xn = H.shift(L, nu, 1), xm = H.shift(L, mu, 1), xmn = H.shift(L, nu, -1),
              xmnm = H.shift(xmn, mu, 1);
    const M3 w = mul(mul(H.link(u, L, nu), H.link(u, xn, mu)), dag(H.link(u, xm, nu)));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) c.e[a][b] += beta * w.e[a][b];
    const M3 t = mul(mul(dag(H.link(u, xmn, nu)), H.link(u, xmn, mu)), H.link(u, xmnm, nu));
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) c.e[a][b] += beta * t.e[a][b];
  }
  return c;
}

// su2up, G/heatbath.f90:239-323
void su2up(std::vector<double>& z, int nvhalf, int nhit) {
  const double twoPi = (double)6.283185307179586f;
  std::vector<double> a0(nvhalf, 0.0), dk(nvhalf), id(nvhalf, 0.0), rn(4 * (size_t)nvhalf);
  for (int i = 0; i < nvhalf; ++i)
    dk[i] = 1.0 / std::sqrt(z[4 * i] * z[4 * i] + z[4 * i + 1] * z[4 * i + 1] + z[4 * i + 2] * z[4 * i + 2] +
                            z[4 * i + 3] * z[4 * i + 3]);
  for (int ihit = 1; ihit <= nhit; ++ihit) {
    for (;;) {
      int inotup = nvhalf;
      for (int i = 0; i < nvhalf; ++i) inotup = inotup - (int)id[i];
      if (inotup == 0) break;
      oq_rnds(4 * inotup, rn.data());
      int j = -3;  // 1-based index into rn
      for (int i = 0; i < nvhalf; ++i) {
        if (id[i] != 1.0) {
          j += 4;
          const double tt = std::cos(twoPi * rn[j + 1]);
          const double d2 = -(std::log(rn[j - 1]) + std::log(rn[j]) * tt * tt) * dk[i] * 3.0;
          if (rn[j + 2] * rn[j + 2] <= (1.0 - 0.5 * d2)) {
            id[i] = 1.0;
            a0[i] = 1.0 - d2;
          }
        }
      }
    }
  }
  oq_rnds(2 * nvhalf, rn.data());
  for (int i = 0; i < nvhalf; ++i) {
    const int j = 2 * i;  // 0-based rn(i + i - 1)
    const double rad = 1.0 - a0[i] * a0[i];
    const double a3 = std::sqrt(rad) * (2.0 * rn[j] - 1.0);
    const double rad2 = std::sqrt(std::fabs(rad - a3 * a3));
    const double theta = twoPi * rn[j + 1];
    const double a1 = rad2 * std::cos(theta), a2 = rad2 * std::sin(theta);
    double* zi = &z[4 * (size_t)i];
    const double z1 = zi[0], z2 = zi[1], z3 = zi[2], z4 = zi[3];
    zi[0] = dk[i] * (a0[i] * z1 + a1 * z2 + a2 * z3 + a3 * z4);
    zi[1] = dk[i] * (-a0[i] * z2 + a1 * z1 + a2 * z4 - a3 * z3);
    zi[2] = dk[i] * (-a0[i] * z3 - a1 * z4 + a2 * z1 + a3 * z2);
    zi[3] = dk[i] * (-a0[i] * z4 + a1 * z3 - a2 * z2 + a3 * z1);
  }
}

}  // namespace

// phbup for subgroups (p, q) = (0,1), (1,2), (0,2) with w = u c^+ (phbsub1..3):
//   z1 = Re(w_pp + w_qq), z2 = Im(w_pq + w_qp), z3 = s (Re w_pq - Re w_qp),
//   z4 = Im w_pp - Im w_qq, s = -1 for rows 2,3 and +1 otherwise;
// then rows (p, q) of u <- [[z1 + i z4, s z3 + i z2], [-s z3 + i z2, z1 - i z4]] rows (p, q)
// (sprd1).  Sweeps as the reference's sweep; u is the reference layout, in place.
extern "C" void oq_heatbath(const oq_geom* g, double* u, double beta, int nsweeps, int nhit, double* plaq) {
  const HbLattice H(g);
  const int nv = g->nvhalf;
  std::vector<M3> c(nv), lk(nv);
  std::vector<double> z(4 * (size_t)nv);
  const int P[3] = {0, 1, 0}, Q[3] = {1, 2, 2};
  const double S[3] = {1.0, -1.0, 1.0};
  for (int sw = 0; sw < nsweeps; ++sw) {
    for (int ieo = 1; ieo <= 2; ++ieo)
      for (int ibl = 1; ibl <= 16; ++ibl)
        for (int mu = 0; mu < 4; ++mu) {
          const int* Ls = &H.lex[((size_t)(ibl - 1) * 2 + (ieo - 1)) * nv];
          for (int i = 0; i < nv; ++i) c[i] = staple(H, u, Ls[i], mu, beta);
          for (int i = 0; i < nv; ++i) lk[i] = H.link(u, Ls[i], mu);
          for (int s = 0; s < 3; ++s) {
            const int p = P[s], q = Q[s];
            for (int i = 0; i < nv; ++i) {
              const M3 w = mul(lk[i], dag(c[i]));
              z[4 * i] = w.e[p][p].real() + w.e[q][q].real();
              z[4 * i + 1] = w.e[p][q].imag() + w.e[q][p].imag();
              z[4 * i + 2] = S[s] * (w.e[p][q].real() - w.e[q][p].real());
              z[4 * i + 3] = w.e[p][p].imag() - w.e[q][q].imag();
            }
            su2up(z, nv, nhit);
            for (int i = 0; i < nv; ++i) {
              const double* zi = &z[4 * (size_t)i];
              const C v00(zi[0], zi[3]), v01(S[s] * zi[2], zi[1]), v10(-S[s] * zi[2], zi[1]), v11(zi[0], -zi[3]);
              for (int b = 0; b < 3; ++b) {
                const C up = lk[i].e[p][b], uq = lk[i].e[q][b];
                lk[i].e[p][b] = v00 * up + v01 * uq;
                lk[i].e[q][b] = v10 * up + v11 * uq;
              }
            }
          }
          for (int i = 0; i < nv; ++i) H.set(u, Ls[i], mu, lk[i]);
        }
    if (plaq) plaq[sw] = oq_aveplaq(g, u);
  }
}
