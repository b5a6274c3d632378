// CPU oracle (test infrastructure): perturbative vacuum expectation values of the loop
// operators, a literal restatement of twvev, Q/vevbleft.f90:757-2536.
//
// For every lattice site x (lexicographic, t outermost) and every unit vector
// z2 = e(x, icolor, idirac) (:1110-1130), the hopping expansion of the twisted-mass
// propagator is built order by order in the arrays sb1..sb6 (:1168-1450):
//   * GammaMultiply (GammaMultiplyP / GammaMultiplyM, :8163-8873) rotates the previous
//     order at one site by the twist angle and hops it to the 8 neighbours with the
//     Wilson projectors (r -/+ gamma_mu), periodic in space and, with dobndry = 0,
//     periodic in time without a boundary sign; dobndry = 1 blocks the time hops across
//     the last slice (:8269-8301);
//   * order n is seeded from the sites of the diamond shells the reference enumerates
//     (bx, by, bz, +-bt with |b|_1 = md, :1172-1430), site by site, so a site reached
//     from two unwrapped offsets on a small lattice is hopped twice, as in the
//     reference;
//   * the orders are rotated once more at x and its 8 neighbours (:1583-1690) and
//     combined with xk(n) = (kappa cos(delta))^n into s0 (orders 1 and 3, or 5),
//     s1 and pscalar (orders 2 and 4, or 6) (:1700-1800);
//   * gammaCurrentCalcP / gammaCurrentCalcM (:9735-10495) form the point-split
//     currents, scalarCalc (:9261-9299) psibar psi and psibar gamma5 psi, and the
//     sums go into opertemp(op, t, momentum, isb) with the momentum factors ffac / fas
//     of :955-985 (:1870-2025);
//   * the orders are zeroed on the shells the reference zeroes (:2037-2227) and
//     opertemp is copied into Jvev (:2233-2280).
// The unused running sums xrr2 .. xsj3pi (written only under an "if (.false.)" print,
// :2361-2470) are not restated.  Arithmetic follows the reference's expression order.
//
// oq_twvev_sites restricts the site loop to a given list of sites and returns their
// opertemp contributions (used by the tests to compare single sites with an
// independent full-lattice expansion).
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle_impl.h"

namespace {

struct VevLattice {
  int nx, ny, nz, nt, nxyz, nxyzt;
  // 1-based coordinates, periodic wrap as the reference's mod(a-1+n,n)+1
  int site(int x, int y, int z, int t) const {
    return x + nx * (y - 1) + nx * ny * (z - 1) + nxyz * (t - 1);
  }
  static int wrap(int a, int n) { return ((a - 1) % n + n) % n + 1; }
};

struct VevState {
  const VevLattice& L;
  int ir;
  bool fixbc;
  double cosd, sind;
  // links: uss(site, mu 1..3, ri, a, b) and usp(site, ri, a, b), 1-based
  std::vector<double> U;
  // sb1..sb6 real / imaginary, z2, z3: [site][colour][spin]
  std::vector<double> sbr[7], sbi[7], z2, z3, z3i;
  std::vector<double> s0, s1, pscalar;
  std::vector<double> rhor, rhoi, j1pr, j1pi, j2pr, j2pi, j3pr, j3pi, psir, psii, psur, psui;

  explicit VevState(const VevLattice& l) : L(l) {
    const size_t n = (size_t)L.nxyzt * 12;
    U.assign((size_t)L.nxyzt * 4 * 2 * 9, 0.0);
    for (int k = 1; k <= 6; ++k) {
      sbr[k].assign(n, 0.0);
      sbi[k].assign(n, 0.0);
    }
    z2.assign(n, 0.0);
    z3.assign(n, 0.0);
    z3i.assign(n, 0.0);
    for (auto* v : {&s0, &s1, &pscalar, &rhor, &rhoi, &j1pr, &j1pi, &j2pr, &j2pi, &j3pr, &j3pi, &psir,
                    &psii, &psur, &psui})
      v->assign((size_t)L.nxyzt + 1, 0.0);
  }
  static size_t fi(int site, int c, int d) { return ((size_t)(site - 1) * 3 + (c - 1)) * 4 + (d - 1); }
  double& uss(int site, int mu, int ri, int a, int b) {
    return U[(((size_t)(site - 1) * 4 + (mu - 1)) * 2 + (ri - 1)) * 9 + 3 * (a - 1) + (b - 1)];
  }
  double& usp(int site, int ri, int a, int b) { return uss(site, 4, ri, a, b); }

  // GammaMultiplyP (ir = 1) / GammaMultiplyM (ir = -1), :8163-8873.  The M form negates
  // the diagonal (Wilson) terms and swaps the time projectors; its off-diagonal terms
  // are those of the P form.
  void gamma_multiply(std::vector<double>& o_r, std::vector<double>& o_i, const std::vector<double>& x_r,
                      const std::vector<double>& x_i, int ax, int ay, int az, int at) {
    const int nx = L.nx, ny = L.ny, nz = L.nz, nt = L.nt;
    const int bx = VevLattice::wrap(ax, nx), by = VevLattice::wrap(ay, ny), bz = VevLattice::wrap(az, nz),
              bt = VevLattice::wrap(at, nt);
    const int ahere = L.site(bx, by, bz, bt);
    const int leftx = L.site(VevLattice::wrap(bx - 1, nx), by, bz, bt);
    const int rightx = L.site(VevLattice::wrap(bx + 1, nx), by, bz, bt);
    const int lefty = L.site(bx, VevLattice::wrap(by - 1, ny), bz, bt);
    const int righty = L.site(bx, VevLattice::wrap(by + 1, ny), bz, bt);
    const int leftz = L.site(bx, by, VevLattice::wrap(bz - 1, nz), bt);
    const int rightz = L.site(bx, by, VevLattice::wrap(bz + 1, nz), bt);
    const int leftt = L.site(bx, by, bz, VevLattice::wrap(bt - 1, nt));
    const int rightt = L.site(bx, by, bz, VevLattice::wrap(bt + 1, nt));
    double mr[4][5], mi[4][5];  // multsb1 at ahere, [colour][spin] 1-based
    for (int kc = 1; kc <= 3; ++kc)
      for (int kd = 1; kd <= 4; ++kd) {
        mr[kc][kd] = x_r[fi(ahere, kc, kd)];
        mi[kc][kd] = x_i[fi(ahere, kc, kd)];
      }
    for (int kc = 1; kc <= 3; ++kc) {
      const double sr1 = mr[kc][1], si1 = mi[kc][1], sr2 = mr[kc][2], si2 = mi[kc][2];
      mr[kc][1] = cosd * mr[kc][1] - sind * mr[kc][3];
      mi[kc][1] = cosd * mi[kc][1] - sind * mi[kc][3];
      mr[kc][2] = cosd * mr[kc][2] - sind * mr[kc][4];
      mi[kc][2] = cosd * mi[kc][2] - sind * mi[kc][4];
      mr[kc][3] = cosd * mr[kc][3] + sind * sr1;
      mi[kc][3] = cosd * mi[kc][3] + sind * si1;
      mr[kc][4] = cosd * mr[kc][4] + sind * sr2;
      mi[kc][4] = cosd * mi[kc][4] + sind * si2;
    }
    const double rs = ir;         // diagonal-term sign
    const double tf = 2.0 * ir;   // time-term factor
    auto R = [&](int s, int c, int d) -> double& { return o_r[fi(s, c, d)]; };
    auto I = [&](int s, int c, int d) -> double& { return o_i[fi(s, c, d)]; };
    for (int kd = 1; kd <= 4; ++kd)
      for (int ac = 1; ac <= 3; ++ac)
        for (int kc = 1; kc <= 3; ++kc) {
          const double vr = mr[kc][kd], vi = mi[kc][kd];
          if (!(vr != 0.0 || vi != 0.0)) continue;
          // point-split J_4 (time): U_mu(x) to leftt, U_mu^+(x) to rightt
          const bool left_t = ir == 1 ? (kd == 3 || kd == 4) : (kd == 1 || kd == 2);
          if (left_t && (!fixbc || bt != 1)) {
            R(leftt, ac, kd) = R(leftt, ac, kd) + tf * usp(leftt, 1, ac, kc) * vr - tf * usp(leftt, 2, ac, kc) * vi;
            I(leftt, ac, kd) = I(leftt, ac, kd) + tf * usp(leftt, 2, ac, kc) * vr + tf * usp(leftt, 1, ac, kc) * vi;
          } else if (!left_t && (!fixbc || bt != nt)) {
            R(rightt, ac, kd) = R(rightt, ac, kd) + tf * usp(ahere, 1, kc, ac) * vr + tf * usp(ahere, 2, kc, ac) * vi;
            I(rightt, ac, kd) = I(rightt, ac, kd) - tf * usp(ahere, 2, kc, ac) * vr + tf * usp(ahere, 1, kc, ac) * vi;
          }
          // J_1: diagonal part
          R(leftx, ac, kd) = R(leftx, ac, kd) + rs * uss(leftx, 1, 1, ac, kc) * vr - rs * uss(leftx, 1, 2, ac, kc) * vi;
          I(leftx, ac, kd) = I(leftx, ac, kd) + rs * uss(leftx, 1, 1, ac, kc) * vi + rs * uss(leftx, 1, 2, ac, kc) * vr;
          R(rightx, ac, kd) = R(rightx, ac, kd) + rs * uss(ahere, 1, 1, kc, ac) * vr + rs * uss(ahere, 1, 2, kc, ac) * vi;
          I(rightx, ac, kd) = I(rightx, ac, kd) + rs * uss(ahere, 1, 1, kc, ac) * vi - rs * uss(ahere, 1, 2, kc, ac) * vr;
          // J_1: off-diagonal part
          R(leftx, ac, 5 - kd) = R(leftx, ac, 5 - kd) - uss(leftx, 1, 1, ac, kc) * vr + uss(leftx, 1, 2, ac, kc) * vi;
          I(leftx, ac, 5 - kd) = I(leftx, ac, 5 - kd) - uss(leftx, 1, 1, ac, kc) * vi - uss(leftx, 1, 2, ac, kc) * vr;
          R(rightx, ac, 5 - kd) = R(rightx, ac, 5 - kd) + uss(ahere, 1, 1, kc, ac) * vr + uss(ahere, 1, 2, kc, ac) * vi;
          I(rightx, ac, 5 - kd) = I(rightx, ac, 5 - kd) + uss(ahere, 1, 1, kc, ac) * vi - uss(ahere, 1, 2, kc, ac) * vr;
          // J_2: diagonal part
          R(lefty, ac, kd) = R(lefty, ac, kd) + rs * uss(lefty, 2, 1, ac, kc) * vr - rs * uss(lefty, 2, 2, ac, kc) * vi;
          I(lefty, ac, kd) = I(lefty, ac, kd) + rs * uss(lefty, 2, 2, ac, kc) * vr + rs * uss(lefty, 2, 1, ac, kc) * vi;
          R(righty, ac, kd) = R(righty, ac, kd) + rs * uss(ahere, 2, 1, kc, ac) * vr + rs * uss(ahere, 2, 2, kc, ac) * vi;
          I(righty, ac, kd) = I(righty, ac, kd) - rs * uss(ahere, 2, 2, kc, ac) * vr + rs * uss(ahere, 2, 1, kc, ac) * vi;
          // J_2: off-diagonal part
          if (kd % 2 == 0) {
            R(lefty, ac, 5 - kd) = R(lefty, ac, 5 - kd) - uss(lefty, 2, 2, ac, kc) * vr - uss(lefty, 2, 1, ac, kc) * vi;
            I(lefty, ac, 5 - kd) = I(lefty, ac, 5 - kd) + uss(lefty, 2, 1, ac, kc) * vr - uss(lefty, 2, 2, ac, kc) * vi;
            R(righty, ac, 5 - kd) = R(righty, ac, 5 - kd) - uss(ahere, 2, 2, kc, ac) * vr + uss(ahere, 2, 1, kc, ac) * vi;
            I(righty, ac, 5 - kd) = I(righty, ac, 5 - kd) - uss(ahere, 2, 1, kc, ac) * vr - uss(ahere, 2, 2, kc, ac) * vi;
          } else {
            R(lefty, ac, 5 - kd) = R(lefty, ac, 5 - kd) + uss(lefty, 2, 2, ac, kc) * vr + uss(lefty, 2, 1, ac, kc) * vi;
            I(lefty, ac, 5 - kd) = I(lefty, ac, 5 - kd) - uss(lefty, 2, 1, ac, kc) * vr + uss(lefty, 2, 2, ac, kc) * vi;
            R(righty, ac, 5 - kd) = R(righty, ac, 5 - kd) + uss(ahere, 2, 2, kc, ac) * vr - uss(ahere, 2, 1, kc, ac) * vi;
            I(righty, ac, 5 - kd) = I(righty, ac, 5 - kd) + uss(ahere, 2, 1, kc, ac) * vr + uss(ahere, 2, 2, kc, ac) * vi;
          }
          // J_3: diagonal part
          R(leftz, ac, kd) = R(leftz, ac, kd) + rs * uss(leftz, 3, 1, ac, kc) * vr - rs * uss(leftz, 3, 2, ac, kc) * vi;
          I(leftz, ac, kd) = I(leftz, ac, kd) + rs * uss(leftz, 3, 2, ac, kc) * vr + rs * uss(leftz, 3, 1, ac, kc) * vi;
          R(rightz, ac, kd) = R(rightz, ac, kd) + rs * uss(ahere, 3, 1, kc, ac) * vr + rs * uss(ahere, 3, 2, kc, ac) * vi;
          I(rightz, ac, kd) = I(rightz, ac, kd) - rs * uss(ahere, 3, 2, kc, ac) * vr + rs * uss(ahere, 3, 1, kc, ac) * vi;
          // J_3: off-diagonal part
          if (kd % 2 == 1) {
            const int td = 3 / kd;
            R(leftz, ac, td) = R(leftz, ac, td) - uss(leftz, 3, 1, ac, kc) * vr + uss(leftz, 3, 2, ac, kc) * vi;
            I(leftz, ac, td) = I(leftz, ac, td) - uss(leftz, 3, 2, ac, kc) * vr - uss(leftz, 3, 1, ac, kc) * vi;
            R(rightz, ac, td) = R(rightz, ac, td) + uss(ahere, 3, 1, kc, ac) * vr + uss(ahere, 3, 2, kc, ac) * vi;
            I(rightz, ac, td) = I(rightz, ac, td) - uss(ahere, 3, 2, kc, ac) * vr + uss(ahere, 3, 1, kc, ac) * vi;
          } else {
            const int td = 8 / kd;
            R(leftz, ac, td) = R(leftz, ac, td) + uss(leftz, 3, 1, ac, kc) * vr - uss(leftz, 3, 2, ac, kc) * vi;
            I(leftz, ac, td) = I(leftz, ac, td) + uss(leftz, 3, 2, ac, kc) * vr + uss(leftz, 3, 1, ac, kc) * vi;
            R(rightz, ac, td) = R(rightz, ac, td) - uss(ahere, 3, 1, kc, ac) * vr - uss(ahere, 3, 2, kc, ac) * vi;
            I(rightz, ac, td) = I(rightz, ac, td) + uss(ahere, 3, 2, kc, ac) * vr - uss(ahere, 3, 1, kc, ac) * vi;
          }
        }
  }

  // gammaCurrentCalcP (ir = 1) / gammaCurrentCalcM (ir = -1), :9735-10495: the
  // unit vector z2 is e(ahere, icolor, idirac).
  void current(const std::vector<double>& s, int jd, int icolor, int jc, int jri, int ahere, int leftx,
               int rightx, int lefty, int righty, int leftz, int rightz, int leftt, int rightt, int ittt) {
    const int nt = L.nt;
    for (auto* v : {&rhor, &rhoi}) (*v)[ahere] = (*v)[leftt] = 0.0;
    for (auto* v : {&j1pr, &j1pi}) (*v)[ahere] = (*v)[leftx] = 0.0;
    for (auto* v : {&j2pr, &j2pi}) (*v)[ahere] = (*v)[lefty] = 0.0;
    for (auto* v : {&j3pr, &j3pi}) (*v)[ahere] = (*v)[leftz] = 0.0;
    auto Z = [&](int d) { return z2[fi(ahere, icolor, d)]; };
    const double rs = ir, tf = 2.0 * ir;
    // J_4: r = 1 takes spins 1,2 at leftt and 3,4 at ahere; r = -1 the reverse
    const bool lt = ir == 1 ? (jd == 1 || jd == 2) : (jd == 3 || jd == 4);
    if (lt && (!fixbc || ittt != 1)) {
      if (jri == 1) {
        rhor[leftt] = rhor[leftt] + tf * s[leftt] * usp(leftt, 1, jc, icolor) * Z(jd);
        rhoi[leftt] = rhoi[leftt] - tf * s[leftt] * usp(leftt, 2, jc, icolor) * Z(jd);
      } else {
        rhor[leftt] = rhor[leftt] + tf * s[leftt] * usp(leftt, 2, jc, icolor) * Z(jd);
        rhoi[leftt] = rhoi[leftt] + tf * s[leftt] * usp(leftt, 1, jc, icolor) * Z(jd);
      }
    } else if (!lt && (!fixbc || ittt != nt)) {
      if (jri == 1) {
        rhor[ahere] = rhor[ahere] - tf * s[rightt] * usp(ahere, 1, icolor, jc) * Z(jd);
        rhoi[ahere] = rhoi[ahere] - tf * s[rightt] * usp(ahere, 2, icolor, jc) * Z(jd);
      } else {
        rhor[ahere] = rhor[ahere] + tf * s[rightt] * usp(ahere, 2, icolor, jc) * Z(jd);
        rhoi[ahere] = rhoi[ahere] - tf * s[rightt] * usp(ahere, 1, icolor, jc) * Z(jd);
      }
    }
    // J_mu, mu = 1..3: diagonal part (sign r) and off-diagonal part
    struct Cur {
      std::vector<double>*pr, *pi;
      int left, right, mu;
    } cur[3] = {{&j1pr, &j1pi, leftx, rightx, 1}, {&j2pr, &j2pi, lefty, righty, 2}, {&j3pr, &j3pi, leftz, rightz, 3}};
    for (auto& C : cur) {
      std::vector<double>&pr = *C.pr, &pi = *C.pi;
      const int lf = C.left, rt = C.right, mu = C.mu;
      if (jri == 1) {
        pr[ahere] = pr[ahere] - rs * s[rt] * uss(ahere, mu, 1, icolor, jc) * Z(jd);
        pr[lf] = pr[lf] + rs * s[lf] * uss(lf, mu, 1, jc, icolor) * Z(jd);
        pi[ahere] = pi[ahere] - rs * s[rt] * uss(ahere, mu, 2, icolor, jc) * Z(jd);
        pi[lf] = pi[lf] - rs * s[lf] * uss(lf, mu, 2, jc, icolor) * Z(jd);
      } else {
        pr[ahere] = pr[ahere] + rs * s[rt] * uss(ahere, mu, 2, icolor, jc) * Z(jd);
        pr[lf] = pr[lf] + rs * s[lf] * uss(lf, mu, 2, jc, icolor) * Z(jd);
        pi[ahere] = pi[ahere] - rs * s[rt] * uss(ahere, mu, 1, icolor, jc) * Z(jd);
        pi[lf] = pi[lf] + rs * s[lf] * uss(lf, mu, 1, jc, icolor) * Z(jd);
      }
    }
    // J_1 off-diagonal (spin 5 - jd)
    {
      const int od = 5 - jd;
      if (jri == 1) {
        j1pr[ahere] = j1pr[ahere] + s[rightx] * uss(ahere, 1, 1, icolor, jc) * Z(od);
        j1pr[leftx] = j1pr[leftx] + s[leftx] * uss(leftx, 1, 1, jc, icolor) * Z(od);
        j1pi[ahere] = j1pi[ahere] + s[rightx] * uss(ahere, 1, 2, icolor, jc) * Z(od);
        j1pi[leftx] = j1pi[leftx] - s[leftx] * uss(leftx, 1, 2, jc, icolor) * Z(od);
      } else {
        j1pr[ahere] = j1pr[ahere] - s[rightx] * uss(ahere, 1, 2, icolor, jc) * Z(od);
        j1pr[leftx] = j1pr[leftx] + s[leftx] * uss(leftx, 1, 2, jc, icolor) * Z(od);
        j1pi[ahere] = j1pi[ahere] + s[rightx] * uss(ahere, 1, 1, icolor, jc) * Z(od);
        j1pi[leftx] = j1pi[leftx] + s[leftx] * uss(leftx, 1, 1, jc, icolor) * Z(od);
      }
    }
    // J_2 off-diagonal (spin 5 - jd, phase by the parity of jd)
    {
      const int od = 5 - jd;
      if (jd % 2 == 1) {
        if (jri == 1) {
          j2pr[ahere] = j2pr[ahere] - s[righty] * uss(ahere, 2, 2, icolor, jc) * Z(od);
          j2pr[lefty] = j2pr[lefty] + s[lefty] * uss(lefty, 2, 2, jc, icolor) * Z(od);
          j2pi[ahere] = j2pi[ahere] + s[righty] * uss(ahere, 2, 1, icolor, jc) * Z(od);
          j2pi[lefty] = j2pi[lefty] + s[lefty] * uss(lefty, 2, 1, jc, icolor) * Z(od);
        } else {
          j2pr[ahere] = j2pr[ahere] - s[righty] * uss(ahere, 2, 1, icolor, jc) * Z(od);
          j2pr[lefty] = j2pr[lefty] - s[lefty] * uss(lefty, 2, 1, jc, icolor) * Z(od);
          j2pi[ahere] = j2pi[ahere] - s[righty] * uss(ahere, 2, 2, icolor, jc) * Z(od);
          j2pi[lefty] = j2pi[lefty] + s[lefty] * uss(lefty, 2, 2, jc, icolor) * Z(od);
        }
      } else {
        if (jri == 1) {
          j2pr[ahere] = j2pr[ahere] + s[righty] * uss(ahere, 2, 2, icolor, jc) * Z(od);
          j2pr[lefty] = j2pr[lefty] - s[lefty] * uss(lefty, 2, 2, jc, icolor) * Z(od);
          j2pi[ahere] = j2pi[ahere] - s[righty] * uss(ahere, 2, 1, icolor, jc) * Z(od);
          j2pi[lefty] = j2pi[lefty] - s[lefty] * uss(lefty, 2, 1, jc, icolor) * Z(od);
        } else {
          j2pr[ahere] = j2pr[ahere] + s[righty] * uss(ahere, 2, 1, icolor, jc) * Z(od);
          j2pr[lefty] = j2pr[lefty] + s[lefty] * uss(lefty, 2, 1, jc, icolor) * Z(od);
          j2pi[ahere] = j2pi[ahere] + s[righty] * uss(ahere, 2, 2, icolor, jc) * Z(od);
          j2pi[lefty] = j2pi[lefty] - s[lefty] * uss(lefty, 2, 2, jc, icolor) * Z(od);
        }
      }
    }
    // J_3 off-diagonal (spin 3/jd for odd jd, 8/jd for even jd)
    if (jd % 2 == 1) {
      const int od = 3 / jd;
      if (jri == 1) {
        j3pr[ahere] = j3pr[ahere] + s[rightz] * uss(ahere, 3, 1, icolor, jc) * Z(od);
        j3pr[leftz] = j3pr[leftz] + s[leftz] * uss(leftz, 3, 1, jc, icolor) * Z(od);
        j3pi[ahere] = j3pi[ahere] + s[rightz] * uss(ahere, 3, 2, icolor, jc) * Z(od);
        j3pi[leftz] = j3pi[leftz] - s[leftz] * uss(leftz, 3, 2, jc, icolor) * Z(od);
      } else {
        j3pr[ahere] = j3pr[ahere] - s[rightz] * uss(ahere, 3, 2, icolor, jc) * Z(od);
        j3pr[leftz] = j3pr[leftz] + s[leftz] * uss(leftz, 3, 2, jc, icolor) * Z(od);
        j3pi[ahere] = j3pi[ahere] + s[rightz] * uss(ahere, 3, 1, icolor, jc) * Z(od);
        j3pi[leftz] = j3pi[leftz] + s[leftz] * uss(leftz, 3, 1, jc, icolor) * Z(od);
      }
    } else {
      const int od = 8 / jd;
      if (jri == 1) {
        j3pr[ahere] = j3pr[ahere] - s[rightz] * uss(ahere, 3, 1, icolor, jc) * Z(od);
        j3pr[leftz] = j3pr[leftz] - s[leftz] * uss(leftz, 3, 1, jc, icolor) * Z(od);
        j3pi[ahere] = j3pi[ahere] - s[rightz] * uss(ahere, 3, 2, icolor, jc) * Z(od);
        j3pi[leftz] = j3pi[leftz] + s[leftz] * uss(leftz, 3, 2, jc, icolor) * Z(od);
      } else {
        j3pr[ahere] = j3pr[ahere] + s[rightz] * uss(ahere, 3, 2, icolor, jc) * Z(od);
        j3pr[leftz] = j3pr[leftz] - s[leftz] * uss(leftz, 3, 2, jc, icolor) * Z(od);
        j3pi[ahere] = j3pi[ahere] - s[rightz] * uss(ahere, 3, 1, icolor, jc) * Z(od);
        j3pi[leftz] = j3pi[leftz] - s[leftz] * uss(leftz, 3, 1, jc, icolor) * Z(od);
      }
    }
  }

  // scalarCalc, :9261-9299 (signal 1: psibar psi, 2: psibar gamma5 psi)
  void scalar(const std::vector<double>& sc, int idirac, int icolor, int jri, int ahere, int signal) {
    const double z = z2[fi(ahere, icolor, idirac)];
    if (signal == 1) {
      psir[ahere] = 0.0;
      psii[ahere] = 0.0;
      if (jri == 1) psir[ahere] = psir[ahere] + sc[ahere] * z;
      else psii[ahere] = psii[ahere] + sc[ahere] * z;
    } else {
      psur[ahere] = 0.0;
      psui[ahere] = 0.0;
      if (jri == 1) psur[ahere] = psur[ahere] + sc[ahere] * z;
      else psui[ahere] = psui[ahere] + sc[ahere] * z;
    }
  }
};

// The diamond shell |b|_1 = md in the reference's order: bx, by, bz ascending, then
// bt = md - |bx| - |by| - |bz| and, when bt /= 0, -bt.
template <class F>
void shell(int md, F&& f) {
  for (int bx = -md; bx <= md; ++bx)
    for (int by = -(md - std::abs(bx)); by <= md - std::abs(bx); ++by)
      for (int bz = -(md - std::abs(bx) - std::abs(by)); bz <= md - std::abs(bx) - std::abs(by); ++bz) {
        const int bt = md - std::abs(bx) - std::abs(by) - std::abs(bz);
        f(bx, by, bz, bt);
        if (bt != 0) f(bx, by, bz, -bt);
      }
}

// opertemp(op 1..12, t 1..nt, ix 1..5, isb 0..1) -> [((isb * 5 + (ix-1)) * nt + (t-1)) * 12 + op-1]
void vev_sites(const oq_geom* g, const double* u, double kappa, double delta, const int io[3], int dobndry,
               int ir, int nsub, const int* sites, int nsites, double* opertemp) {
  const VevLattice L{g->n[0], g->n[1], g->n[2], g->n[3], g->n[0] * g->n[1] * g->n[2],
                     g->n[0] * g->n[1] * g->n[2] * g->n[3]};
  const int nx = L.nx, ny = L.ny, nz = L.nz, nt = L.nt;
  VevState S(L);
  S.ir = ir;
  S.fixbc = dobndry == 1;
  // utouss: links to lexicographic order
  for (int t = 0; t < nt; ++t)
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const int xc[4] = {x, y, z, t};
          int isite, ieo, ibl, gblclr, ibleo;
          oq_site_of_coords(g, xc, &isite, &ieo, &ibl, &gblclr, &ibleo);
          const int s = L.site(x + 1, y + 1, z + 1, t + 1);
          for (int mu = 1; mu <= 4; ++mu)
            for (int a = 1; a <= 3; ++a)
              for (int b = 1; b <= 3; ++b) {
                S.uss(s, mu, 1, a, b) = u[g->ui(2 * (3 * (a - 1) + (b - 1)) + 1, isite, mu, ieo, ibl)];
                S.uss(s, mu, 2, a, b) = u[g->ui(2 * (3 * (a - 1) + (b - 1)) + 2, isite, mu, ieo, ibl)];
              }
        }
  if (S.fixbc)  // usp = 0 on the last time slice (:1050-1066)
    for (int z = 1; z <= nz; ++z)
      for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x)
          for (int ri = 1; ri <= 2; ++ri)
            for (int a = 1; a <= 3; ++a)
              for (int b = 1; b <= 3; ++b) S.usp(L.site(x, y, z, nt), ri, a, b) = 0.0;
  // momentum factors (:955-985)
  std::vector<double> ffac((size_t)L.nxyzt * 5), fas1(ffac.size()), fas2(ffac.size()), fas3(ffac.size());
  auto FI = [&](int isp, int k) { return (size_t)(isp - 1) * 5 + k; };
  const double pmom1 = 8.0 * std::atan(1.0) / nx, pmom2 = 8.0 * std::atan(1.0) / ny,
               pmom3 = 8.0 * std::atan(1.0) / nz;
  for (int itr = 1; itr <= nt; ++itr)
    for (int isz = 1; isz <= nz; ++isz) {
      const double dz = (double)(isz - io[2]) * pmom3;
      for (int isy = 1; isy <= ny; ++isy) {
        const double dy = (double)(isy - io[1]) * pmom2;
        for (int isx = 1; isx <= nx; ++isx) {
          const double dx = (double)(isx - io[0]) * pmom1;
          const int isp = L.site(isx, isy, isz, itr);
          ffac[FI(isp, 1)] = (std::cos(dx) + std::cos(dy) + std::cos(dz)) / 3.0;
          fas1[FI(isp, 1)] = std::sin(dx);
          fas2[FI(isp, 1)] = std::sin(dy);
          fas3[FI(isp, 1)] = std::sin(dz);
          ffac[FI(isp, 2)] = (std::cos(dx) * std::cos(dy) + std::cos(dx) * std::cos(dz) + std::cos(dy) * std::cos(dz)) / 3.0;
          fas1[FI(isp, 2)] = std::sin(dx) * (std::cos(dy) + std::cos(dz)) / 2.0;
          fas2[FI(isp, 2)] = std::sin(dy) * (std::cos(dx) + std::cos(dz)) / 2.0;
          fas3[FI(isp, 2)] = std::sin(dz) * (std::cos(dx) + std::cos(dy)) / 2.0;
          ffac[FI(isp, 3)] = std::cos(dx) * std::cos(dy) * std::cos(dz);
          fas1[FI(isp, 3)] = std::sin(dx) * std::cos(dy) * std::cos(dz);
          fas2[FI(isp, 3)] = std::sin(dy) * std::cos(dx) * std::cos(dz);
          fas3[FI(isp, 3)] = std::sin(dz) * std::cos(dx) * std::cos(dy);
          ffac[FI(isp, 4)] = (std::cos(2.0 * dx) + std::cos(2.0 * dy) + std::cos(2.0 * dz)) / 3.0;
          fas1[FI(isp, 4)] = std::sin(2.0 * dx);
          fas2[FI(isp, 4)] = std::sin(2.0 * dy);
          fas3[FI(isp, 4)] = std::sin(2.0 * dz);
        }
      }
    }
  S.cosd = std::cos(delta);
  S.sind = std::sin(delta);
  const double cosd = S.cosd, sind = S.sind;
  const double xkappa = kappa * cosd;
  double xk[7];
  xk[1] = xkappa;
  xk[2] = xkappa * xkappa;
  xk[3] = xkappa * xkappa * xkappa;
  xk[4] = (xkappa * xkappa) * (xkappa * xkappa);
  xk[5] = (xkappa * xkappa) * (xkappa * xkappa) * xkappa;
  xk[6] = (xkappa * xkappa) * (xkappa * xkappa) * (xkappa * xkappa);
  const bool twist = std::fabs(delta) > 1.e-12;
  const int cd[5] = {0, 3, 4, 1, 2};
  const double sgn[5] = {0, 1, 1, -1, -1};
  auto OP = [&](int op, int t, int ix, int isb) -> double& {
    return opertemp[((size_t)(isb * 5 + (ix - 1)) * nt + (t - 1)) * 12 + (op - 1)];
  };
  std::memset(opertemp, 0, sizeof(double) * 12 * nt * 5 * 2);
  auto& sbr = S.sbr;
  auto& sbi = S.sbi;
  auto fi = VevState::fi;

  for (int n = 0; n < nsites; ++n) {
    const int ihere = sites[n];
    const int ixx = (ihere - 1) % nx + 1, iyy = ((ihere - 1) / nx) % ny + 1, izz = ((ihere - 1) / (nx * ny)) % nz + 1,
              ittt = (ihere - 1) / L.nxyz + 1;
    for (int idirac = 1; idirac <= 4; ++idirac)
      for (int icolor = 1; icolor <= 3; ++icolor) {
        S.z2[fi(ihere, icolor, idirac)] = 1.0;
        S.z3[fi(ihere, icolor, idirac)] = cosd * S.z2[fi(ihere, icolor, idirac)];
        // first order
        S.gamma_multiply(sbr[1], sbi[1], S.z3, S.z3i, ixx, iyy, izz, ittt);
        // orders 2..6 from the shells
        auto order = [&](int k, int md) {
          shell(md, [&](int bx, int by, int bz, int bt) {
            S.gamma_multiply(sbr[k], sbi[k], sbr[k - 1], sbi[k - 1], ixx + bx, iyy + by, izz + bz, ittt + bt);
          });
        };
        order(2, 1);
        S.gamma_multiply(sbr[3], sbi[3], sbr[2], sbi[2], ixx, iyy, izz, ittt);
        order(3, 2);
        order(4, 1);
        order(4, 3);
        S.gamma_multiply(sbr[5], sbi[5], sbr[4], sbi[4], ixx, iyy, izz, ittt);
        order(5, 2);
        order(6, 1);

        const int leftx = L.site(VevLattice::wrap(ixx - 1, nx), iyy, izz, ittt);
        const int rightx = L.site(VevLattice::wrap(ixx + 1, nx), iyy, izz, ittt);
        const int lefty = L.site(ixx, VevLattice::wrap(iyy - 1, ny), izz, ittt);
        const int righty = L.site(ixx, VevLattice::wrap(iyy + 1, ny), izz, ittt);
        const int leftz = L.site(ixx, iyy, VevLattice::wrap(izz - 1, nz), ittt);
        const int rightz = L.site(ixx, iyy, VevLattice::wrap(izz + 1, nz), ittt);
        const int leftt = L.site(ixx, iyy, izz, VevLattice::wrap(ittt - 1, nt));
        const int rightt = L.site(ixx, iyy, izz, VevLattice::wrap(ittt + 1, nt));
        const int imv[9] = {ihere, leftx, rightx, lefty, righty, leftz, rightz, leftt, rightt};
        // rotation at the end (:1583-1690)
        for (int ii = 0; ii < 9; ++ii)
          for (int jc = 1; jc <= 3; ++jc)
            for (int k = 1; k <= 6; ++k)
              for (auto* a : {&sbr[k], &sbi[k]}) {
                std::vector<double>& v = *a;
                const int ih = imv[ii];
                const double b1 = v[fi(ih, jc, 1)], b2 = v[fi(ih, jc, 2)];
                v[fi(ih, jc, 1)] = cosd * v[fi(ih, jc, 1)] - sind * v[fi(ih, jc, 3)];
                v[fi(ih, jc, 2)] = cosd * v[fi(ih, jc, 2)] - sind * v[fi(ih, jc, 4)];
                v[fi(ih, jc, 3)] = cosd * v[fi(ih, jc, 3)] + sind * b1;
                v[fi(ih, jc, 4)] = cosd * v[fi(ih, jc, 4)] + sind * b2;
              }

        for (int jd = 1; jd <= 4; ++jd)
          for (int jri = 1; jri <= 2; ++jri)
            for (int jc = 1; jc <= 3; ++jc)
              for (int isb = 0; isb <= 1; ++isb) {
                const auto& A = jri == 1 ? sbr : sbi;  // the part s0 / s1 take
                const auto& B = jri == 1 ? sbi : sbr;  // the part pscalar takes
                const double psg = jri == 1 ? 1.0 : -1.0;
                if (isb == 0) {
                  for (int ii = 0; ii < 9; ++ii) {
                    const int ih = imv[ii];
                    S.s0[ih] = twist ? xk[1] * A[1][fi(ih, jc, jd)] + xk[3] * A[3][fi(ih, jc, jd)]
                                     : xk[3] * A[3][fi(ih, jc, jd)];
                  }
                  if (jc == icolor) {
                    if (twist) {
                      S.s1[ihere] = xk[2] * A[2][fi(ihere, jc, jd)] + xk[4] * A[4][fi(ihere, jc, jd)];
                      S.pscalar[ihere] = psg * sgn[jd] *
                                         (xk[2] * B[2][fi(ihere, jc, cd[jd])] + xk[4] * B[4][fi(ihere, jc, cd[jd])]);
                    } else {
                      S.s1[ihere] = xk[4] * A[4][fi(ihere, jc, jd)];
                      S.pscalar[ihere] = psg * sgn[jd] * xk[4] * B[4][fi(ihere, jc, cd[jd])];
                    }
                  }
                } else {
                  for (int ii = 0; ii < 9; ++ii) {
                    const int ih = imv[ii];
                    S.s0[ih] = xk[5] * A[5][fi(ih, jc, jd)];
                  }
                  if (jc == icolor) {
                    S.s1[ihere] = xk[6] * A[6][fi(ihere, jc, jd)];
                    S.pscalar[ihere] = psg * sgn[jd] * xk[6] * B[6][fi(ihere, jc, cd[jd])];
                  }
                }
                S.current(S.s0, jd, icolor, jc, jri, ihere, leftx, rightx, lefty, righty, leftz, rightz, leftt,
                          rightt, ittt);
                if (jc == icolor) {
                  S.scalar(S.s1, jd, jc, jri, ihere, 1);
                  S.scalar(S.pscalar, jd, jc, jri, ihere, 2);
                }
                const int tm1 = ((ittt - 1) - 1 + nt) % nt + 1;
                OP(1, ittt, 1, isb) = OP(1, ittt, 1, isb) + S.rhor[ihere];
                OP(1, tm1, 1, isb) = OP(1, tm1, 1, isb) + S.rhor[leftt];
                OP(2, ittt, 1, isb) = OP(2, ittt, 1, isb) + S.rhoi[ihere];
                OP(2, tm1, 1, isb) = OP(2, tm1, 1, isb) + S.rhoi[leftt];
                if (jc == icolor) {
                  OP(3, ittt, 1, isb) = OP(3, ittt, 1, isb) + S.psir[ihere];
                  OP(4, ittt, 1, isb) = OP(4, ittt, 1, isb) + S.psii[ihere];
                }
                OP(5, ittt, 1, isb) = OP(5, ittt, 1, isb) + S.j1pr[ihere] + S.j1pr[leftx];
                OP(6, ittt, 1, isb) = OP(6, ittt, 1, isb) + S.j1pi[ihere] + S.j1pi[leftx];
                OP(7, ittt, 1, isb) = OP(7, ittt, 1, isb) + S.j2pr[ihere] + S.j2pr[lefty];
                OP(8, ittt, 1, isb) = OP(8, ittt, 1, isb) + S.j2pi[ihere] + S.j2pi[lefty];
                OP(9, ittt, 1, isb) = OP(9, ittt, 1, isb) + S.j3pr[ihere] + S.j3pr[leftz];
                OP(10, ittt, 1, isb) = OP(10, ittt, 1, isb) + S.j3pi[ihere] + S.j3pi[leftz];
                if (jc == icolor) {
                  OP(11, ittt, 1, isb) = OP(11, ittt, 1, isb) + S.psur[ihere];
                  OP(12, ittt, 1, isb) = OP(12, ittt, 1, isb) + S.psui[ihere];
                }
                for (int ix = 2; ix <= 5; ++ix) {
                  const int k = ix - 1;
                  OP(1, ittt, ix, isb) = OP(1, ittt, ix, isb) + S.rhor[ihere] * ffac[FI(ihere, k)];
                  OP(1, tm1, ix, isb) = OP(1, tm1, ix, isb) + S.rhor[leftt] * ffac[FI(leftt, k)];
                  OP(2, ittt, ix, isb) = OP(2, ittt, ix, isb) + S.rhoi[ihere] * ffac[FI(ihere, k)];
                  OP(2, tm1, ix, isb) = OP(2, tm1, ix, isb) + S.rhoi[leftt] * ffac[FI(leftt, k)];
                  if (jc == icolor) {
                    OP(3, ittt, ix, isb) = OP(3, ittt, ix, isb) + S.psir[ihere] * ffac[FI(ihere, k)];
                    OP(4, ittt, ix, isb) = OP(4, ittt, ix, isb) + S.psii[ihere] * ffac[FI(ihere, k)];
                  }
                  OP(5, ittt, ix, isb) = OP(5, ittt, ix, isb) + S.j1pi[ihere] * fas3[FI(ihere, k)] +
                                         S.j1pi[leftx] * fas3[FI(leftx, k)];
                  OP(6, ittt, ix, isb) = OP(6, ittt, ix, isb) + S.j2pi[ihere] * fas1[FI(ihere, k)] +
                                         S.j2pi[lefty] * fas1[FI(lefty, k)];
                  OP(7, ittt, ix, isb) = OP(7, ittt, ix, isb) + S.j3pi[ihere] * fas2[FI(ihere, k)] +
                                         S.j3pi[leftz] * fas2[FI(leftz, k)];
                  OP(8, ittt, ix, isb) = OP(8, ittt, ix, isb) + S.j1pi[ihere] * fas2[FI(ihere, k)] +
                                         S.j1pi[leftx] * fas2[FI(leftx, k)];
                  OP(9, ittt, ix, isb) = OP(9, ittt, ix, isb) + S.j2pi[ihere] * fas3[FI(ihere, k)] +
                                         S.j2pi[lefty] * fas3[FI(lefty, k)];
                  OP(10, ittt, ix, isb) = OP(10, ittt, ix, isb) + S.j3pi[ihere] * fas1[FI(ihere, k)] +
                                          S.j3pi[leftz] * fas1[FI(leftz, k)];
                  if (jc == icolor) {
                    OP(11, ittt, ix, isb) = OP(11, ittt, ix, isb) + S.psur[ihere] * ffac[FI(ihere, k)];
                    OP(12, ittt, ix, isb) = OP(12, ittt, ix, isb) + S.psui[ihere] * ffac[FI(ihere, k)];
                  }
                }
              }

        // zeroing (:2037-2227)
        auto zero_shell = [&](int md, std::initializer_list<int> ks) {
          shell(md, [&](int bx, int by, int bz, int bt) {
            const int s = L.site(VevLattice::wrap(ixx + bx, nx), VevLattice::wrap(iyy + by, ny),
                                 VevLattice::wrap(izz + bz, nz), VevLattice::wrap(ittt + bt, nt));
            for (int jd = 1; jd <= 4; ++jd)
              for (int jc = 1; jc <= 3; ++jc)
                for (int k : ks) sbr[k][fi(s, jc, jd)] = sbi[k][fi(s, jc, jd)] = 0.0;
          });
        };
        if (nsub == 6) {
          zero_shell(6, {6});
          zero_shell(5, {5});
        }
        zero_shell(4, {6, 4});
        zero_shell(3, {3, 5});
        for (int md = 0; md <= 2; ++md) zero_shell(md, {1, 2, 3, 4, 5, 6});
        S.z2[fi(ihere, icolor, idirac)] = 0.0;
        for (int d = 1; d <= 4; ++d) S.z3[fi(ihere, icolor, d)] = 0.0;
      }
  }
}

}  // namespace

extern "C" void oq_twvev_sites(const oq_geom* g, const double* u, double kappa, double delta, const int io[3],
                               int dobndry, int ir, int nsub, const int* sites, int nsites, double* opertemp) {
  vev_sites(g, u, kappa, delta, io, dobndry, ir, nsub, sites, nsites, opertemp);
}

extern "C" void oq_twvev(const oq_geom* g, const double* u, double kappa, double delta, const int io[3],
                         int dobndry, int ir, int nsub, int nmom, int nop, double* Jvev) {
  const int nt = g->n[3], V = g->n[0] * g->n[1] * g->n[2] * nt;
  std::vector<int> sites(V);
  for (int i = 0; i < V; ++i) sites[i] = i + 1;
  std::vector<double> oper((size_t)12 * nt * 5 * 2);
  vev_sites(g, u, kappa, delta, io, dobndry, ir, nsub, sites.data(), V, oper.data());
  // Jvev(2, nt, 6, nmom, nop) <- opertemp (:2233-2280)
  std::memset(Jvev, 0, sizeof(double) * 2 * nt * 6 * nmom * nop);
  auto J = [&](int ri, int t, int lv, int imom, int iop) -> double& {
    return Jvev[(((size_t)(iop - 1) * nmom + (imom - 1)) * 6 + (lv - 1)) * nt * 2 + (size_t)(t - 1) * 2 + (ri - 1)];
  };
  auto O = [&](int op, int t, int ix, int isb) {
    return oper[((size_t)(isb * 5 + (ix - 1)) * nt + (t - 1)) * 12 + (op - 1)];
  };
  for (int t = 1; t <= nt; ++t)
    for (int imom = 1; imom <= nmom; ++imom)
      for (int iop = 1; iop <= 6; ++iop) {
        if (nsub == 4 || nsub == 6) {
          J(1, t, 4, imom, iop) = O(2 * iop - 1, t, imom, 0);
          J(2, t, 4, imom, iop) = O(2 * iop, t, imom, 0);
        }
        if (nsub == 6) {
          J(1, t, 6, imom, iop) = O(2 * iop - 1, t, imom, 1);
          J(2, t, 6, imom, iop) = O(2 * iop, t, imom, 1);
        }
      }
}
