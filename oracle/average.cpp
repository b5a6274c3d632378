// CPU oracle (test infrastructure): the Wilson loop operators of one noise with the
// perturbative subtraction levels of the Wilson driver, restating
//   * average, Q/disconloops.f90:5343-5733: level isub = 1 takes the solution x as it
//     is; level isub >= 2 subtracts from x the hopping expansion of the propagator
//     applied to the noise, sub = b + kappa H b + ... + kappa^(isub+1) H^(isub+1) b,
//     built with Hsingle (H_eo on the odd half, H_oe on the even half) in the order of
//     :5398-5614; the operators of x - sub go through loopops and spacesum into
//     Jtime(:, :, isub, :, :); finally operators 1..4 are multiplied by kappa (:5728-5731);
//   * loopops, :7769-7910 (with mulfor2 :8374-8465, mulbac2 :8574-8675, vgv :8829-8921,
//     vv :8788-8825, gammamultshort Q/diracops.f90:204-257): per site x and direction mu
//       J_mu = conj( y(x+mu)^+ (1 - gamma_mu) U_mu(x)^+ b(x)
//                    - y(x)^+ (1 + gamma_mu) U_mu(x) b(x+mu) ),
//     the neighbours carrying the boundary factor bc(mu) where they cross the lattice
//     edge, J_5 = conj(y^+ b) (+ 12 on subtracted levels), J_{5+mu} = conj(y^+ gamma_mu b),
//     with the complex noise b (this driver keeps its imaginary part);
//   * spacesum, :9012-9124: time-slice sums of all operators at imom = 1 and, for
//     imom = 2..nmom, the caller's momentum factors momfac(isite, ieo, ibl, imom-1, k) on
//     operators 1..5 with the reference's slot assignment.
// Output Jtime(2, nt, nsub, nmom, nop), Fortran order, nop >= 9.
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "oracle_impl.h"

namespace {

using C = std::complex<double>;

// (gamma_mu v)_d in the reference basis (Q/diracops.f90:61-71, gammamultshort)
void gamma_mult(int mu, const C v[4][3], C out[4][3]) {
  const C I(0.0, 1.0);
  for (int c = 0; c < 3; ++c) {
    switch (mu) {
      case 0:
        out[0][c] = v[3][c], out[1][c] = v[2][c], out[2][c] = v[1][c], out[3][c] = v[0][c];
        break;
      case 1:
        out[0][c] = -I * v[3][c], out[1][c] = I * v[2][c], out[2][c] = -I * v[1][c], out[3][c] = I * v[0][c];
        break;
      case 2:
        out[0][c] = v[2][c], out[1][c] = -v[3][c], out[2][c] = v[0][c], out[3][c] = -v[1][c];
        break;
      default:
        out[0][c] = v[0][c], out[1][c] = v[1][c], out[2][c] = -v[2][c], out[3][c] = -v[3][c];
        break;
    }
  }
}

struct AvLattice {
  const oq_geom* g;
  int n[4], V;
  std::vector<int> isite, ieo, ibl, ibleo, par;
  explicit AvLattice(const oq_geom* geo) : g(geo) {
    for (int d = 0; d < 4; ++d) n[d] = g->n[d];
    V = n[0] * n[1] * n[2] * n[3];
    isite.resize(V), ieo.resize(V), ibl.resize(V), ibleo.resize(V), par.resize(V);
    for (int L = 0; L < V; ++L) {
      const int xc[4] = {L % n[0], (L / n[0]) % n[1], (L / (n[0] * n[1])) % n[2], L / (n[0] * n[1] * n[2])};
      int gblclr;
      oq_site_of_coords(g, xc, &isite[L], &ieo[L], &ibl[L], &gblclr, &ibleo[L]);
      par[L] = gblclr;
    }
  }
  // neighbour in direction mu (+1 / -1) and the boundary factor of that hop
  int nb(int L, int mu, int s, double* f) const {
    int c[4] = {L % n[0], (L / n[0]) % n[1], (L / (n[0] * n[1])) % n[2], L / (n[0] * n[1] * n[2])};
    int v = c[mu] + s;
    *f = 1.0;
    if (v < 0 || v >= n[mu]) *f = g->bc[mu];
    c[mu] = (v + n[mu]) % n[mu];
    return c[0] + n[0] * (c[1] + n[1] * (c[2] + n[2] * c[3]));
  }
  void spinor(const double* he, const double* ho, int L, C v[4][3]) const {
    const double* h = par[L] == 1 ? he : ho;
    for (int d = 0; d < 4; ++d)
      for (int c = 0; c < 3; ++c)
        v[d][c] = C(h[g->gi(2 * c + 1, isite[L], d + 1, ieo[L], ibleo[L])],
                    h[g->gi(2 * c + 2, isite[L], d + 1, ieo[L], ibleo[L])]);
  }
  C link(const double* u, int L, int mu, int a, int b) const {
    return C(u[g->ui(2 * (3 * a + b) + 1, isite[L], mu + 1, ieo[L], ibl[L])],
             u[g->ui(2 * (3 * a + b) + 2, isite[L], mu + 1, ieo[L], ibl[L])]);
  }
};

C dot(const C a[4][3], const C b[4][3]) {  // a^+ b
  C s = 0.0;
  for (int d = 0; d < 4; ++d)
    for (int c = 0; c < 3; ++c) s += std::conj(a[d][c]) * b[d][c];
  return s;
}


// loopops at lexicographic site s: the nine operators of y against the noise b.
void site_ops(const AvLattice& L, const double* u, const double* ye, const double* yo, const double* be,
              const double* bo, int s, int ksub, C op[10]) {
  C y[4][3], b[4][3], yn[4][3], bn[4][3], w[4][3], gv[4][3];
  L.spinor(ye, yo, s, y);
  L.spinor(be, bo, s, b);
  for (int mu = 0; mu < 4; ++mu) {
    double f;
    const int sn = L.nb(s, mu, 1, &f);
    L.spinor(ye, yo, sn, yn);
    L.spinor(be, bo, sn, bn);
    // A = f y(x+mu)^+ (1 - gamma_mu) U^+ b(x)
    C ub[4][3];
    for (int d = 0; d < 4; ++d)
      for (int a = 0; a < 3; ++a) {
        C t = 0.0;
        for (int c = 0; c < 3; ++c) t += std::conj(L.link(u, s, mu, c, a)) * b[d][c];
        ub[d][a] = t;
      }
    gamma_mult(mu, ub, gv);
    for (int d = 0; d < 4; ++d)
      for (int a = 0; a < 3; ++a) w[d][a] = ub[d][a] - gv[d][a];
    C A = dot(yn, w) * f;
    // B = - y(x)^+ (1 + gamma_mu) U f b(x+mu)
    for (int d = 0; d < 4; ++d)
      for (int a = 0; a < 3; ++a) {
        C t = 0.0;
        for (int c = 0; c < 3; ++c) t += L.link(u, s, mu, a, c) * (f * bn[d][c]);
        ub[d][a] = t;
      }
    gamma_mult(mu, ub, gv);
    for (int d = 0; d < 4; ++d)
      for (int a = 0; a < 3; ++a) w[d][a] = -(ub[d][a] + gv[d][a]);
    const C B = dot(y, w);
    op[mu] = std::conj(A + B);
  }
  C s5 = dot(y, b);
  if (ksub == 1) s5 += 12.0;
  op[4] = std::conj(s5);
  for (int mu = 0; mu < 4; ++mu) {
    gamma_mult(mu, b, gv);
    op[5 + mu] = std::conj(dot(y, gv));
  }
}

}  // namespace

extern "C" void oq_average(const oq_geom* g, const double* u, const double* be, const double* bo, const double* xe,
                           const double* xo, double kappa, int nsub, int nmom, int nop, const double* momfac,
                           double* Jtime) {
  const AvLattice L(g);
  const int nt = g->n[3], nv = g->nvhalf;
  const size_t nh = (size_t)6 * g->ntotal * 4 * 2 * 8;  // one half vector, reference layout
  std::vector<double> b_e(be, be + nh), b_o(bo, bo + nh);
  std::vector<double> sub1e(nh, 0.0), sub1o(nh, 0.0), sub2e(nh, 0.0), sub2o(nh, 0.0), sube(nh, 0.0),
      subo(nh, 0.0), ye(nh, 0.0), yo(nh, 0.0);
  std::memset(Jtime, 0, sizeof(double) * 2 * nt * nsub * nmom * nop);
  auto J = [&](int ri, int t, int isub, int im, int iop) -> double& {
    return Jtime[((((size_t)iop * nmom + im) * nsub + isub) * nt + t) * 2 + ri];
  };
  auto MF = [&](int Ls, int im, int k) {  // momfac(isite, ieo, ibl, imom-1, k), 1-based k
    return momfac[(((((size_t)(k - 1) * (nmom - 1) + (im - 2)) * 16 + (L.ibl[Ls] - 1)) * 2 + (L.ieo[Ls] - 1)) * nv +
                   (L.isite[Ls] - 1))];
  };
  auto axpy = [&](std::vector<double>& y, double a, const std::vector<double>& x) {
    for (size_t i = 0; i < nh; ++i) y[i] = y[i] + a * x[i];
  };
  auto H = [&](std::vector<double>& out, std::vector<double>& in, int gblclr) {
    oq::hsingle(g, out.data(), u, in.data(), 0, gblclr);
  };
  for (int isub = 1; isub <= nsub; ++isub) {
    int ksub = 1;
    switch (isub) {
      case 1:  // no subtraction
        ksub = 0;
        std::fill(sube.begin(), sube.end(), 0.0);
        std::fill(subo.begin(), subo.end(), 0.0);
        break;
      case 2:  // O(kappa), O(kappa^2), O(kappa^3)
        H(sub1e, b_o, 1);
        H(sub1o, b_e, 2);
        sube = b_e;
        subo = b_o;
        axpy(sube, kappa, sub1e);
        axpy(subo, kappa, sub1o);
        H(sub2e, sub1o, 1);
        H(sub2o, sub1e, 2);
        axpy(sube, kappa * kappa, sub2e);
        axpy(subo, kappa * kappa, sub2o);
        H(sub1e, sub2o, 1);
        H(sub1o, sub2e, 2);
        axpy(sube, kappa * kappa * kappa, sub1e);
        axpy(subo, kappa * kappa * kappa, sub1o);
        break;
      default: {  // O(kappa^(isub+1)): alternate between the two scratch pairs
        const double xk = std::pow(kappa, isub + 1);
        if (isub % 2 == 1) {
          H(sub2e, sub1o, 1);
          H(sub2o, sub1e, 2);
          axpy(sube, xk, sub2e);
          axpy(subo, xk, sub2o);
        } else {
          H(sub1e, sub2o, 1);
          H(sub1o, sub2e, 2);
          axpy(sube, xk, sub1e);
          axpy(subo, xk, sub1o);
        }
        break;
      }
    }
    for (size_t i = 0; i < nh; ++i) {
      ye[i] = xe[i] - sube[i];
      yo[i] = xo[i] - subo[i];
    }
    // loopops per site, then spacesum
    for (int s = 0; s < L.V; ++s) {
      C op[10];
      site_ops(L, u, ye.data(), yo.data(), b_e.data(), b_o.data(), s, ksub, op);
      const int t = s / (L.n[0] * L.n[1] * L.n[2]);
      for (int iop = 0; iop < 9 && iop < nop; ++iop) {
        J(0, t, isub - 1, 0, iop) += op[iop].real();
        J(1, t, isub - 1, 0, iop) += op[iop].imag();
      }
      for (int im = 2; im <= nmom; ++im) {
        J(0, t, isub - 1, im - 1, 0) += MF(s, im, 3) * op[0].imag();
        J(1, t, isub - 1, im - 1, 0) += MF(s, im, 2) * op[0].imag();
        J(0, t, isub - 1, im - 1, 1) += MF(s, im, 1) * op[1].imag();
        J(1, t, isub - 1, im - 1, 1) += MF(s, im, 3) * op[1].imag();
        J(0, t, isub - 1, im - 1, 2) += MF(s, im, 2) * op[2].imag();
        J(1, t, isub - 1, im - 1, 2) += MF(s, im, 1) * op[2].imag();
        J(0, t, isub - 1, im - 1, 3) += MF(s, im, 4) * op[3].real();
        J(1, t, isub - 1, im - 1, 3) += MF(s, im, 4) * op[3].imag();
        J(0, t, isub - 1, im - 1, 4) += MF(s, im, 5) * op[4].real();
        J(1, t, isub - 1, im - 1, 4) += MF(s, im, 5) * op[4].imag();
      }
    }
  }
  for (int iop = 0; iop < 4; ++iop)
    for (int im = 0; im < nmom; ++im)
      for (int isub = 0; isub < nsub; ++isub)
        for (int t = 0; t < nt; ++t)
          for (int ri = 0; ri < 2; ++ri) J(ri, t, isub, im, iop) = kappa * J(ri, t, isub, im, iop);
}

// momfacs, Q/disconloops.f90:8925-8984: the momentum factors spacesum takes,
// momfac(nvhalf, 2, 16, 4, 5) for imom - 1 = 1..4, components 1..3 sine-type along
// x, y, z and 4 cosine-type, component 5 a copy of 4, about the origin io (1-based).
// twoPi is a default-kind literal in the reference, so its value is single precision.
extern "C" void oq_momfacs(const oq_geom* g, const int io[3], double* momfac) {
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2], nt = g->n[3], nv = g->nvhalf;
  const double twoPi = (double)6.283185307179586f;
  auto M = [&](int isite, int ieo, int ibl, int im, int k) -> double& {
    return momfac[((((size_t)(k - 1) * 4 + (im - 1)) * 16 + (ibl - 1)) * 2 + (ieo - 1)) * nv + (isite - 1)];
  };
  for (int it = 1; it <= nt; ++it)
    for (int iz = 1; iz <= nz; ++iz) {
      const double dz = twoPi * (double)(iz - io[2]) / (double)nz;
      for (int iy = 1; iy <= ny; ++iy) {
        const double dy = twoPi * (double)(iy - io[1]) / (double)ny;
        for (int ix = 1; ix <= nx; ++ix) {
          const double dx = twoPi * (double)(ix - io[0]) / (double)nx;
          const int xc[4] = {ix - 1, iy - 1, iz - 1, it - 1};
          int isite, ieo, ibl, gblclr, ibleo;
          oq_site_of_coords(g, xc, &isite, &ieo, &ibl, &gblclr, &ibleo);
          M(isite, ieo, ibl, 1, 1) = std::sin(dx);
          M(isite, ieo, ibl, 1, 2) = std::sin(dy);
          M(isite, ieo, ibl, 1, 3) = std::sin(dz);
          M(isite, ieo, ibl, 1, 4) = (std::cos(dx) + std::cos(dy) + std::cos(dz)) / 3.0;
          M(isite, ieo, ibl, 2, 1) = std::sin(dx) * (std::cos(dy) + std::cos(dz)) / 2.0;
          M(isite, ieo, ibl, 2, 2) = std::sin(dy) * (std::cos(dx) + std::cos(dz)) / 2.0;
          M(isite, ieo, ibl, 2, 3) = std::sin(dz) * (std::cos(dx) + std::cos(dy)) / 2.0;
          M(isite, ieo, ibl, 2, 4) = (std::cos(dx) * std::cos(dy) + std::cos(dx) * std::cos(dz) + std::cos(dy) * std::cos(dz)) / 3.0;
          M(isite, ieo, ibl, 3, 1) = std::sin(dx) * std::cos(dy) * std::cos(dz);
          M(isite, ieo, ibl, 3, 2) = std::sin(dy) * std::cos(dx) * std::cos(dz);
          M(isite, ieo, ibl, 3, 3) = std::sin(dz) * std::cos(dx) * std::cos(dy);
          M(isite, ieo, ibl, 3, 4) = std::cos(dx) * std::cos(dy) * std::cos(dz);
          M(isite, ieo, ibl, 4, 1) = std::sin(2.0 * dx);
          M(isite, ieo, ibl, 4, 2) = std::sin(2.0 * dy);
          M(isite, ieo, ibl, 4, 3) = std::sin(2.0 * dz);
          M(isite, ieo, ibl, 4, 4) = (std::cos(2.0 * dx) + std::cos(2.0 * dy) + std::cos(2.0 * dz)) / 3.0;
          for (int im = 1; im <= 4; ++im) M(isite, ieo, ibl, im, 5) = M(isite, ieo, ibl, im, 4);
        }
      }
    }
}

// The operators of y against b at zero momentum summed per time slice, operators 1..4
// times kappa: J(2, nt, 9) (loopops with ksub, spacesum at imom = 1).
extern "C" void oq_loop_slices(const oq_geom* g, const double* u, const double* be, const double* bo,
                               const double* ye, const double* yo, int ksub, double kappa, double* J) {
  const AvLattice L(g);
  const int nt = g->n[3];
  std::memset(J, 0, sizeof(double) * 2 * nt * 9);
  for (int s = 0; s < L.V; ++s) {
    C op[10];
    site_ops(L, u, ye, yo, be, bo, s, ksub, op);
    const int t = s / (L.n[0] * L.n[1] * L.n[2]);
    for (int iop = 0; iop < 9; ++iop) {
      J[((size_t)iop * nt + t) * 2] += op[iop].real();
      J[((size_t)iop * nt + t) * 2 + 1] += op[iop].imag();
    }
  }
  for (int iop = 0; iop < 4; ++iop)
    for (int k = 0; k < 2 * nt; ++k) J[(size_t)iop * 2 * nt + k] *= kappa;
}
