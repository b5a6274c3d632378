// CPU oracle (test infrastructure): level-0 (unsubtracted) disconnected-loop traces of
// one noise vector, restating
//   * twAverage, Q/vevbleft.f90:2541-4704, with nsub = 0 and zero momentum (imom = 1):
//     the per-site loop :4011-4503 (z2 / z2sub set from the noise at :4012-4013,
//     the isb = 0 propagator combinations sprop / pscalar at :4139-4143 and :4226-4229,
//     the accumulation into opertemp at :4381-4432) and the copy into Jvev at :4519-4535;
//   * currentCalc2P, Q/vevbleft.f90:10863-11247 (the r = +1 branch of currentCalc2,
//     :10832-10859): point-split currents, with dobndry = 1 skipping the time current
//     across the t boundary (:10932-10966) and zeroing the last time slice of links
//     (twAverage :2912-2926);
//   * scalarCalc, Q/vevbleft.f90:9261-9299: psibar psi and psibar gamma5 psi;
//   * changenoise / changevector / utouss (:13166, :12989, :12854): the noise's real
//     part, the propagator and the links gathered to lexicographic order;
//   * the caller's kappa scaling of every operator but 2 and 6
//     (Q/disconloops.f90:4045-4049).  The division by the number of noises and by
//     nx*ny*nz (:4161-4164) is left to the caller, as in the reference.
// Output J(2, nt, 6), Fortran order: J[(iop * nt + t) * 2 + ri]; op 1 = J4 point-split
// time current, 2 = psibar psi, 3..5 = J1..J3 point-split spatial currents,
// 6 = psibar gamma5 psi.  Arithmetic follows the reference's expression order.
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle_impl.h"

namespace {

struct Lex {
  int nx, ny, nz, nt;
  int site(int x, int y, int z, int t) const { return x + nx * (y + ny * (z + nz * t)); }
};

}  // namespace

extern "C" void oq_twaverage_mom(const oq_geom* g, const double* be, const double* bo, const double* xe,
                                 const double* xo, const double* u, double kappa, double delta, const int io[3],
                                 int dobndry, int nmom, int ir, double* J);

extern "C" void oq_twaverage_level0(const oq_geom* g, const double* be, const double* bo,
                                    const double* xe, const double* xo, const double* u,
                                    double kappa, double delta, int dobndry, double* J) {
  const int io[3] = {1, 1, 1};
  oq_twaverage_mom(g, be, bo, xe, xo, u, kappa, delta, io, dobndry, 1, 1, J);
}

// The same traces with twAverage's momentum projections (:4434-4503) and either Wilson r
// (currentCalc2, :10832-10859): imom 2..5 weight
// rho, psibar psi and psibar gamma5 psi by ffac and the imaginary parts of the
// currents by fas1..3 at the site each value sits on; J(2, nt, nmom, 6).
extern "C" void oq_twaverage_mom(const oq_geom* g, const double* be, const double* bo, const double* xe,
                                 const double* xo, const double* u, double kappa, double delta, const int io[3],
                                 int dobndry, int nmom, int ir, double* J) {
  // Wilson r = +-1: currentCalc2P / currentCalc2M (:10863-11635) differ by the sign of
  // the diagonal (Wilson) terms and by the spins and sign of the time current
  const double rs = ir, tf = 2.0 * ir;
  const Lex L{g->n[0], g->n[1], g->n[2], g->n[3]};
  const int V = L.nx * L.ny * L.nz * L.nt;
  // lexicographic gathers: [site][colour][spin] (spin, colour 0-based)
  std::vector<double> Pr((size_t)V * 12), Pi((size_t)V * 12), Er((size_t)V * 12);
  // links U_mu(site)[a][b], re/im: [site][mu][ri][a][b]
  std::vector<double> U((size_t)V * 4 * 2 * 9);
  auto E = [&](int s, int c, int d) { return Er[((size_t)s * 3 + c) * 4 + d]; };
  auto Ul = [&](int s, int mu, int ri, int a, int b) -> double& {
    return U[(((size_t)s * 4 + mu) * 2 + ri) * 9 + 3 * a + b];
  };
  for (int t = 0; t < L.nt; ++t)
    for (int z = 0; z < L.nz; ++z)
      for (int y = 0; y < L.ny; ++y)
        for (int x = 0; x < L.nx; ++x) {
          const int xc[4] = {x, y, z, t};
          int isite, ieo, ibl, gblclr, ibleo;
          oq_site_of_coords(g, xc, &isite, &ieo, &ibl, &gblclr, &ibleo);
          const double* hx = gblclr == 1 ? xe : xo;
          const double* hb = gblclr == 1 ? be : bo;
          const int s = L.site(x, y, z, t);
          for (int c = 0; c < 3; ++c)
            for (int d = 0; d < 4; ++d) {
              const size_t k = ((size_t)s * 3 + c) * 4 + d;
              Pr[k] = hx[g->gi(2 * c + 1, isite, d + 1, ieo, ibleo)];
              Pi[k] = hx[g->gi(2 * c + 2, isite, d + 1, ieo, ibleo)];
              Er[k] = hb[g->gi(2 * c + 1, isite, d + 1, ieo, ibleo)];
            }
          for (int mu = 0; mu < 4; ++mu)
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) {
                Ul(s, mu, 0, a, b) = u[g->ui(2 * (3 * a + b) + 1, isite, mu + 1, ieo, ibl)];
                Ul(s, mu, 1, a, b) = u[g->ui(2 * (3 * a + b) + 2, isite, mu + 1, ieo, ibl)];
              }
        }
  const bool fixbc = dobndry == 1;
  if (fixbc)  // usp = 0 on the last time slice
    for (int z = 0; z < L.nz; ++z)
      for (int y = 0; y < L.ny; ++y)
        for (int x = 0; x < L.nx; ++x)
          for (int ri = 0; ri < 2; ++ri)
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) Ul(L.site(x, y, z, L.nt - 1), 3, ri, a, b) = 0.0;

  const double cosd = std::cos(delta), sind = std::sin(delta);
  const int cd[4] = {2, 3, 0, 1};
  const double sgn[4] = {1.0, 1.0, -1.0, -1.0};
  std::vector<double> op((size_t)12 * L.nt * 5, 0.0);
  auto OPm = [&](int k, int t, int ix) -> double& { return op[((size_t)ix * 12 + k) * L.nt + t]; };
  auto OP = [&](int k, int t) -> double& { return OPm(k, t, 0); };
  std::vector<double> ffac, fas1, fas2, fas3;  // [site][k 0..3]
  oq_momentum_factors(g->n, io, ffac, fas1, fas2, fas3);
  auto F = [&](const std::vector<double>& f, int site, int k) { return f[(size_t)site * 4 + k]; };

  for (int t = 0; t < L.nt; ++t)
    for (int z = 0; z < L.nz; ++z)
      for (int y = 0; y < L.ny; ++y)
        for (int x = 0; x < L.nx; ++x) {
          const int h = L.site(x, y, z, t);
          const int lx = L.site((x + L.nx - 1) % L.nx, y, z, t), rx = L.site((x + 1) % L.nx, y, z, t);
          const int ly = L.site(x, (y + L.ny - 1) % L.ny, z, t), ry = L.site(x, (y + 1) % L.ny, z, t);
          const int lz = L.site(x, y, (z + L.nz - 1) % L.nz, t), rz = L.site(x, y, (z + 1) % L.nz, t);
          const int lt = L.site(x, y, z, (t + L.nt - 1) % L.nt), rt = L.site(x, y, z, (t + 1) % L.nt);
          const int tm1 = (t + L.nt - 1) % L.nt;
          for (int d = 0; d < 4; ++d)
            for (int c = 0; c < 3; ++c) {
              const double z2 = E(h, c, d);         // z2(ihere, icolor, idirac)
              const double z2sub = E(h, c, cd[d]);  // z2sub(ihere, icolor, cd(idirac))
              const size_t k = ((size_t)h * 3 + c) * 4;
              for (int jri = 1; jri <= 2; ++jri) {
                double s, ps;
                if (jri == 1) {
                  s = Pr[k + d] - cosd * (cosd * z2 - sgn[d] * sind * z2sub);
                  ps = sgn[d] * Pi[k + cd[d]];
                } else {
                  s = Pi[k + d];
                  ps = -sgn[d] * (Pr[k + cd[d]] - cosd * (cosd * z2sub - sgn[cd[d]] * sind * z2));
                }
                // currentCalc2P: values at ahere and at its left neighbours, zeroed per call
                double rhor_h = 0, rhoi_h = 0, rhor_l = 0, rhoi_l = 0;
                double j1r_h = 0, j1i_h = 0, j1r_l = 0, j1i_l = 0;
                double j2r_h = 0, j2i_h = 0, j2r_l = 0, j2i_l = 0;
                double j3r_h = 0, j3i_h = 0, j3r_l = 0, j3i_l = 0;
                const int jd = d + 1;  // 1-based spin index of the reference
                const int od = 5 - jd - 1, o3 = (jd % 2 == 1 ? 3 / jd : 8 / jd) - 1;
                for (int jc = 0; jc < 3; ++jc) {
                  // point-split J4: r = 1 takes spins 1,2 at ahere and 3,4 at leftt
                  // (currentCalc2P); r = -1 the reverse, with the opposite sign (currentCalc2M)
                  const bool hset = ir == 1 ? (jd == 1 || jd == 2) : (jd == 3 || jd == 4);
                  if (hset && (!fixbc || t != L.nt - 1)) {
                    if (jri == 1) {
                      rhor_h = rhor_h + tf * s * Ul(h, 3, 0, c, jc) * E(rt, jc, d);
                      rhoi_h = rhoi_h - tf * s * Ul(h, 3, 1, c, jc) * E(rt, jc, d);
                    } else {
                      rhor_h = rhor_h + tf * s * Ul(h, 3, 1, c, jc) * E(rt, jc, d);
                      rhoi_h = rhoi_h + tf * s * Ul(h, 3, 0, c, jc) * E(rt, jc, d);
                    }
                  } else if (!hset && (!fixbc || t != 0)) {
                    if (jri == 1) {
                      rhor_l = rhor_l - tf * s * Ul(lt, 3, 0, jc, c) * E(lt, jc, d);
                      rhoi_l = rhoi_l - tf * s * Ul(lt, 3, 1, jc, c) * E(lt, jc, d);
                    } else {
                      rhor_l = rhor_l + tf * s * Ul(lt, 3, 1, jc, c) * E(lt, jc, d);
                      rhoi_l = rhoi_l - tf * s * Ul(lt, 3, 0, jc, c) * E(lt, jc, d);
                    }
                  }
                  // point-split J1
                  if (jri == 1) {
                    j1r_l = j1r_l - rs * s * Ul(lx, 0, 0, jc, c) * E(lx, jc, d) + s * Ul(lx, 0, 0, jc, c) * E(lx, jc, od);
                    j1i_l = j1i_l - rs * s * Ul(lx, 0, 1, jc, c) * E(lx, jc, d) + s * Ul(lx, 0, 1, jc, c) * E(lx, jc, od);
                    j1r_h = j1r_h + rs * s * Ul(h, 0, 0, c, jc) * E(rx, jc, d) + s * Ul(h, 0, 0, c, jc) * E(rx, jc, od);
                    j1i_h = j1i_h - rs * s * Ul(h, 0, 1, c, jc) * E(rx, jc, d) - s * Ul(h, 0, 1, c, jc) * E(rx, jc, od);
                  } else {
                    j1r_l = j1r_l + rs * s * Ul(lx, 0, 1, jc, c) * E(lx, jc, d) - s * Ul(lx, 0, 1, jc, c) * E(lx, jc, od);
                    j1i_l = j1i_l - rs * s * Ul(lx, 0, 0, jc, c) * E(lx, jc, d) + s * Ul(lx, 0, 0, jc, c) * E(lx, jc, od);
                    j1r_h = j1r_h + rs * s * Ul(h, 0, 1, c, jc) * E(rx, jc, d) + s * Ul(h, 0, 1, c, jc) * E(rx, jc, od);
                    j1i_h = j1i_h + rs * s * Ul(h, 0, 0, c, jc) * E(rx, jc, d) + s * Ul(h, 0, 0, c, jc) * E(rx, jc, od);
                  }
                  // point-split J2, diagonal part
                  if (jri == 1) {
                    j2r_l = j2r_l - rs * s * Ul(ly, 1, 0, jc, c) * E(ly, jc, d);
                    j2i_l = j2i_l - rs * s * Ul(ly, 1, 1, jc, c) * E(ly, jc, d);
                    j2r_h = j2r_h + rs * s * Ul(h, 1, 0, c, jc) * E(ry, jc, d);
                    j2i_h = j2i_h - rs * s * Ul(h, 1, 1, c, jc) * E(ry, jc, d);
                  } else {
                    j2r_l = j2r_l + rs * s * Ul(ly, 1, 1, jc, c) * E(ly, jc, d);
                    j2i_l = j2i_l - rs * s * Ul(ly, 1, 0, jc, c) * E(ly, jc, d);
                    j2r_h = j2r_h + rs * s * Ul(h, 1, 1, c, jc) * E(ry, jc, d);
                    j2i_h = j2i_h + rs * s * Ul(h, 1, 0, c, jc) * E(ry, jc, d);
                  }
                  // J2, off-diagonal part
                  if (jd % 2 == 1) {
                    if (jri == 1) {
                      j2r_l = j2r_l - s * Ul(ly, 1, 1, jc, c) * E(ly, jc, od);
                      j2i_l = j2i_l + s * Ul(ly, 1, 0, jc, c) * E(ly, jc, od);
                      j2r_h = j2r_h + s * Ul(h, 1, 1, c, jc) * E(ry, jc, od);
                      j2i_h = j2i_h + s * Ul(h, 1, 0, c, jc) * E(ry, jc, od);
                    } else {
                      j2r_l = j2r_l - s * Ul(ly, 1, 0, jc, c) * E(ly, jc, od);
                      j2i_l = j2i_l - s * Ul(ly, 1, 1, jc, c) * E(ly, jc, od);
                      j2r_h = j2r_h - s * Ul(h, 1, 0, c, jc) * E(ry, jc, od);
                      j2i_h = j2i_h + s * Ul(h, 1, 1, c, jc) * E(ry, jc, od);
                    }
                  } else {
                    if (jri == 1) {
                      j2r_l = j2r_l + s * Ul(ly, 1, 1, jc, c) * E(ly, jc, od);
                      j2i_l = j2i_l - s * Ul(ly, 1, 0, jc, c) * E(ly, jc, od);
                      j2r_h = j2r_h - s * Ul(h, 1, 1, c, jc) * E(ry, jc, od);
                      j2i_h = j2i_h - s * Ul(h, 1, 0, c, jc) * E(ry, jc, od);
                    } else {
                      j2r_l = j2r_l + s * Ul(ly, 1, 0, jc, c) * E(ly, jc, od);
                      j2i_l = j2i_l + s * Ul(ly, 1, 1, jc, c) * E(ly, jc, od);
                      j2r_h = j2r_h + s * Ul(h, 1, 0, c, jc) * E(ry, jc, od);
                      j2i_h = j2i_h - s * Ul(h, 1, 1, c, jc) * E(ry, jc, od);
                    }
                  }
                  // point-split J3, diagonal part
                  if (jri == 1) {
                    j3r_l = j3r_l - rs * s * Ul(lz, 2, 0, jc, c) * E(lz, jc, d);
                    j3i_l = j3i_l - rs * s * Ul(lz, 2, 1, jc, c) * E(lz, jc, d);
                    j3r_h = j3r_h + rs * s * Ul(h, 2, 0, c, jc) * E(rz, jc, d);
                    j3i_h = j3i_h - rs * s * Ul(h, 2, 1, c, jc) * E(rz, jc, d);
                  } else {
                    j3r_l = j3r_l + rs * s * Ul(lz, 2, 1, jc, c) * E(lz, jc, d);
                    j3i_l = j3i_l - rs * s * Ul(lz, 2, 0, jc, c) * E(lz, jc, d);
                    j3r_h = j3r_h + rs * s * Ul(h, 2, 1, c, jc) * E(rz, jc, d);
                    j3i_h = j3i_h + rs * s * Ul(h, 2, 0, c, jc) * E(rz, jc, d);
                  }
                  // J3, off-diagonal part
                  if (jd % 2 == 1) {
                    if (jri == 1) {
                      j3r_l = j3r_l + s * Ul(lz, 2, 0, jc, c) * E(lz, jc, o3);
                      j3i_l = j3i_l + s * Ul(lz, 2, 1, jc, c) * E(lz, jc, o3);
                      j3r_h = j3r_h + s * Ul(h, 2, 0, c, jc) * E(rz, jc, o3);
                      j3i_h = j3i_h - s * Ul(h, 2, 1, c, jc) * E(rz, jc, o3);
                    } else {
                      j3r_l = j3r_l - s * Ul(lz, 2, 1, jc, c) * E(lz, jc, o3);
                      j3i_l = j3i_l + s * Ul(lz, 2, 0, jc, c) * E(lz, jc, o3);
                      j3r_h = j3r_h + s * Ul(h, 2, 1, c, jc) * E(rz, jc, o3);
                      j3i_h = j3i_h + s * Ul(h, 2, 0, c, jc) * E(rz, jc, o3);
                    }
                  } else {
                    if (jri == 1) {
                      j3r_l = j3r_l - s * Ul(lz, 2, 0, jc, c) * E(lz, jc, o3);
                      j3i_l = j3i_l - s * Ul(lz, 2, 1, jc, c) * E(lz, jc, o3);
                      j3r_h = j3r_h - s * Ul(h, 2, 0, c, jc) * E(rz, jc, o3);
                      j3i_h = j3i_h + s * Ul(h, 2, 1, c, jc) * E(rz, jc, o3);
                    } else {
                      j3r_l = j3r_l + s * Ul(lz, 2, 1, jc, c) * E(lz, jc, o3);
                      j3i_l = j3i_l - s * Ul(lz, 2, 0, jc, c) * E(lz, jc, o3);
                      j3r_h = j3r_h - s * Ul(h, 2, 1, c, jc) * E(rz, jc, o3);
                      j3i_h = j3i_h - s * Ul(h, 2, 0, c, jc) * E(rz, jc, o3);
                    }
                  }
                }
                // scalarCalc: psi = value * z2, real slot for jri = 1, imaginary for 2
                const double psir = jri == 1 ? s * z2 : 0.0, psii = jri == 2 ? s * z2 : 0.0;
                const double psur = jri == 1 ? ps * z2 : 0.0, psui = jri == 2 ? ps * z2 : 0.0;
                OP(0, t) += rhor_h;
                OP(0, tm1) += rhor_l;
                OP(1, t) += rhoi_h;
                OP(1, tm1) += rhoi_l;
                OP(2, t) += psir;
                OP(3, t) += psii;
                OP(4, t) = OP(4, t) + j1r_h + j1r_l;
                OP(5, t) = OP(5, t) + j1i_h + j1i_l;
                OP(6, t) = OP(6, t) + j2r_h + j2r_l;
                OP(7, t) = OP(7, t) + j2i_h + j2i_l;
                OP(8, t) = OP(8, t) + j3r_h + j3r_l;
                OP(9, t) = OP(9, t) + j3i_h + j3i_l;
                OP(10, t) += psur;
                OP(11, t) += psui;
                for (int ix = 1; ix < 5; ++ix) {
                  const int k = ix - 1;
                  const double ff = F(ffac, h, k);
                  OPm(0, t, ix) += rhor_h * ff;
                  OPm(0, tm1, ix) += rhor_l * F(ffac, lt, k);
                  OPm(1, t, ix) += rhoi_h * ff;
                  OPm(1, tm1, ix) += rhoi_l * F(ffac, lt, k);
                  OPm(2, t, ix) += psir * ff;
                  OPm(3, t, ix) += psii * ff;
                  OPm(4, t, ix) = OPm(4, t, ix) + j1i_h * F(fas3, h, k) + j1i_l * F(fas3, lx, k);
                  OPm(5, t, ix) = OPm(5, t, ix) + j2i_h * F(fas1, h, k) + j2i_l * F(fas1, ly, k);
                  OPm(6, t, ix) = OPm(6, t, ix) + j3i_h * F(fas2, h, k) + j3i_l * F(fas2, lz, k);
                  OPm(7, t, ix) = OPm(7, t, ix) + j1i_h * F(fas2, h, k) + j1i_l * F(fas2, lx, k);
                  OPm(8, t, ix) = OPm(8, t, ix) + j2i_h * F(fas3, h, k) + j2i_l * F(fas3, ly, k);
                  OPm(9, t, ix) = OPm(9, t, ix) + j3i_h * F(fas1, h, k) + j3i_l * F(fas1, lz, k);
                  OPm(10, t, ix) += psur * ff;
                  OPm(11, t, ix) += psui * ff;
                }
              }
            }
        }
  for (int iop = 0; iop < 6; ++iop) {
    const double f = (iop == 1 || iop == 5) ? 1.0 : kappa;  // ops 2 and 6 unscaled
    for (int im = 0; im < nmom; ++im)
      for (int t = 0; t < L.nt; ++t)
        for (int ri = 0; ri < 2; ++ri) {
          const double v = OPm(2 * iop + ri, t, im);
          J[(((size_t)iop * nmom + im) * L.nt + t) * 2 + ri] = f == 1.0 ? v : f * v;
        }
  }
}
