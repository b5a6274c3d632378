// Internal helpers of the CPU oracle (test infrastructure only; see oracle.h).
#pragma once
#include <cstddef>
#include <cmath>
#include <vector>

#include "oracle.h"

// The timing build of the oracle (liboracle_omp.so, -fopenmp) splits the site loops over
// the host threads; the default build ignores these and runs in the reference's serial
// order.  Only loops whose iterations touch disjoint entries (or reduce into OQ_SUM)
// are split, so the arithmetic per entry is the reference's.
#ifdef _OPENMP
#define OQ_PAR_FOR _Pragma("omp parallel for schedule(static)")
#define OQ_PAR_FOR2 _Pragma("omp parallel for collapse(2) schedule(static)")
#define OQ_PAR_FOR3 _Pragma("omp parallel for collapse(3) schedule(static)")
#define OQ_PAR_SUM3 _Pragma("omp parallel for collapse(3) schedule(static) reduction(+ : re, im)")
#else
#define OQ_PAR_FOR
#define OQ_PAR_FOR2
#define OQ_PAR_FOR3
#define OQ_PAR_SUM3
#endif

struct oq_geom {
  int n[4];
  int bc[4];
  double c1[4], c2[4];  // coact(3,1,mu), coact(3,2,mu)
  int nvhalf, nbmax, ntotal;
  int nms[4];
  std::vector<int> lv, lvbc;  // (nvhalf, 4, 2), 1-based values
  std::vector<int> ib;        // (nbmax, 4, 2, 2)
  bool lbd[16][4];
  int iblv[16][4];
  int vecbl[2][8];
  int vecblinv[2][16];

  // Index of g(a, site, id, ieo, ibleo) (all 1-based) in a (6,ntotal,4,2,8) array.
  size_t gi(int a, int site, int id, int ieo, int ibleo) const {
    return (size_t)(a - 1) +
           6 * ((size_t)(site - 1) +
                (size_t)ntotal * ((size_t)(id - 1) + 4 * ((size_t)(ieo - 1) + 2 * (size_t)(ibleo - 1))));
  }
  // Index of u(a, site, mu, ieo, ibl) in a (18,ntotal,4,2,16) array.
  size_t ui(int a, int site, int mu, int ieo, int ibl) const {
    return (size_t)(a - 1) +
           18 * ((size_t)(site - 1) +
                 (size_t)ntotal * ((size_t)(mu - 1) + 4 * ((size_t)(ieo - 1) + 2 * (size_t)(ibl - 1))));
  }
  size_t vsize() const { return (size_t)6 * ntotal * 4 * 2 * 8; }
  size_t usize() const { return (size_t)18 * ntotal * 4 * 2 * 16; }
  int& LV(int i, int mu, int ieo) { return lv[(size_t)(i - 1) + (size_t)nvhalf * ((mu - 1) + 4 * (ieo - 1))]; }
  int& LVBC(int i, int mu, int ieo) { return lvbc[(size_t)(i - 1) + (size_t)nvhalf * ((mu - 1) + 4 * (ieo - 1))]; }
  const int& LVBC(int i, int mu, int ieo) const {
    return lvbc[(size_t)(i - 1) + (size_t)nvhalf * ((mu - 1) + 4 * (ieo - 1))];
  }
  int& IB(int i, int mu, int side, int ieo) {
    return ib[(size_t)(i - 1) + (size_t)nbmax * ((mu - 1) + 4 * ((side - 1) + 2 * (ieo - 1)))];
  }
  int IB(int i, int mu, int side, int ieo) const {
    return ib[(size_t)(i - 1) + (size_t)nbmax * ((mu - 1) + 4 * ((side - 1) + 2 * (ieo - 1)))];
  }

  // f(k) for every real entry with isite <= nvhalf.
  template <class F>
  void for_interior(F f) const {
    OQ_PAR_FOR3
    for (int ibleo = 1; ibleo <= 8; ++ibleo)
      for (int ieo = 1; ieo <= 2; ++ieo)
        for (int id = 1; id <= 4; ++id)
          for (int s = 1; s <= nvhalf; ++s)
            for (int a = 1; a <= 6; ++a) f(gi(a, s, id, ieo, ibleo));
  }
  // f(s1,s2,s3,s4): offsets of the same (a, site, ieo, ibleo) entry for spins 1..4.
  // complex_stride: visit a = 1,3,5 only (f handles re and im).
  template <class F>
  void for_spin_range(F f, int smax, bool complex_stride) const {
    OQ_PAR_FOR3
    for (int ibleo = 1; ibleo <= 8; ++ibleo)
      for (int ieo = 1; ieo <= 2; ++ieo)
        for (int s = 1; s <= smax; ++s)
          for (int a = 1; a <= 6; a += complex_stride ? 2 : 1)
            f(gi(a, s, 1, ieo, ibleo), gi(a, s, 2, ieo, ibleo), gi(a, s, 3, ieo, ibleo),
              gi(a, s, 4, ieo, ibleo));
  }
  template <class F>
  void for_spin_interior(F f, bool complex_stride = false) const {
    for_spin_range(f, nvhalf, complex_stride);
  }
  template <class F>
  void for_spin_all(F f) const {
    for_spin_range(f, ntotal, false);
  }
};

struct oq_defl {
  int nmax, kmax;
  int k;                       // deflation vectors held: k+1 in vtemp
  std::vector<double> vtemp;   // (kmax+1) vectors of g->vsize()
  std::vector<double> hcnew;   // (2, nmax+1, nmax) Fortran order
  std::vector<double> beg;     // one vector
  size_t vsize;
};

namespace oq {
void hsingle(const oq_geom* g, double* gout, const double* u, double* gin, int idag,
             int gblclr);
void hdouble(const oq_geom* g, double* he, const double* u, double* ge, int idag,
             double kappa);
void hdbletm(const oq_geom* g, double* he, const double* u, double* ge, int idag,
             const double kappa[2]);
void gamma5mult(const oq_geom* g, double* he, const double* u, double* ge, int idag,
                const double kappa[2]);
double vecdot_re(const oq_geom* g, const double* a, const double* b, double* im);
double twonorm_c(const double* x, int n);
}  // namespace oq

// Momentum factors of the loop operators (Q/vevbleft.f90:955-985 and twAverage's copy):
// per lexicographic site (t outermost) and k = 0..3 (imom 2..5), origin io (1-based).
inline void oq_momentum_factors(const int n[4], const int io[3], std::vector<double>& ffac,
                                std::vector<double>& fas1, std::vector<double>& fas2,
                                std::vector<double>& fas3) {
  const int nx = n[0], ny = n[1], nz = n[2], nt = n[3];
  const size_t V = (size_t)nx * ny * nz * nt;
  ffac.assign(V * 4, 0.0);
  fas1.assign(V * 4, 0.0);
  fas2.assign(V * 4, 0.0);
  fas3.assign(V * 4, 0.0);
  const double p1 = 8.0 * std::atan(1.0) / nx, p2 = 8.0 * std::atan(1.0) / ny, p3 = 8.0 * std::atan(1.0) / nz;
  for (int t = 0; t < nt; ++t)
    for (int z = 0; z < nz; ++z) {
      const double dz = (double)(z + 1 - io[2]) * p3;
      for (int y = 0; y < ny; ++y) {
        const double dy = (double)(y + 1 - io[1]) * p2;
        for (int x = 0; x < nx; ++x) {
          const double dx = (double)(x + 1 - io[0]) * p1;
          const size_t s = (size_t)(x + nx * (y + ny * (z + (size_t)nz * t))) * 4;
          ffac[s + 0] = (std::cos(dx) + std::cos(dy) + std::cos(dz)) / 3.0;
          fas1[s + 0] = std::sin(dx);
          fas2[s + 0] = std::sin(dy);
          fas3[s + 0] = std::sin(dz);
          ffac[s + 1] = (std::cos(dx) * std::cos(dy) + std::cos(dx) * std::cos(dz) + std::cos(dy) * std::cos(dz)) / 3.0;
          fas1[s + 1] = std::sin(dx) * (std::cos(dy) + std::cos(dz)) / 2.0;
          fas2[s + 1] = std::sin(dy) * (std::cos(dx) + std::cos(dz)) / 2.0;
          fas3[s + 1] = std::sin(dz) * (std::cos(dx) + std::cos(dy)) / 2.0;
          ffac[s + 2] = std::cos(dx) * std::cos(dy) * std::cos(dz);
          fas1[s + 2] = std::sin(dx) * std::cos(dy) * std::cos(dz);
          fas2[s + 2] = std::sin(dy) * std::cos(dx) * std::cos(dz);
          fas3[s + 2] = std::sin(dz) * std::cos(dx) * std::cos(dy);
          ffac[s + 3] = (std::cos(2.0 * dx) + std::cos(2.0 * dy) + std::cos(2.0 * dz)) / 3.0;
          fas1[s + 3] = std::sin(2.0 * dx);
          fas2[s + 3] = std::sin(2.0 * dy);
          fas3[s + 3] = std::sin(2.0 * dz);
        }
      }
    }
}
