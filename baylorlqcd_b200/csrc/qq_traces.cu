// Level-0 (unsubtracted) disconnected-loop traces of one noise vector on the GPU: the
// operators twAverage accumulates at nsub = 0 and zero momentum (Q/vevbleft.f90
// :2541-4704 with currentCalc2P :10863-11247 and scalarCalc :9261-9299), with the
// caller's kappa scaling (Q/disconloops.f90:4045-4049).
//
// The reference scatters every propagator entry through hand-unrolled sign tables;
// those sums are, per site y and direction mu, the bilinears
//   J_mu(y) = eta(y+mu)^T (1+gamma_mu) U_mu(y)^+ x'(y) - eta(y)^T (1-gamma_mu) U_mu(y) x'(y+mu)
//   psibar psi (y) = eta(y)^T x'(y),   psibar gamma5 psi (y) = eta(y)^T gamma5 x'(y)
// with eta the real part of the noise (twAverage uses only that), x the solution and
// x' = x - cos(delta) (cos(delta) - sin(delta) i gamma5) eta (the noise subtraction
// of :4139-4143 and :4226-4229), periodic neighbours without the boundary sign, and
// the time current of the last slice dropped when dobndry = 1.  One thread per
// lexicographic site evaluates them straight from the reference-layout noise and
// solution and the context's links; a second kernel sums each time slice in a fixed
// order, so results are deterministic.  The test suite checks these closed forms
// against a literal CPU restatement of the reference's loops.
#include <cmath>
#include <cstring>
#include <vector>

#include "qq_ctx.h"

namespace qq {
namespace {

constexpr int kTraceVals = 12;  // 6 complex operators per site, in output order

struct Spin12 {
  cplx<double> v[4][3];  // [spin][colour]
};

// (gamma_mu v)_d = ph[mu][d] v_{pm[mu][d]} in the reference basis (Q/diracops.f90:61-71)
__device__ __constant__ int kGamPerm[4][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}, {0, 1, 2, 3}};
__device__ __constant__ double kGamRe[4][4] = {{1, 1, 1, 1}, {0, 0, 0, 0}, {1, -1, 1, -1}, {1, 1, -1, -1}};
__device__ __constant__ double kGamIm[4][4] = {{0, 0, 0, 0}, {-1, 1, -1, 1}, {0, 0, 0, 0}, {0, 0, 0, 0}};

__device__ inline void ref_index(const Geom& g, const int* x, int* isite, int* ieo, int* ibleo) {
  ref_site(g, x, isite, ieo, ibleo);
}

// Noise real part and x' at site x (coordinates), from the reference layout.
__device__ inline void load_site(const Geom& g, const RefDims& rd, const double* be, const double* bo,
                                 const double* xe, const double* xo, const int* x, double cosd,
                                 double sind, double eta[4][3], Spin12& xp) {
  int isite, ieo, ibleo;
  ref_index(g, x, &isite, &ieo, &ibleo);
  const bool even = ((x[0] + x[1] + x[2] + x[3]) & 1) == 0;
  const double* hb = even ? be : bo;
  const double* hx = even ? xe : xo;
#pragma unroll
  for (int d = 0; d < 4; ++d)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t k = ref_gi(rd, 2 * c + 1, isite, d + 1, ieo, ibleo);
      eta[d][c] = hb[k];
      xp.v[d][c] = {hx[k], hx[k + 1]};
    }
  // x' = x - cos^2 eta + cos sin (J eta), (J v)_d = sgn(d) v_{cd(d)}
  const double c2 = cosd * cosd, cs = cosd * sind;
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const int e = d ^ 2;
    const double sg = d < 2 ? 1.0 : -1.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) xp.v[d][c].re += -c2 * eta[d][c] + cs * sg * eta[e][c];
  }
}

// sum_{d,c} eta_d,c [ (r + s gamma_mu) w ]_d,c  (Wilson r = +-1)
__device__ inline cplx<double> proj_dot(const double eta[4][3], int mu, double r, double s,
                                        const cplx<double> w[4][3]) {
  cplx<double> acc{0.0, 0.0};
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const int e = kGamPerm[mu][d];
    const double pr = s * kGamRe[mu][d], pi = s * kGamIm[mu][d];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const cplx<double> gw{pr * w[e][c].re - pi * w[e][c].im, pr * w[e][c].im + pi * w[e][c].re};
      acc.re += eta[d][c] * (r * w[d][c].re + gw.re);
      acc.im += eta[d][c] * (r * w[d][c].im + gw.im);
    }
  }
  return acc;
}

template <int RECON>
__global__ void __launch_bounds__(128) trace_sites_kernel(Geom g, RefDims rd, const double* be,
                                                          const double* bo, const double* xe,
                                                          const double* xo, const void* gauge,
                                                          double kappa, double r, double cosd, double sind,
                                                          int dobndry, double* val) {
  const int V = 2 * g.vh;
  const int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= V) return;
  int x[4];
  {
    int r = L;
    x[0] = r % g.n[0];
    r /= g.n[0];
    x[1] = r % g.n[1];
    r /= g.n[1];
    x[2] = r % g.n[2];
    x[3] = r / g.n[2];
  }
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1, s = L >> 1;
  double eta[4][3];
  Spin12 xp;
  load_site(g, rd, be, bo, xe, xo, x, cosd, sind, eta, xp);
  double out[kTraceVals];
  // psibar psi and psibar gamma5 psi: (gamma5 v)_d = -i sgn(d) v_{cd(d)}
  cplx<double> sc{0.0, 0.0}, ps{0.0, 0.0};
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const double sg = d < 2 ? 1.0 : -1.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      sc.re += eta[d][c] * xp.v[d][c].re;
      sc.im += eta[d][c] * xp.v[d][c].im;
      const cplx<double> v = xp.v[d ^ 2][c];  // -i sg v = sg (v.im, -v.re)
      ps.re += eta[d][c] * (sg * v.im);
      ps.im += eta[d][c] * (-sg * v.re);
    }
  }
  out[2] = sc.re;
  out[3] = sc.im;
  out[10] = ps.re;
  out[11] = ps.im;
  const int slot[4] = {4, 6, 8, 0};  // J1, J2, J3, J4
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    cplx<double> jm{0.0, 0.0};
    if (!(mu == 3 && dobndry == 1 && x[3] == g.n[3] - 1)) {
      int y[4] = {x[0], x[1], x[2], x[3]};
      y[mu] = y[mu] + 1 == g.n[mu] ? 0 : y[mu] + 1;
      double etaf[4][3];
      Spin12 xpf;
      load_site(g, rd, be, bo, xe, xo, y, cosd, sind, etaf, xpf);
      Su3<double> u;
      LinkIO<P64, RECON>::load(gauge, g.vh, p, mu, s, u);
      cplx<double> w[4][3];
      // a = eta(y+mu)^T (1 + gamma_mu) U^+ x'(y)
#pragma unroll
      for (int d = 0; d < 4; ++d)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          cplx<double> t{0.0, 0.0};
#pragma unroll
          for (int b = 0; b < 3; ++b) t = cadd(t, cmulconj(u.e[b][a], xp.v[d][b]));
          w[d][a] = t;
        }
      const cplx<double> av = proj_dot(etaf, mu, r, 1.0, w);
      // b = eta(y)^T (1 - gamma_mu) U x'(y+mu)
#pragma unroll
      for (int d = 0; d < 4; ++d)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          cplx<double> t{0.0, 0.0};
#pragma unroll
          for (int b = 0; b < 3; ++b) t = cadd(t, cmul(u.e[a][b], xpf.v[d][b]));
          w[d][a] = t;
        }
      const cplx<double> bv = proj_dot(eta, mu, r, -1.0, w);
      jm = {kappa * (av.re - bv.re), kappa * (av.im - bv.im)};
    }
    out[slot[mu]] = jm.re;
    out[slot[mu] + 1] = jm.im;
  }
#pragma unroll
  for (int k = 0; k < kTraceVals; ++k) val[(size_t)k * V + L] = out[k];
}

// Momentum projections imom 2..5 (twAverage :4434-4503): output slot o takes per-site
// value kMomSrc[o] times factor kMomFac[o] of the site (0 = ffac, 1..3 = fas1..3), i.e.
// rho, psibar psi, psibar gamma5 psi by ffac and (Im J1 fas3, Im J2 fas1),
// (Im J3 fas2, Im J1 fas2), (Im J2 fas3, Im J3 fas1) for operators 3, 4, 5.
__device__ __constant__ int kMomSrc[kTraceVals] = {0, 1, 2, 3, 5, 7, 9, 5, 7, 9, 10, 11};
__device__ __constant__ int kMomFac[kTraceVals] = {0, 0, 0, 0, 3, 1, 2, 2, 3, 1, 0, 0};

// One block per (time slice, momentum): fixed-order sum of the slice's sites ->
// J[((iop * nmom + imom) * nt + t) * 2 + ri]; mfac[spatial site][imom - 2][4].
__global__ void __launch_bounds__(256) trace_slices_kernel(const double* val, int V, int v3, int nt,
                                                           const double* mfac, int nmom, double* J) {
  const int t = blockIdx.x, km = blockIdx.y;
  __shared__ double red[kTraceVals][256];
  double acc[kTraceVals];
#pragma unroll
  for (int k = 0; k < kTraceVals; ++k) acc[k] = 0.0;
  for (int i = threadIdx.x; i < v3; i += blockDim.x) {
    const size_t L = (size_t)t * v3 + i;
    if (km == 0) {
#pragma unroll
      for (int k = 0; k < kTraceVals; ++k) acc[k] += val[(size_t)k * V + L];
    } else {
      const double* f = mfac + ((size_t)i * 4 + (km - 1)) * 4;
#pragma unroll
      for (int k = 0; k < kTraceVals; ++k) acc[k] += val[(size_t)kMomSrc[k] * V + L] * f[kMomFac[k]];
    }
  }
#pragma unroll
  for (int k = 0; k < kTraceVals; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int k = 0; k < kTraceVals; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < kTraceVals) {
    const int k = threadIdx.x, iop = k / 2, ri = k % 2;
    J[(((size_t)iop * nmom + km) * nt + t) * 2 + ri] = red[k][0];
  }
}

}  // namespace

void momentum_table(const int* n, const int io[3], std::vector<double>& mf) {
  const int nx = n[0], ny = n[1], nz = n[2];
  mf.assign((size_t)nx * ny * nz * 16, 0.0);
  const double p1 = 8.0 * std::atan(1.0) / nx, p2 = 8.0 * std::atan(1.0) / ny, p3 = 8.0 * std::atan(1.0) / nz;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const double dx = (double)(x + 1 - io[0]) * p1, dy = (double)(y + 1 - io[1]) * p2,
                     dz = (double)(z + 1 - io[2]) * p3;
        const double cx = std::cos(dx), cy = std::cos(dy), cz = std::cos(dz), sx = std::sin(dx), sy = std::sin(dy),
                     sz = std::sin(dz);
        const double v[16] = {(cx + cy + cz) / 3.0,
                              sx,
                              sy,
                              sz,
                              (cx * cy + cx * cz + cy * cz) / 3.0,
                              sx * (cy + cz) / 2.0,
                              sy * (cx + cz) / 2.0,
                              sz * (cx + cy) / 2.0,
                              cx * cy * cz,
                              sx * cy * cz,
                              sy * cx * cz,
                              sz * cx * cy,
                              (std::cos(2.0 * dx) + std::cos(2.0 * dy) + std::cos(2.0 * dz)) / 3.0,
                              std::sin(2.0 * dx),
                              std::sin(2.0 * dy),
                              std::sin(2.0 * dz)};
        std::memcpy(mf.data() + (size_t)(x + nx * (y + ny * z)) * 16, v, sizeof(v));
      }
}

int traces_mom(qq_ctx* c, const double* be, const double* bo, const double* xe, const double* xo,
               double kappa, double delta, const int io[3], int dobndry, int nmom, double* J, int ir = 1);

int traces_level0(qq_ctx* c, const double* be, const double* bo, const double* xe,
                  const double* xo, double kappa, double delta, int dobndry, double* J) {
  const int io[3] = {1, 1, 1};
  return traces_mom(c, be, bo, xe, xo, kappa, delta, io, dobndry, 1, J);
}

int traces_mom(qq_ctx* c, const double* be, const double* bo, const double* xe, const double* xo,
               double kappa, double delta, const int io[3], int dobndry, int nmom, double* J, int ir) {
  if (ir != 1 && ir != -1) return set_error(QQ_BAD_ARG, "ir must be 1 or -1");
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  if (dobndry != 0 && dobndry != 1) return set_error(QQ_BAD_ARG, "dobndry must be 0 or 1");
  if (nmom < 1 || nmom > 5) return set_error(QQ_BAD_ARG, "nmom must be 1..5");
  const size_t nref = c->ref_doubles();
  const double *dbe, *dbo, *dxe, *dxo;
  QQ_TRY(stage_in(c, 0, be, nref, &dbe));
  QQ_TRY(stage_in(c, 1, bo, nref, &dbo));
  QQ_TRY(stage_in(c, 2, xe, nref, &dxe));
  QQ_TRY(stage_in(c, 3, xo, nref, &dxo));
  const int V = 2 * c->g.vh, nt = c->g.n[3], v3 = V / nt;
  const size_t nval = (size_t)kTraceVals * V, nJ = (size_t)kTraceVals * nt * nmom,
               nmf = nmom > 1 ? (size_t)v3 * 16 : 0;
  QQ_CK(c->trace_buf.alloc(sizeof(double) * (nval + nJ + nmf)));
  double* val = c->trace_buf.as<double>();
  double* dJ = val + nval;
  double* dmf = dJ + nJ;
  std::vector<double> mf;
  if (nmom > 1) {
    momentum_table(c->g.n, io, mf);
    QQ_CK(cudaMemcpyAsync(dmf, mf.data(), sizeof(double) * nmf, cudaMemcpyHostToDevice, c->st));
  }
  const dim3 grd((V + 127) / 128);
  if (c->recon64 == 18)
    trace_sites_kernel<18><<<grd, 128, 0, c->st>>>(c->g, c->rd, dbe, dbo, dxe, dxo, c->gauge64.p, kappa, (double)ir,
                                                   std::cos(delta), std::sin(delta), dobndry, val);
  else
    trace_sites_kernel<12><<<grd, 128, 0, c->st>>>(c->g, c->rd, dbe, dbo, dxe, dxo, c->gauge64.p, kappa, (double)ir,
                                                   std::cos(delta), std::sin(delta), dobndry, val);
  QQ_CK(cudaGetLastError());
  trace_slices_kernel<<<dim3(nt, nmom), 256, 0, c->st>>>(val, V, v3, nt, dmf, nmom, dJ);
  QQ_CK(cudaGetLastError());
  count_launch(2);
  QQ_CK(cudaMemcpyAsync(J, dJ, sizeof(double) * nJ, cudaMemcpyDefault, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));  // also keeps mf alive until its copy is done
  return QQ_OK;
}

}  // namespace qq
