// Wilson loop operators of one noise with the perturbative subtraction levels of the
// Wilson driver (qq_average): average, Q/disconloops.f90:5343-5733, with loopops
// (:7769-7910) and spacesum (:9012-9124).
//
// Level 1 uses the solution x; level k >= 2 subtracts sub_k = sum_{n=0}^{k+1} kappa^n H^n b,
// the hopping expansion of the propagator applied to the noise b, built as the reference
// builds it (H = Hsingle on each half, the powers kept in two alternating scratch pairs).
// For y = x - sub_k, one thread per lexicographic site evaluates loopops in closed form:
//   J_mu = conj( y(x+mu)^+ (1 - gamma_mu) U_mu(x)^+ b(x) - y(x)^+ (1 + gamma_mu) U_mu(x) b(x+mu) )
//   J_5 = conj(y^+ b) (+ 12 on levels k >= 2),  J_{5+mu} = conj(y^+ gamma_mu b),
// neighbours across the lattice edge times bc(mu), the complex noise kept whole.  A
// second kernel sums each (time slice, momentum) in a fixed order: every operator at
// imom = 1, and the caller's momentum factors momfac(isite, ieo, ibl, imom-1, k) on
// operators 1..5 in spacesum's slots.  Operators 1..4 are then multiplied by kappa.
// The test suite checks this against the CPU restatement of the reference's loops,
// which is itself checked against an independent numpy statement.
#include <cmath>
#include <cstring>
#include <vector>

#include "qq_ctx.h"

namespace qq {
namespace {

constexpr int kAvVals = 18;  // 9 complex operators per site

using C2 = cplx<double>;

__device__ inline void load_ref(const Geom& g, const RefDims& rd, const double* he, const double* ho,
                                const int* x, C2 v[4][3]) {
  int isite, ieo, ibleo;
  ref_site(g, x, &isite, &ieo, &ibleo);
  const double* h = ((x[0] + x[1] + x[2] + x[3]) & 1) == 0 ? he : ho;
#pragma unroll
  for (int d = 0; d < 4; ++d)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t k = ref_gi(rd, 2 * c + 1, isite, d + 1, ieo, ibleo);
      v[d][c] = {h[k], h[k + 1]};
    }
}

// (gamma_mu v) in the reference basis (Q/diracops.f90:61-71, gammamultshort :204-257)
__device__ inline void gamma_mult(int mu, const C2 v[4][3], C2 o[4][3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (mu == 0) {
      o[0][c] = v[3][c], o[1][c] = v[2][c], o[2][c] = v[1][c], o[3][c] = v[0][c];
    } else if (mu == 1) {  // (-i v3, i v2, -i v1, i v0)
      o[0][c] = {v[3][c].im, -v[3][c].re}, o[1][c] = {-v[2][c].im, v[2][c].re};
      o[2][c] = {v[1][c].im, -v[1][c].re}, o[3][c] = {-v[0][c].im, v[0][c].re};
    } else if (mu == 2) {
      o[0][c] = v[2][c], o[1][c] = {-v[3][c].re, -v[3][c].im}, o[2][c] = v[0][c];
      o[3][c] = {-v[1][c].re, -v[1][c].im};
    } else {
      o[0][c] = v[0][c], o[1][c] = v[1][c], o[2][c] = {-v[2][c].re, -v[2][c].im};
      o[3][c] = {-v[3][c].re, -v[3][c].im};
    }
  }
}

__device__ inline C2 vdot(const C2 a[4][3], const C2 b[4][3]) {  // a^+ b
  C2 s{0.0, 0.0};
#pragma unroll
  for (int d = 0; d < 4; ++d)
#pragma unroll
    for (int c = 0; c < 3; ++c) s = cadd(s, cmulconj(a[d][c], b[d][c]));
  return s;
}

template <int RECON>
__global__ void __launch_bounds__(128) loopops_kernel(Geom g, RefDims rd, const double* ye, const double* yo,
                                                      const double* be, const double* bo, const void* gauge,
                                                      int ksub, double* val) {
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
  C2 y[4][3], b[4][3];
  load_ref(g, rd, ye, yo, x, y);
  load_ref(g, rd, be, bo, x, b);
  double out[kAvVals];
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    int xn[4] = {x[0], x[1], x[2], x[3]};
    double f = 1.0;
    if (xn[mu] + 1 == g.n[mu]) {
      xn[mu] = 0;
      f = g.bcd[mu];
    } else {
      xn[mu] += 1;
    }
    C2 yn[4][3], bn[4][3], w[4][3], gw[4][3];
    load_ref(g, rd, ye, yo, xn, yn);
    load_ref(g, rd, be, bo, xn, bn);
    Su3<double> u;
    LinkIO<P64, RECON>::load(gauge, g.vh, p, mu, s, u);
    // A = f y(x+mu)^+ (1 - gamma_mu) U^+ b(x)
#pragma unroll
    for (int d = 0; d < 4; ++d)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        C2 t{0.0, 0.0};
#pragma unroll
        for (int c = 0; c < 3; ++c) t = cadd(t, cmulconj(u.e[c][a], b[d][c]));
        w[d][a] = t;
      }
    gamma_mult(mu, w, gw);
#pragma unroll
    for (int d = 0; d < 4; ++d)
#pragma unroll
      for (int a = 0; a < 3; ++a) w[d][a] = csub(w[d][a], gw[d][a]);
    const C2 A0 = vdot(yn, w);
    const C2 A{f * A0.re, f * A0.im};
    // B = - y(x)^+ (1 + gamma_mu) U f b(x+mu)
#pragma unroll
    for (int d = 0; d < 4; ++d)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        C2 t{0.0, 0.0};
#pragma unroll
        for (int c = 0; c < 3; ++c) t = cadd(t, cmul(u.e[a][c], bn[d][c]));
        w[d][a] = {f * t.re, f * t.im};
      }
    gamma_mult(mu, w, gw);
#pragma unroll
    for (int d = 0; d < 4; ++d)
#pragma unroll
      for (int a = 0; a < 3; ++a) w[d][a] = {-(w[d][a].re + gw[d][a].re), -(w[d][a].im + gw[d][a].im)};
    const C2 B = vdot(y, w);
    out[2 * mu] = A.re + B.re;
    out[2 * mu + 1] = -(A.im + B.im);
  }
  const C2 s5 = vdot(y, b);
  out[8] = s5.re + (ksub ? 12.0 : 0.0);
  out[9] = -s5.im;
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    C2 gb[4][3];
    gamma_mult(mu, b, gb);
    const C2 v = vdot(y, gb);
    out[10 + 2 * mu] = v.re;
    out[11 + 2 * mu] = -v.im;
  }
#pragma unroll
  for (int k = 0; k < kAvVals; ++k) val[(size_t)k * V + L] = out[k];
}

// spacesum's momentum slots (:9057-9085) for operators 1..5, imom >= 2: output
// (op, re/im) takes value kSrc of the site times momfac component kFac (1-based)
__device__ __constant__ int kSrc[10] = {1, 1, 3, 3, 5, 5, 6, 7, 8, 9};
__device__ __constant__ int kFac[10] = {3, 2, 1, 3, 2, 1, 4, 4, 5, 5};

// One block per (time slice, momentum): J[((iop * nmom + im) * nt + t) * 2 + ri], iop < 9.
__global__ void __launch_bounds__(256) spacesum_kernel(Geom g, const double* val, int nt, const double* momfac,
                                                       int nmom, double* J) {
  const int t = blockIdx.x, km = blockIdx.y;
  const int V = 2 * g.vh, v3 = V / nt;
  __shared__ double red[kAvVals][256];
  double acc[kAvVals];
#pragma unroll
  for (int k = 0; k < kAvVals; ++k) acc[k] = 0.0;
  for (int i = threadIdx.x; i < v3; i += blockDim.x) {
    const size_t L = (size_t)t * v3 + i;
    if (km == 0) {
#pragma unroll
      for (int k = 0; k < kAvVals; ++k) acc[k] += val[(size_t)k * V + L];
    } else {
      const int x[4] = {i % g.n[0], (i / g.n[0]) % g.n[1], i / (g.n[0] * g.n[1]), t};
      int isite, ieo, ibleo;
      ref_site(g, x, &isite, &ieo, &ibleo);
      const int ibl = 1 + (x[0] & 1) + 2 * (x[1] & 1) + 4 * (x[2] & 1) + 8 * (x[3] & 1);
      const size_t nvh = (size_t)g.vh / 16;  // the reference's nvhalf (sites per parity and block)
      const size_t base = ((((size_t)(km - 1)) * 16 + (ibl - 1)) * 2 + (ieo - 1)) * nvh + (isite - 1);
      const size_t kstride = (size_t)(nmom - 1) * 16 * 2 * nvh;
#pragma unroll
      for (int o = 0; o < 10; ++o) acc[o] += val[(size_t)kSrc[o] * V + L] * momfac[(kFac[o] - 1) * kstride + base];
    }
  }
#pragma unroll
  for (int k = 0; k < kAvVals; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int k = 0; k < kAvVals; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < kAvVals) {
    const int k = threadIdx.x, iop = k / 2, ri = k % 2;
    if (km == 0 || k < 10) J[(((size_t)iop * nmom + km) * nt + t) * 2 + ri] = red[k][0];
  }
}

__global__ void axpy_kernel(double* y, double a, const double* x, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = y[i] + a * x[i];
}

__global__ void diff_kernel(double* y, const double* x, const double* s, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = x[i] - s[i];
}

}  // namespace

// Loop operators of the reference-layout device halves y (solution side) and b (noise)
// at zero momentum, summed per time slice, without the kappa factors: loopops with
// ksub, then spacesum at imom = 1.  J_host[(iop * nt + t) * 2 + ri], iop < 9.
// Scratch: val holds 18 V doubles, Jdev 18 nt doubles.
int loop_slices(qq_ctx* c, const double* ye, const double* yo, const double* be, const double* bo, int ksub,
                double* val, double* Jdev, double* J_host) {
  const int nt = c->g.n[3], V = 2 * c->g.vh;
  count_launch(2);
  if (c->recon64 == 18)
    loopops_kernel<18><<<(V + 127) / 128, 128, 0, c->st>>>(c->g, c->rd, ye, yo, be, bo, c->gauge64.p, ksub, val);
  else
    loopops_kernel<12><<<(V + 127) / 128, 128, 0, c->st>>>(c->g, c->rd, ye, yo, be, bo, c->gauge64.p, ksub, val);
  QQ_CK(cudaGetLastError());
  spacesum_kernel<<<dim3(nt, 1), 256, 0, c->st>>>(c->g, val, nt, nullptr, 1, Jdev);
  QQ_CK(cudaGetLastError());
  QQ_CK(cudaMemcpyAsync(J_host, Jdev, sizeof(double) * 18 * nt, cudaMemcpyDeviceToHost, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

}  // namespace qq

using namespace qq;

extern "C" int qq_average(qq_ctx* c, const double* be, const double* bo, const double* xe, const double* xo,
                          double kappa, int nsub, int nmom, int nop, const double* momfac, double* Jtime) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!be || !bo || !xe || !xo || !Jtime) return set_error(QQ_BAD_ARG, "null argument");
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  if (nsub < 1 || nsub > 6) return set_error(QQ_BAD_ARG, "nsub must be 1..6");
  if (nmom < 1 || nmom > 5) return set_error(QQ_BAD_ARG, "nmom must be 1..5");
  if (nop < 9) return set_error(QQ_BAD_ARG, "nop must be at least 9");
  if (nmom > 1 && !momfac) return set_error(QQ_BAD_ARG, "momfac is needed for nmom > 1");
  QQ_CK(cudaSetDevice(c->device));
  const size_t nv = c->ref_doubles();
  const int nt = c->g.n[3], V = 2 * c->g.vh;
  // device copies: noise, solution, the expansion scratch pairs, the subtraction and y
  DevBuf buf;
  QQ_CK(buf.alloc(sizeof(double) * nv * 12));
  double* d = buf.as<double>();
  double *b_e = d, *b_o = d + nv, *x_e = d + 2 * nv, *x_o = d + 3 * nv, *s1e = d + 4 * nv, *s1o = d + 5 * nv,
         *s2e = d + 6 * nv, *s2o = d + 7 * nv, *sue = d + 8 * nv, *suo = d + 9 * nv, *y_e = d + 10 * nv,
         *y_o = d + 11 * nv;
  QQ_CK(cudaMemsetAsync(d, 0, sizeof(double) * nv * 12, c->st));
  QQ_CK(cudaMemcpyAsync(b_e, be, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(b_o, bo, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(x_e, xe, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(x_o, xo, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  const size_t nmf = nmom > 1 ? (size_t)5 * (nmom - 1) * 16 * 2 * (c->g.vh / 16) : 0;
  DevBuf dmf, dval, dJ;
  if (nmf) {
    QQ_CK(dmf.alloc(sizeof(double) * nmf));
    QQ_CK(cudaMemcpyAsync(dmf.p, momfac, sizeof(double) * nmf, cudaMemcpyDefault, c->st));
  }
  QQ_CK(dval.alloc(sizeof(double) * kAvVals * V));
  const size_t nJl = (size_t)9 * nmom * nt * 2;
  QQ_CK(dJ.alloc(sizeof(double) * nJl));
  std::vector<double> Jl(nJl), out((size_t)2 * nt * nsub * nmom * nop, 0.0);
  const int eblocks = 4 * 148;
  auto H = [&](double* o, const double* in, int gblclr) { return qq_hsingle(c, o, in, 0, gblclr); };
  auto axpy = [&](double* y, double a, const double* x) {
    count_launch();
    axpy_kernel<<<eblocks, 256, 0, c->st>>>(y, a, x, nv);
    return cudaGetLastError() == cudaSuccess ? QQ_OK : set_error(QQ_CUDA_ERR, "axpy launch");
  };
  for (int isub = 1; isub <= nsub; ++isub) {
    int ksub = 1;
    if (isub == 1) {
      ksub = 0;
      QQ_CK(cudaMemsetAsync(sue, 0, sizeof(double) * nv, c->st));
      QQ_CK(cudaMemsetAsync(suo, 0, sizeof(double) * nv, c->st));
    } else if (isub == 2) {  // O(kappa) .. O(kappa^3), :5398-5489
      QQ_TRY(H(s1e, b_o, 1));
      QQ_TRY(H(s1o, b_e, 2));
      QQ_CK(cudaMemcpyAsync(sue, b_e, sizeof(double) * nv, cudaMemcpyDeviceToDevice, c->st));
      QQ_CK(cudaMemcpyAsync(suo, b_o, sizeof(double) * nv, cudaMemcpyDeviceToDevice, c->st));
      QQ_TRY(axpy(sue, kappa, s1e));
      QQ_TRY(axpy(suo, kappa, s1o));
      QQ_TRY(H(s2e, s1o, 1));
      QQ_TRY(H(s2o, s1e, 2));
      QQ_TRY(axpy(sue, kappa * kappa, s2e));
      QQ_TRY(axpy(suo, kappa * kappa, s2o));
      QQ_TRY(H(s1e, s2o, 1));
      QQ_TRY(H(s1o, s2e, 2));
      QQ_TRY(axpy(sue, kappa * kappa * kappa, s1e));
      QQ_TRY(axpy(suo, kappa * kappa * kappa, s1o));
    } else {  // O(kappa^(isub+1)), the scratch pairs alternating (:5490-5614)
      const double xk = std::pow(kappa, isub + 1);
      if (isub % 2 == 1) {
        QQ_TRY(H(s2e, s1o, 1));
        QQ_TRY(H(s2o, s1e, 2));
        QQ_TRY(axpy(sue, xk, s2e));
        QQ_TRY(axpy(suo, xk, s2o));
      } else {
        QQ_TRY(H(s1e, s2o, 1));
        QQ_TRY(H(s1o, s2e, 2));
        QQ_TRY(axpy(sue, xk, s1e));
        QQ_TRY(axpy(suo, xk, s1o));
      }
    }
    count_launch(2);
    diff_kernel<<<eblocks, 256, 0, c->st>>>(y_e, x_e, sue, nv);
    diff_kernel<<<eblocks, 256, 0, c->st>>>(y_o, x_o, suo, nv);
    QQ_CK(cudaGetLastError());
    count_launch(2);
    if (c->recon64 == 18)
      loopops_kernel<18><<<(V + 127) / 128, 128, 0, c->st>>>(c->g, c->rd, y_e, y_o, b_e, b_o, c->gauge64.p, ksub,
                                                              dval.as<double>());
    else
      loopops_kernel<12><<<(V + 127) / 128, 128, 0, c->st>>>(c->g, c->rd, y_e, y_o, b_e, b_o, c->gauge64.p, ksub,
                                                              dval.as<double>());
    QQ_CK(cudaGetLastError());
    QQ_CK(cudaMemsetAsync(dJ.p, 0, sizeof(double) * nJl, c->st));
    count_launch();
    spacesum_kernel<<<dim3(nt, nmom), 256, 0, c->st>>>(c->g, dval.as<double>(), nt, dmf.as<double>(), nmom,
                                                       dJ.as<double>());
    QQ_CK(cudaGetLastError());
    QQ_CK(cudaMemcpyAsync(Jl.data(), dJ.p, sizeof(double) * nJl, cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    for (int iop = 0; iop < 9; ++iop)
      for (int im = 0; im < nmom; ++im)
        for (int t = 0; t < nt; ++t)
          for (int ri = 0; ri < 2; ++ri)
            out[((((size_t)iop * nmom + im) * nsub + (isub - 1)) * nt + t) * 2 + ri] =
                Jl[(((size_t)iop * nmom + im) * nt + t) * 2 + ri];
  }
  // operators 1..4 times kappa (:5728-5731)
  for (int iop = 0; iop < 4; ++iop)
    for (size_t e = (size_t)iop * nmom * nsub * nt * 2; e < (size_t)(iop + 1) * nmom * nsub * nt * 2; ++e)
      out[e] = kappa * out[e];
  QQ_CK(cudaMemcpy(Jtime, out.data(), sizeof(double) * out.size(), cudaMemcpyDefault));
  return QQ_OK;
}

// momfacs, Q/disconloops.f90:8925-8984 (host only): the momentum factors qq_average
// takes, momfac(nvhalf, 2, 16, 4, 5), nvhalf = nx ny nz nt / 32.  The reference's twoPi
// is a default-kind literal, so it carries the single-precision value.
extern "C" int qq_momfacs(const int dims[4], const int io[3], double* momfac) {
  if (!dims || !io || !momfac) return set_error(QQ_BAD_ARG, "null argument");
  Geom g{};
  for (int d = 0; d < 4; ++d) {
    if (dims[d] < 4 || dims[d] % 4 != 0) return set_error(QQ_BAD_ARG, "lattice extents must be multiples of 4");
    g.n[d] = dims[d];
    g.bc[d] = 1;
  }
  geom_finish(g);
  const int nx = dims[0], ny = dims[1], nz = dims[2], nt = dims[3];
  const size_t nv = (size_t)nx * ny * nz * nt / 32;
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
          const int x[4] = {ix - 1, iy - 1, iz - 1, it - 1};
          int isite, ieo, ibleo;
          ref_site(g, x, &isite, &ieo, &ibleo);
          const int ibl = 1 + (x[0] & 1) + 2 * (x[1] & 1) + 4 * (x[2] & 1) + 8 * (x[3] & 1);
          const double cx = std::cos(dx), cy = std::cos(dy), cz = std::cos(dz);
          const double sx = std::sin(dx), sy = std::sin(dy), sz = std::sin(dz);
          const double v[4][4] = {{sx, sy, sz, (cx + cy + cz) / 3.0},
                                  {sx * (cy + cz) / 2.0, sy * (cx + cz) / 2.0, sz * (cx + cy) / 2.0,
                                   (cx * cy + cx * cz + cy * cz) / 3.0},
                                  {sx * cy * cz, sy * cx * cz, sz * cx * cy, cx * cy * cz},
                                  {std::sin(2.0 * dx), std::sin(2.0 * dy), std::sin(2.0 * dz),
                                   (std::cos(2.0 * dx) + std::cos(2.0 * dy) + std::cos(2.0 * dz)) / 3.0}};
          for (int im = 1; im <= 4; ++im) {
            for (int k = 1; k <= 4; ++k) M(isite, ieo, ibl, im, k) = v[im - 1][k - 1];
            M(isite, ieo, ibl, im, 5) = v[im - 1][3];
          }
        }
      }
    }
  return QQ_OK;
}
