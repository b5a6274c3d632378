// Local meson correlators of a propagator column (qq_pionrho): pionrho,
// Q/quark.f90:1033-1212.  For the solution (xe, xo) of one source spin idsrc, per time
// slice t and summed over the slice's sites, colours and the real and imaginary parts:
//   pion(t)  += sum |x|^2 over the four spins (the reference's gamma_5 rotation at two
//               time slices permutes spins with signs and leaves the sum unchanged)
//   rho(t)   += rsgn(idsrc) sum (|x_1|^2 - |x_2|^2 - |x_3|^2 + |x_4|^2),
//               rsgn = (1, -1, -1, 1)  (third component of the vector current)
//   decay(t) += sum (|x_1|^2 + |x_2|^2 - |x_3|^2 - |x_4|^2)  (fourth axial component)
// in FP64.  The sites of one time slice and parity are a contiguous range of the
// checkerboard index, so one thread block reduces each (slice, parity) in a fixed
// order and the host adds the two parities.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "qq_ctx.h"

namespace qq {
namespace {

constexpr int kMesonThreads = 256;

__global__ void __launch_bounds__(kMesonThreads) pionrho_kernel(int vt, Spinor f, int vh, double* partial) {
  __shared__ double red[3][kMesonThreads];
  const int t = blockIdx.x;
  double a[3] = {0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < vt; i += blockDim.x) {
    const int s = t * vt + i;
    cplx<double> v[12];
    SpinorIO<P64>::load(f.data, f.norm, vh, s, v);
    double sp[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      sp[d] = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) sp[d] += v[3 * d + c].re * v[3 * d + c].re + v[3 * d + c].im * v[3 * d + c].im;
    }
    a[0] += sp[0] + sp[1] + sp[2] + sp[3];
    a[1] += sp[0] - sp[1] - sp[2] + sp[3];
    a[2] += sp[0] + sp[1] - sp[2] - sp[3];
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) red[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 3; ++q) partial[(size_t)t * 3 + q] = red[q][0];
}

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_pionrho(qq_ctx* c, const double* xe, const double* xo, int idsrc, double* pion, double* rho,
                          double* decay) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!xe || !xo || !pion || !rho || !decay) return set_error(QQ_BAD_ARG, "null argument");
  if (idsrc < 1 || idsrc > 4) return set_error(QQ_BAD_ARG, "idsrc must be 1..4");
  QQ_CK(cudaSetDevice(c->device));
  const int nt = c->g.n[3];
  const int vt = c->g.vh / nt;  // sites of one parity on one time slice
  const size_t nv = c->ref_doubles();
  Tmp f(c, P64);
  DevBuf part;
  QQ_CK(part.alloc(sizeof(double) * 3 * nt * 2));
  for (int p = 0; p < 2; ++p) {
    const double* d = nullptr;
    QQ_TRY(stage_in(c, 1, p == 0 ? xe : xo, nv, &d));
    QQ_TRY(ref_to_field(c, d, p, f.sp()));
    count_launch();
    pionrho_kernel<<<nt, kMesonThreads, 0, c->st>>>(vt, f.sp(), c->g.vh, part.as<double>() + (size_t)p * 3 * nt);
    QQ_CK(cudaGetLastError());
  }
  std::vector<double> h(6 * (size_t)nt);
  QQ_CK(cudaMemcpyAsync(h.data(), part.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  const double rsgn[4] = {1.0, -1.0, -1.0, 1.0};
  std::vector<double> out(3 * (size_t)nt);
  double* dst[3] = {pion, rho, decay};
  for (int q = 0; q < 3; ++q) {
    QQ_CK(cudaMemcpy(out.data() + (size_t)q * nt, dst[q], sizeof(double) * nt, cudaMemcpyDefault));
    for (int t = 0; t < nt; ++t) {
      const double v = h[(size_t)t * 3 + q] + h[(size_t)(3 * nt) + (size_t)t * 3 + q];
      out[(size_t)q * nt + t] += q == 1 ? rsgn[idsrc - 1] * v : v;
    }
    QQ_CK(cudaMemcpy(dst[q], out.data() + (size_t)q * nt, sizeof(double) * nt, cudaMemcpyDefault));
  }
  return QQ_OK;
}

// ---------------------------------------------------------------------------------------
// Sink smearing and the momentum-projected two-point functions of mesoncorr.
//
// smear, Q/diracops.f90:712-858: nsmear sweeps of
//   h <- (1 - 6 a) h + a sum_{mu = 1..3} [ U_mu(x) h(x+mu) + U_mu(x-mu)^+ h(x-mu) ]
// (spin diagonal, the spatial links only, bc(mu) on hops across the edge), both halves
// updated from the previous sweep.  One thread per lexicographic site, reference layout
// in and out, two device buffers alternating.
//
// mesoncorr, Q/quark.f90:1297-2137 (the correlator part): for the propagator columns q
// and qbar (source colour jc, spin jd) and each operator pair ii = (jop, iop) of the
// reference's table, per site
//   bit = sum_{id, jd} s(jop, jd, iop, id) sum_{ic, jc} q(jc, jd; ic, jd2(iop, id))
//                                                   conj(qbar(jc, jd2(jop, jd); ic, id))
// with the reference's signs sgnj(jop, jd) sgni(iop, id), negated when both operators
// carry rootm1 = -1 and replaced by i conj(bit) when exactly one does (:1906-1918); then
// corr(t, p, ii) = sum over the slice of bit e^{2 pi i p.(x - src)/L}, p in [-4, 4]^3.
// The phase sum is done one axis at a time (x, then y, then z) instead of per site.
// The reference evaluates only the P->P, S->P and P->S pairs (jop, iop <= 2 without
// S->S, :1869-1870); channels = 1 evaluates all 28.
// ---------------------------------------------------------------------------------------
namespace qq {
namespace {

using C2 = cplx<double>;

__device__ inline size_t ref_index(const Geom& g, const RefDims& rd, const int* x, int c, int d) {
  int isite, ieo, ibleo;
  ref_site(g, x, &isite, &ieo, &ibleo);
  return ref_gi(rd, 2 * c + 1, isite, d + 1, ieo, ibleo);
}

__device__ inline void lex_coords(const Geom& g, int L, int* x) {
  x[0] = L % g.n[0];
  L /= g.n[0];
  x[1] = L % g.n[1];
  L /= g.n[1];
  x[2] = L % g.n[2];
  x[3] = L / g.n[2];
}

template <int RECON>
__global__ void __launch_bounds__(128) smear_kernel(Geom g, RefDims rd, const void* gauge, double a, double b,
                                                    const double* ge, const double* go, double* he, double* ho) {
  const int V = 2 * g.vh;
  const int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= V) return;
  int x[4];
  lex_coords(g, L, x);
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
  const double* src = p == 0 ? ge : go;
  double* dst = p == 0 ? he : ho;
  C2 acc[4][3];
#pragma unroll
  for (int d = 0; d < 4; ++d)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[d][c] = {0.0, 0.0};
#pragma unroll
  for (int mu = 0; mu < 3; ++mu) {
    // forward: U_mu(x) h(x+mu)
    {
      int y[4] = {x[0], x[1], x[2], x[3]};
      double f = 1.0;
      if (++y[mu] == g.n[mu]) {
        y[mu] = 0;
        f = g.bcd[mu];
      }
      const double* hs = p == 0 ? go : ge;
      Su3<double> u;
      LinkIO<P64, RECON>::load(gauge, g.vh, p, mu, L >> 1, u);
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        C2 v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const size_t k = ref_index(g, rd, y, c, d);
          v[c] = {f * hs[k], f * hs[k + 1]};
        }
#pragma unroll
        for (int a3 = 0; a3 < 3; ++a3)
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[d][a3] = cadd(acc[d][a3], cmul(u.e[a3][c], v[c]));
      }
    }
    // backward: U_mu(x-mu)^+ h(x-mu)
    {
      int y[4] = {x[0], x[1], x[2], x[3]};
      double f = 1.0;
      if (y[mu] == 0) {
        y[mu] = g.n[mu] - 1;
        f = g.bcd[mu];
      } else {
        --y[mu];
      }
      const double* hs = p == 0 ? go : ge;
      const int Ly = y[0] + g.n[0] * (y[1] + g.n[1] * (y[2] + g.n[2] * y[3]));
      Su3<double> u;
      LinkIO<P64, RECON>::load(gauge, g.vh, 1 - p, mu, Ly >> 1, u);
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        C2 v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const size_t k = ref_index(g, rd, y, c, d);
          v[c] = {f * hs[k], f * hs[k + 1]};
        }
#pragma unroll
        for (int a3 = 0; a3 < 3; ++a3)
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[d][a3] = cadd(acc[d][a3], cmulconj(u.e[c][a3], v[c]));
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 4; ++d)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t k = ref_index(g, rd, x, c, d);
      dst[k] = b * src[k] + a * acc[d][c].re;
      dst[k + 1] = b * src[k + 1] + a * acc[d][c].im;
    }
}

// The operator tables of mesoncorr (Q/quark.f90:1485-1634): rootm1, jd2, sgni, sgnj for
// the 16 operators, and the (jop, iop) pairs of the 28 correlators with corrsp set.
__constant__ int kRootm1[16] = {-1, 1, -1, 1, -1, -1, 1, -1, 1, 1, 1, -1, 1, -1, 1, -1};
__constant__ int kJd2[16][4] = {{3, 4, 1, 2}, {1, 2, 3, 4}, {2, 1, 4, 3}, {2, 1, 4, 3}, {1, 2, 3, 4}, {3, 4, 1, 2},
                                {4, 3, 2, 1}, {4, 3, 2, 1}, {3, 4, 1, 2}, {1, 2, 3, 4}, {3, 4, 1, 2}, {4, 3, 2, 1},
                                {4, 3, 2, 1}, {2, 1, 4, 3}, {2, 1, 4, 3}, {1, 2, 3, 4}};
__constant__ signed char kSgni[16][4] = {{-1, -1, 1, 1}, {1, 1, 1, 1},   {-1, -1, 1, 1}, {1, -1, -1, 1},
                                         {-1, 1, 1, -1}, {1, 1, 1, 1},   {-1, -1, -1, -1}, {1, -1, 1, -1},
                                         {-1, 1, -1, 1}, {-1, -1, 1, 1}, {1, -1, -1, 1}, {-1, 1, 1, -1},
                                         {1, 1, -1, -1}, {1, 1, 1, 1},   {-1, 1, -1, 1}, {1, -1, 1, -1}};
__constant__ signed char kSgnj[16][4] = {{1, 1, -1, -1}, {1, 1, 1, 1},   {1, 1, -1, -1}, {-1, 1, 1, -1},
                                         {1, -1, -1, 1}, {1, 1, 1, 1},   {1, 1, 1, 1},   {-1, 1, -1, 1},
                                         {1, -1, 1, -1}, {-1, -1, 1, 1}, {-1, 1, 1, -1}, {1, -1, -1, 1},
                                         {-1, -1, 1, 1}, {1, 1, 1, 1},   {-1, 1, -1, 1}, {1, -1, 1, -1}};
constexpr int kPairs = 28;
const int kJop[kPairs] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 6, 2, 3, 4, 5, 7, 8, 9};
const int kIop[kPairs] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 2, 6, 7, 8, 9, 10, 3, 4, 5, 6, 2, 1, 14, 15, 16, 14, 15, 16};

// bit(x, ch) for the channels listed in pairs (jop, iop, 1-based): one thread per
// (site, channel); q and qbar hold 12 columns of two reference-layout halves each.
__global__ void __launch_bounds__(128) meson_bits_kernel(Geom g, RefDims rd, size_t half, const double* q,
                                                         const double* qbar, int nch, const int2* pairs,
                                                         double2* bits) {
  const int V = 2 * g.vh;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= (long)V * nch) return;
  const int L = (int)(t % V), ch = (int)(t / V);
  const int jop = pairs[ch].x, iop = pairs[ch].y;
  int x[4];
  lex_coords(g, L, x);
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
  C2 sum{0.0, 0.0};
  for (int id = 0; id < 4; ++id)
    for (int jd = 0; jd < 4; ++jd) {
      const int dq = kJd2[iop - 1][id] - 1;     // sink spin of q
      const int sqb = kJd2[jop - 1][jd] - 1;    // source spin of qbar
      C2 b{0.0, 0.0};
      for (int jc = 0; jc < 3; ++jc)
        for (int ic = 0; ic < 3; ++ic) {
          const double* qc = q + ((size_t)(jc * 4 + jd) * 2 + p) * half;
          const double* bc = qbar + ((size_t)(jc * 4 + sqb) * 2 + p) * half;
          const size_t kq = ref_index(g, rd, x, ic, dq), kb = ref_index(g, rd, x, ic, id);
          const C2 a{qc[kq], qc[kq + 1]}, c{bc[kb], bc[kb + 1]};
          b = cadd(b, cmulconj(c, a));  // a conj(c)
        }
      const double s = (double)kSgnj[jop - 1][jd] * (double)kSgni[iop - 1][id];
      sum = cadd(sum, C2{s * b.re, s * b.im});
    }
  const int r1 = kRootm1[jop - 1], r2 = kRootm1[iop - 1];
  double2 out;
  if (r1 == 1 && r2 == 1)
    out = make_double2(sum.re, sum.im);
  else if (r1 == -1 && r2 == -1)
    out = make_double2(-sum.re, -sum.im);
  else
    out = make_double2(sum.im, sum.re);  // i conj(sum)
  bits[t] = out;
}

// One axis of the momentum projection: in (outer, n, inner) complex -> out (outer, 9, inner)
// with out(o, p, i) = sum_k in(o, k, i) (cos, sin)[p][k].
__global__ void dft_axis_kernel(const double2* in, long outer, int n, long inner, const double2* phase,
                                double2* out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= outer * 9 * inner) return;
  const long i = t % inner, pp = (t / inner) % 9, o = t / (inner * 9);
  double re = 0.0, im = 0.0;
  for (int k = 0; k < n; ++k) {
    const double2 v = in[(o * n + k) * inner + i];
    const double2 e = phase[pp * n + k];
    re += v.x * e.x - v.y * e.y;
    im += v.x * e.y + v.y * e.x;
  }
  out[t] = make_double2(re, im);
}

}  // namespace
}  // namespace qq

extern "C" int qq_smear(qq_ctx* c, double* he, double* ho, const double* ge, const double* go, double asmear,
                        int nsmear) {
  if (!c || !he || !ho || !ge || !go) return set_error(QQ_BAD_ARG, "null argument");
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  if (nsmear < 0) return set_error(QQ_BAD_ARG, "nsmear must be >= 0");
  QQ_CK(cudaSetDevice(c->device));
  const size_t nv = c->ref_doubles();
  const int V = 2 * c->g.vh;
  DevBuf buf;
  QQ_CK(buf.alloc(sizeof(double) * 4 * nv));
  double* A = buf.as<double>();
  double* B = A + 2 * nv;
  QQ_CK(cudaMemcpyAsync(A, ge, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(A + nv, go, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemsetAsync(B, 0, sizeof(double) * 2 * nv, c->st));
  const double bs = 1.0 - 6.0 * asmear;
  for (int it = 0; it < nsmear; ++it) {
    count_launch();
    if (c->recon64 == 18)
      smear_kernel<18><<<(V + 127) / 128, 128, 0, c->st>>>(c->g, c->rd, c->gauge64.p, asmear, bs, A, A + nv, B, B + nv);
    else
      smear_kernel<12><<<(V + 127) / 128, 128, 0, c->st>>>(c->g, c->rd, c->gauge64.p, asmear, bs, A, A + nv, B, B + nv);
    QQ_CK(cudaGetLastError());
    std::swap(A, B);
  }
  QQ_CK(cudaMemcpyAsync(he, A, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(ho, A + nv, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

extern "C" int qq_mesoncorr(qq_ctx* c, const double* q, const double* qbar, const int src[4], int channels,
                            double* corrRe, double* corrIm) {
  if (!c || !q || !src || !corrRe || !corrIm) return set_error(QQ_BAD_ARG, "null argument");
  if (channels != 0 && channels != 1) return set_error(QQ_BAD_ARG, "channels must be 0 or 1");
  for (int d = 0; d < 4; ++d)
    if (src[d] < 1 || src[d] > c->g.n[d]) return set_error(QQ_BAD_ARG, "source outside the lattice");
  QQ_CK(cudaSetDevice(c->device));
  const size_t nv = c->ref_doubles(), cols = 24 * nv;
  const int nx = c->g.n[0], ny = c->g.n[1], nz = c->g.n[2], nt = c->g.n[3], V = 2 * c->g.vh;
  std::vector<int2> pairs;
  std::vector<int> which;
  for (int ii = 0; ii < kPairs; ++ii) {
    const int j = kJop[ii], i = kIop[ii];
    if (channels == 1 || (j <= 2 && i <= 2 && !(j == 1 && i == 1))) {
      pairs.push_back(make_int2(j, i));
      which.push_back(ii);
    }
  }
  const int nch = (int)pairs.size();
  DevBuf dq, dp, db, dt1, dt2, dph;
  QQ_CK(dq.alloc(sizeof(double) * (qbar && qbar != q ? 2 : 1) * cols));
  QQ_CK(cudaMemcpyAsync(dq.p, q, sizeof(double) * cols, cudaMemcpyDefault, c->st));
  const double* dqbar = dq.as<double>();
  if (qbar && qbar != q) {
    QQ_CK(cudaMemcpyAsync(dq.as<double>() + cols, qbar, sizeof(double) * cols, cudaMemcpyDefault, c->st));
    dqbar = dq.as<double>() + cols;
  }
  QQ_CK(dp.alloc(sizeof(int2) * nch));
  QQ_CK(cudaMemcpyAsync(dp.p, pairs.data(), sizeof(int2) * nch, cudaMemcpyHostToDevice, c->st));
  QQ_CK(db.alloc(sizeof(double2) * (size_t)V * nch));
  count_launch();
  meson_bits_kernel<<<(unsigned)(((long)V * nch + 127) / 128), 128, 0, c->st>>>(
      c->g, c->rd, nv, dq.as<double>(), dqbar, nch, dp.as<int2>(), db.as<double2>());
  QQ_CK(cudaGetLastError());
  // phases e^{2 pi i p (x - s) / n}, p = -4..4, per axis
  const double twoPi = 6.283185307179586;
  std::vector<double2> ph(9 * (size_t)(nx + ny + nz));
  const int ns[3] = {nx, ny, nz};
  size_t off[3] = {0, 9 * (size_t)nx, 9 * (size_t)(nx + ny)};
  for (int a = 0; a < 3; ++a)
    for (int pp = 0; pp < 9; ++pp)
      for (int k = 0; k < ns[a]; ++k) {
        const double arg = twoPi * (double)((pp - 4) * (k + 1 - src[a])) / (double)ns[a];
        ph[off[a] + (size_t)pp * ns[a] + k] = make_double2(std::cos(arg), std::sin(arg));
      }
  QQ_CK(dph.alloc(sizeof(double2) * ph.size()));
  QQ_CK(cudaMemcpyAsync(dph.p, ph.data(), sizeof(double2) * ph.size(), cudaMemcpyHostToDevice, c->st));
  // bits are (ch, t, z, y, x); project x, then y, then z
  const long s1 = (long)nch * nt * nz * ny * 9, s2 = (long)nch * nt * nz * 81, s3 = (long)nch * nt * 729;
  QQ_CK(dt1.alloc(sizeof(double2) * std::max(s1, s3)));
  QQ_CK(dt2.alloc(sizeof(double2) * std::max(s2, s3)));
  const double2* P = dph.as<double2>();
  count_launch(3);
  dft_axis_kernel<<<(unsigned)((s1 + 255) / 256), 256, 0, c->st>>>(db.as<double2>(), (long)nch * nt * nz * ny, nx, 1,
                                                                    P + off[0], dt1.as<double2>());
  dft_axis_kernel<<<(unsigned)((s2 + 255) / 256), 256, 0, c->st>>>(dt1.as<double2>(), (long)nch * nt * nz, ny, 9,
                                                                    P + off[1], dt2.as<double2>());
  dft_axis_kernel<<<(unsigned)((s3 + 255) / 256), 256, 0, c->st>>>(dt2.as<double2>(), (long)nch * nt, nz, 81,
                                                                    P + off[2], dt1.as<double2>());
  QQ_CK(cudaGetLastError());
  std::vector<double2> h(s3);
  QQ_CK(cudaMemcpyAsync(h.data(), dt1.p, sizeof(double2) * s3, cudaMemcpyDeviceToHost, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  // h is (ch, t, pz, py, px); the reference's corr(t, px, py, pz, ii)
  const size_t ncorr = (size_t)nt * 729 * kPairs;
  std::vector<double> re(ncorr, 0.0), im(ncorr, 0.0);
  for (int ch = 0; ch < nch; ++ch)
    for (int t = 0; t < nt; ++t)
      for (int pz = 0; pz < 9; ++pz)
        for (int py = 0; py < 9; ++py)
          for (int px = 0; px < 9; ++px) {
            const double2 v = h[((((size_t)ch * nt + t) * 9 + pz) * 9 + py) * 9 + px];
            const size_t o = t + (size_t)nt * (px + 9 * (py + 9 * (pz + 9 * (size_t)which[ch])));
            re[o] = v.x;
            im[o] = v.y;
          }
  QQ_CK(cudaMemcpy(corrRe, re.data(), sizeof(double) * ncorr, cudaMemcpyDefault));
  QQ_CK(cudaMemcpy(corrIm, im.data(), sizeof(double) * ncorr, cudaMemcpyDefault));
  return QQ_OK;
}
