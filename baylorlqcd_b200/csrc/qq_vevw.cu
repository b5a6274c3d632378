// The Wilson loop driver's perturbative vacuum values (vev, Q/disconloops.f90:4653-5339)
// and the driver around it (discon, :3445-3608).
//
// vev: for every site x and plane mu < nu the plaquette
//   P = U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
// (setmmf / mmd, G/gaugetools.f90:680-717, 908-984) gives Re Tr P and Im Tr P, which are
// summed per time slice with the reference's weights: plain (tsum / ssum for planes with
// and without the time direction), cosine weights averaged over the plaquette's four
// corners (mtsum / mssum), corner differences (j4sum), sine weights for the currents
// (j12t ... j32t on time planes, j12s ... j32s on space planes), with the phases
// cos / sin(2 pi k (x - io) / n), k = 1 and 2, of the 1-based coordinates (no wrap at the
// edge, as the reference computes them; its twoPi is a default-kind literal, so the
// single-precision value).  The host scales the sums by 8 kappa^4 and the reference's
// multiplicities and assembles Jvev(2, nt, 5, 5) (:5204-5310), negated.
//
// One thread per site, a block per (time slice, split, plane); each plane's code keeps
// only the sums it adds to (18 to 21 of the 65) and reads the momentum phases
// from a small table the host fills once per call; the sums are reduced per block in a
// fixed order (warp shuffles, then the warps in order) and a second kernel adds the splits and
// planes in order on the device.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "qq_ctx.h"

namespace qq {
namespace {

using C2 = cplx<double>;

// slots of the 65 per-slice sums
enum VevSlot {
  V_TSUM = 0, V_SSUM = 1, V_J1T = 2, V_J2T = 3, V_J3T = 4,
  V_MT = 5, V_MS = 9, V_J4 = 13,                           // four momenta each
  V_J12S = 17, V_J13S = 21, V_J21S = 25, V_J23S = 29, V_J31S = 33, V_J32S = 37,
  V_J12T = 41, V_J13T = 45, V_J21T = 49, V_J23T = 53, V_J31T = 57, V_J32T = 61,
  kVevVals = 65
};
constexpr int kVevSplit = 8;
constexpr int kVevThreads = 256;

__device__ inline void su3_mul(const Su3<double>& a, const Su3<double>& b, Su3<double>& c) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      C2 s{0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) s = cadd(s, cmul(a.e[i][k], b.e[k][j]));
      c.e[i][j] = s;
    }
}
// c = a b^+
__device__ inline void su3_mul_dag(const Su3<double>& a, const Su3<double>& b, Su3<double>& c) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      C2 s{0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 3; ++k) s = cadd(s, cmulconj(b.e[j][k], a.e[i][k]));
      c.e[i][j] = s;
    }
}

template <int RECON>
__device__ inline void link_at(const Geom& g, const void* gauge, const int* x, int mu, Su3<double>& u) {
  const int L = x[0] + g.n[0] * (x[1] + g.n[1] * (x[2] + g.n[2] * x[3]));
  const int p = (x[0] + x[1] + x[2] + x[3]) & 1;
  LinkIO<P64, RECON>::load(gauge, g.vh, p, mu, L >> 1, u);
}

struct Trig {  // cos, sin, cos 2, sin 2 per spatial axis at one corner
  double c[3], s[3], c2[3], s2[3];
};

constexpr bool in4(int k, int b) { return k >= b && k < b + 4; }

// The sums plane (MU, NU) adds to (0-based directions, MU < NU); the others stay zero
// for it, so its kernel keeps only these in registers.
__host__ __device__ constexpr bool vev_touches(int MU, int NU, int k) {
  return k == (NU == 3 ? V_TSUM : V_SSUM) || in4(k, NU == 3 ? V_MT : V_MS) || (NU == 3 && in4(k, V_J4)) ||
         (NU == 3 && k == V_J1T + MU) || (NU == 3 && MU == 0 && (in4(k, V_J13T) || in4(k, V_J12T))) ||
         (NU == 3 && MU == 1 && (in4(k, V_J21T) || in4(k, V_J23T))) ||
         (NU == 3 && MU == 2 && (in4(k, V_J32T) || in4(k, V_J31T))) ||
         (MU == 0 && NU != 3 && (in4(k, V_J13S) || in4(k, V_J12S))) ||
         (((MU == 1 && NU == 2) || (MU == 0 && NU == 1)) && (in4(k, V_J21S) || in4(k, V_J23S))) ||
         (NU == 2 && (in4(k, V_J32S) || in4(k, V_J31S)));
}

// One plane (MU, NU) of every site of time slice blockIdx.x, split blockIdx.y of kVevSplit.
// tab holds the momentum phases: tab[((a * 2 + sh) * 4 + f) * nmax + x] for spatial axis a,
// 0-based coordinate x shifted by sh, f = cos, sin of twoPi (x + 1 + sh - io_a) / n_a and
// cos, sin of twice that argument -- the values the reference forms per site, computed
// once on the host.  partial[((t * kVevSplit + split) * 6 + plane) * kVevVals + k].
template <int RECON, int MU, int NU>
__device__ __forceinline__ void vev_plane(const Geom& g, const void* gauge, const double* tab, int nmax,
                                          double* partial, double (*red)[kVevVals]) {
  constexpr int kPlane = MU == 0 ? NU - 1 : MU == 1 ? NU + 1 : 5;  // (0,1) .. (2,3) -> 0 .. 5
  const int t = blockIdx.x, split = blockIdx.y;
  const int vs = g.n[0] * g.n[1] * g.n[2];
  const int chunk = (vs + kVevSplit - 1) / kVevSplit;
  const int i0 = split * chunk, i1 = min(vs, i0 + chunk);
  double acc[kVevVals];
#pragma unroll
  for (int k = 0; k < kVevVals; ++k) acc[k] = 0.0;
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const int x[4] = {i % g.n[0], (i / g.n[0]) % g.n[1], i / (g.n[0] * g.n[1]), t};
    // corner trig: index 0 the site, 1 + axis a: shifted by one along spatial axis a
    double cb[3][2], sb[3][2], c2b[3][2], s2b[3][2];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int sh = 0; sh < 2; ++sh) {
        const double* e = tab + (size_t)(a * 2 + sh) * 4 * nmax + x[a];
        cb[a][sh] = __ldg(e);
        sb[a][sh] = __ldg(e + nmax);
        c2b[a][sh] = __ldg(e + 2 * nmax);
        s2b[a][sh] = __ldg(e + 3 * nmax);
      }
    Su3<double> umu, unu, ua, ub, s1, s2, P;
      {
        constexpr int mu = MU, nu = NU;
        int xm[4] = {x[0], x[1], x[2], x[3]}, xn[4] = {x[0], x[1], x[2], x[3]};
        xm[mu] = (xm[mu] + 1) % g.n[mu];
        xn[nu] = (xn[nu] + 1) % g.n[nu];
        link_at<RECON>(g, gauge, x, mu, umu);
        link_at<RECON>(g, gauge, x, nu, unu);
        link_at<RECON>(g, gauge, xm, nu, ua);  // U_nu(x + mu)
        link_at<RECON>(g, gauge, xn, mu, ub);  // U_mu(x + nu)
        su3_mul(umu, ua, s1);                  // U_mu(x) U_nu(x+mu)
        su3_mul_dag(s1, ub, s2);               // ... U_mu(x+nu)^+
        su3_mul_dag(s2, unu, P);               // ... U_nu(x)^+
        const double re = P.e[0][0].re + P.e[1][1].re + P.e[2][2].re;
        const double im = P.e[0][0].im + P.e[1][1].im + P.e[2][2].im;
        constexpr int M = mu + 1, N = nu + 1;  // the reference's 1-based directions
        // the four corners: 0 site, 1 site + mu, 2 site + nu, 3 site + mu + nu
        Trig cr[4];
#pragma unroll
        for (int v = 0; v < 4; ++v)
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const int sh = ((v & 1) && a == mu) || ((v & 2) && a == nu) ? 1 : 0;
            cr[v].c[a] = cb[a][sh];
            cr[v].s[a] = sb[a][sh];
            cr[v].c2[a] = c2b[a][sh];
            cr[v].s2[a] = s2b[a][sh];
          }
        const Trig& c0 = cr[0];
        if (N == 4) {
          acc[V_TSUM] += re;
        } else {
          acc[V_SSUM] += re;
        }
        {  // corner-averaged cosines (:4947-5004)
          double f1 = 0.0, f2 = 0.0, f3 = 0.0, f4 = 0.0;
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const Trig& q = cr[v];
            f1 += q.c[0] + q.c[1] + q.c[2];
            f2 += q.c[0] * q.c[1] + q.c[0] * q.c[2] + q.c[1] * q.c[2];
            f3 += q.c[0] * q.c[1] * q.c[2];
            f4 += q.c2[0] + q.c2[1] + q.c2[2];
          }
          const int base = N == 4 ? V_MT : V_MS;
          acc[base + 0] += f1 / 3.0 * re;
          acc[base + 1] += f2 / 3.0 * re;
          acc[base + 2] += f3 * re;
          acc[base + 3] += f4 / 3.0 * re;
        }
        if (N == 4) {  // corner 0 minus corner 1 (:5005-5029)
          const Trig& q = cr[1];
          const double f1 = (c0.c[0] + c0.c[1] + c0.c[2] - q.c[0] - q.c[1] - q.c[2]) / 3.0;
          const double f2 = (c0.c[0] * c0.c[1] + c0.c[0] * c0.c[2] + c0.c[1] * c0.c[2] - q.c[0] * q.c[1] -
                             q.c[0] * q.c[2] - q.c[1] * q.c[2]) /
                            3.0;
          const double f3 = c0.c[0] * c0.c[1] * c0.c[2] - q.c[0] * q.c[1] * q.c[2];
          const double f4 = (c0.c2[0] + c0.c2[1] + c0.c2[2] - q.c2[0] - q.c2[1] - q.c2[2]) / 3.0;
          acc[V_J4 + 0] -= f1 * im;
          acc[V_J4 + 1] -= f2 * im;
          acc[V_J4 + 2] -= f3 * im;
          acc[V_J4 + 3] -= f4 * im;
        }
        // sine weight of axis a at corner q against the other two axes' cosines
        auto sw = [&](const Trig& q, int a, double* f) {
          const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
          f[0] = q.s[a];
          f[1] = q.s[a] * (q.c[b] + q.c[c]) / 2.0;
          f[2] = q.s[a] * q.c[b] * q.c[c];
          f[3] = q.s2[a];
        };
        auto add = [&](int slot, const double* f, double w) {
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[slot + k] += w * f[k];
        };
        // sine differences: corner 0 minus corner v
        auto swd = [&](int v, int a, double* f) {
          double f0[4], fv[4];
          sw(c0, a, f0);
          sw(cr[v], a, fv);
#pragma unroll
          for (int k = 0; k < 4; ++k) f[k] = f0[k] - fv[k];
        };
        double f[4];
        if (M == 1 && N == 4) {  // :5030-5053
          acc[V_J1T] += im;
          sw(c0, 2, f);
          add(V_J13T, f, im);
          sw(c0, 1, f);
          add(V_J12T, f, im);
        }
        if (M == 2 && N == 4) {  // :5054-5077
          acc[V_J2T] += im;
          sw(c0, 0, f);
          add(V_J21T, f, im);
          sw(c0, 2, f);
          add(V_J23T, f, im);
        }
        if (M == 3 && N == 4) {  // :5078-5101
          acc[V_J3T] += im;
          sw(c0, 1, f);
          add(V_J32T, f, im);
          sw(c0, 0, f);
          add(V_J31T, f, im);
        }
        if (M == 1 && N != 4) {  // corner 2 (site + nu), :5102-5126
          swd(2, 2, f);
          add(V_J13S, f, im);
          swd(2, 1, f);
          add(V_J12S, f, im);
        }
        if (M == 2 && N == 3) {  // :5127-5148
          swd(2, 0, f);
          add(V_J21S, f, im);
          swd(2, 2, f);
          add(V_J23S, f, im);
        } else if (M == 1 && N == 2) {  // corner 1 (site + mu), :5149-5173
          swd(1, 0, f);
          add(V_J21S, f, -im);
          swd(1, 2, f);
          add(V_J23S, f, -im);
        }
        if (N == 3) {  // corner 1, :5174-5197
          swd(1, 1, f);
          add(V_J32S, f, -im);
          swd(1, 0, f);
          add(V_J31S, f, -im);
        }
      }
  }
  // block reduction in a fixed order: lanes by shuffles, then the warps in order
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kVevVals; ++k) {
    if (!vev_touches(MU, NU, k)) continue;
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][k] = v;
  }
  __syncthreads();
  double* dst = partial + (((size_t)t * kVevSplit + split) * 6 + kPlane) * kVevVals;
  for (int k = threadIdx.x; k < kVevVals; k += blockDim.x) {
    double s = 0.0;
    if (vev_touches(MU, NU, k))
      for (int ww = 0; ww < kVevThreads / 32; ++ww) s += red[ww][k];
    dst[k] = s;
  }
}

// The six planes of a slice split: blockIdx.z = 0 .. 5 for (0,1), (0,2), (0,3), (1,2),
// (1,3), (2,3), so one launch gives every SM several waves of blocks.
template <int RECON>
__global__ void __launch_bounds__(kVevThreads) vev_kernel(Geom g, const void* gauge, const double* tab, int nmax,
                                                          double* partial) {
  __shared__ double red[kVevThreads / 32][kVevVals];
  switch (blockIdx.z) {
    case 0: vev_plane<RECON, 0, 1>(g, gauge, tab, nmax, partial, red); break;
    case 1: vev_plane<RECON, 0, 2>(g, gauge, tab, nmax, partial, red); break;
    case 2: vev_plane<RECON, 0, 3>(g, gauge, tab, nmax, partial, red); break;
    case 3: vev_plane<RECON, 1, 2>(g, gauge, tab, nmax, partial, red); break;
    case 4: vev_plane<RECON, 1, 3>(g, gauge, tab, nmax, partial, red); break;
    default: vev_plane<RECON, 2, 3>(g, gauge, tab, nmax, partial, red); break;
  }
}

// Per time slice and sum: the splits and planes added in a fixed order (split-major, then
// plane), so the host copies back nt x 65 values.  One thread per (slice, sum).
__global__ void vev_fold_kernel(const double* partial, int nt, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt * kVevVals) return;
  const int t = i / kVevVals, k = i - t * kVevVals;
  double s = 0.0;
  for (int sp = 0; sp < kVevSplit; ++sp)
    for (int pl = 0; pl < 6; ++pl) s += partial[(((size_t)t * kVevSplit + sp) * 6 + pl) * kVevVals + k];
  out[i] = s;
}

constexpr int kWsVev = 8192;  // context workspace id of the partial sums and the phase table

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_vev(qq_ctx* c, double kappa, const int io[3], double* Jvev, double* plaq, double* psi) {
  if (!c || !io || !Jvev) return set_error(QQ_BAD_ARG, "null argument");
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  QQ_CK(cudaSetDevice(c->device));
  const int nt = c->g.n[3];
  const double V = 2.0 * c->g.vh;
  // the momentum phases per axis, coordinate and shift (:4823-4945 forms them per site)
  const double twoPi = (double)6.283185307179586f;  // the reference's default-kind literal
  const int nmax = std::max(c->g.n[0], std::max(c->g.n[1], c->g.n[2]));
  std::vector<double> tab((size_t)3 * 2 * 4 * nmax, 0.0);
  for (int a = 0; a < 3; ++a)
    for (int sh = 0; sh < 2; ++sh)
      for (int x = 0; x < c->g.n[a]; ++x) {
        const double X = (double)(sh + x + 1 - io[a]);
        const double arg = twoPi * X / (double)c->g.n[a], arg2 = twoPi * (2.0 * X) / (double)c->g.n[a];
        double* e = tab.data() + (size_t)(a * 2 + sh) * 4 * nmax + x;
        e[0] = std::cos(arg);
        e[nmax] = std::sin(arg);
        e[2 * nmax] = std::cos(arg2);
        e[3 * nmax] = std::sin(arg2);
      }
  const size_t npart = (size_t)nt * kVevSplit * 6 * kVevVals;
  const size_t nout = (size_t)nt * kVevVals;
  double* dp = nullptr;
  QQ_CK(ws_get(c, kWsVev, sizeof(double) * (npart + nout + tab.size()), reinterpret_cast<void**>(&dp)));
  double* dout = dp + npart;
  double* dtab = dout + nout;
  QQ_CK(cudaMemcpyAsync(dtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, c->st));
  const dim3 grd(nt, kVevSplit, 6);
  count_launch(2);
  if (c->recon64 == 18)
    vev_kernel<18><<<grd, kVevThreads, 0, c->st>>>(c->g, c->gauge64.p, dtab, nmax, dp);
  else
    vev_kernel<12><<<grd, kVevThreads, 0, c->st>>>(c->g, c->gauge64.p, dtab, nmax, dp);
  QQ_CK(cudaGetLastError());
  vev_fold_kernel<<<(unsigned)((nout + 255) / 256), 256, 0, c->st>>>(dp, nt, dout);
  QQ_CK(cudaGetLastError());
  std::vector<double> S(nout);  // per slice
  QQ_CK(cudaMemcpyAsync(S.data(), dout, sizeof(double) * nout, cudaMemcpyDeviceToHost, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  auto at = [&](int t, int k) -> double& { return S[(size_t)t * kVevVals + k]; };
  // :5204-5232: the plaquette average, then the normalisations
  double pl = 0.0;
  for (int t = 0; t < nt; ++t) pl += at(t, V_TSUM) + at(t, V_SSUM);
  pl /= 18.0 * V;
  const double factor = 8.0 * kappa * kappa * kappa * kappa;
  for (int t = 0; t < nt; ++t) {
    at(t, V_TSUM) *= 4.0 * factor;
    at(t, V_SSUM) *= 8.0 * factor;
    for (int k = V_J1T; k <= V_J3T; ++k) at(t, k) *= 2.0 * factor;
    for (int k = 0; k < 4; ++k) {
      at(t, V_MT + k) *= factor;
      at(t, V_MS + k) *= 2.0 * factor;
      at(t, V_J4 + k) *= 2.0 * factor;
    }
    for (int k = V_J12S; k < kVevVals; ++k) at(t, k) *= 2.0 * factor;
  }
  double ps = at(0, V_SSUM) + at(0, V_TSUM);
  for (int t = 1; t < nt; ++t) ps += at(t, V_SSUM) + at(t, V_TSUM) + at(t - 1, V_TSUM);
  ps /= V;
  // Jvev(2, nt, 5, 5), Fortran order (:5265-5310), then negated
  std::vector<double> J((size_t)2 * nt * 25, 0.0);
  auto jv = [&](int ri, int t, int im, int op) -> double& {  // 1-based as the reference
    return J[((((size_t)(op - 1) * 5) + (im - 1)) * nt + (t - 1)) * 2 + (ri - 1)];
  };
  jv(1, 1, 1, 5) = at(0, V_SSUM) + at(0, V_TSUM);
  for (int t = 2; t <= nt; ++t) jv(1, t, 1, 5) = at(t - 1, V_SSUM) + at(t - 1, V_TSUM) + at(t - 2, V_TSUM);
  for (int k = 0; k < 4; ++k) {
    jv(1, 1, k + 2, 5) = at(0, V_MS + k) + at(0, V_MT + k);
    for (int t = 2; t <= nt; ++t) jv(1, t, k + 2, 5) = at(t - 1, V_MS + k) + at(t - 1, V_MT + k) + at(t - 2, V_MT + k);
    for (int t = 1; t <= nt; ++t) jv(2, t, k + 2, 4) = at(t - 1, V_J4 + k);
  }
  jv(2, 1, 1, 1) = at(0, V_J1T);
  jv(2, 1, 1, 2) = at(0, V_J2T);
  jv(2, 1, 1, 3) = at(0, V_J3T);
  for (int t = 2; t <= nt; ++t) {
    jv(2, t, 1, 1) = at(t - 1, V_J1T) - at(t - 2, V_J1T);
    jv(2, t, 1, 2) = at(t - 1, V_J2T) - at(t - 2, V_J2T);
    jv(2, t, 1, 3) = at(t - 1, V_J3T) - at(t - 2, V_J3T);
  }
  const struct {
    int ri, op, s, tt;
  } cur[6] = {{1, 1, V_J13S, V_J13T}, {2, 1, V_J21S, V_J21T}, {1, 2, V_J32S, V_J32T},
              {2, 2, V_J12S, V_J12T}, {1, 3, V_J23S, V_J23T}, {2, 3, V_J31S, V_J31T}};
  for (int k = 0; k < 4; ++k)
    for (const auto& q : cur) {
      jv(q.ri, 1, k + 2, q.op) = at(0, q.s + k) + at(0, q.tt + k);
      for (int t = 2; t <= nt; ++t)
        jv(q.ri, t, k + 2, q.op) = at(t - 1, q.s + k) - at(t - 2, q.tt + k) + at(t - 1, q.tt + k);
    }
  for (double& v : J) v = -v;
  QQ_CK(cudaMemcpy(Jvev, J.data(), sizeof(double) * J.size(), cudaMemcpyDefault));
  if (plaq) *plaq = pl;
  if (psi) *psi = ps;
  return QQ_OK;
}
