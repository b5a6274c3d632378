// Learned preconditioner: a gauge-covariant parallel-transport convolution network,
// trained on the GPU and applied as the right preconditioner of flexible GMRES.
//
// A layer maps Cin channels to Cout channels on the full lattice; a channel is one
// colour vector per site.  Nine paths p bring a field to the site x:
//     p = 0           f(x)
//     p = 1 + 2 mu    bc U_mu(x) f(x + mu)            (forward hop)
//     p = 2 + 2 mu    bc U_mu(x - mu)^+ f(x - mu)     (backward hop)
// (bc: the lattice's boundary factor on hops that wrap), and
//     out_co(x) = sum_p sum_ci W[p][co][ci] (T_p f_ci)(x).
// The weights act on channels only, never on colour, so every layer commutes with
// gauge transformations.  The network maps an even-site Dirac vector (channel = spin)
// to an even-site vector: embed with zeros on odd sites, apply the layers, keep the
// even sites.  Layers are linear, so the network is a fixed linear operator.
//
// The adjoint of a layer is the same kernel with weights W'[0] = W[0]^H,
// W'[mu+] = W[mu-]^H, W'[mu-] = W[mu+]^H (T_{mu+}^+ = T_{mu-}).  Training minimises
//     l = (1/S) sum_i |N(b_i) - x_i|^2 / |x_i|^2      (even sites)
// over pairs b_i = A x_i with Gaussian x_i (A = Hdbletm), so the network learns A^-1
// without solves.  Backpropagation: delta_L = dl/d conj(out) = (out - x) / (S |x|^2),
// grad[p][co][ci] = sum_x sum_a delta_co(x)_a conj((T_p f_ci)(x)_a) per layer, then
// delta of the layer's input = adjoint layer applied to delta.  Adam on the real and
// imaginary parts of the weights (host side; the weights are a few thousand numbers).
//
// Fields: FP32 complex, channel-major [channel][colour][lexicographic site L],
// L = x + nx (y + ny (z + nz t)); links: the context's FP32 recon-12 copy, addressed
// by parity (x+y+z+t) mod 2 and checkerboard index L / 2.  Reductions are fixed-order
// (warp shuffles and per-block partials in FP64, then a fixed-order sum over blocks).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "qq_ctx.h"

using qq::DevBuf;

namespace qqnet {

constexpr int kNetMaxLayers = 6;
constexpr int kNetThreads = 128;

struct NetGeom {
  int n[4];
  float bcf[4];
  int V, vh;
};

__device__ inline void lex_coords(const NetGeom& g, int L, int* x) {
  x[0] = L % g.n[0];
  int r = L / g.n[0];
  x[1] = r % g.n[1];
  r /= g.n[1];
  x[2] = r % g.n[2];
  x[3] = r / g.n[2];
}
__device__ inline int lex_index(const NetGeom& g, const int* x) {
  return x[0] + g.n[0] * (x[1] + g.n[1] * (x[2] + g.n[2] * x[3]));
}

// acc += a b (complex) as four FMAs, two per component.
__device__ inline void cmacf(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}

// (T_p f)(x) for one channel: v = f at the path's source site, transported to x.
// Returns false when the path's boundary factor is zero.
struct PathSrc {
  int L;         // source site
  float fac;     // boundary factor
  int mu, back;  // p = 1 + 2 mu + back (p > 0)
};

__device__ inline PathSrc path_src(const NetGeom& g, const int* x, int L, int p) {
  PathSrc s{L, 1.0f, 0, 0};
  if (p == 0) return s;
  s.mu = (p - 1) >> 1;
  s.back = (p - 1) & 1;
  int y[4] = {x[0], x[1], x[2], x[3]};
  if (s.back) {
    if (--y[s.mu] < 0) {
      y[s.mu] = g.n[s.mu] - 1;
      s.fac = g.bcf[s.mu];
    }
  } else {
    if (++y[s.mu] == g.n[s.mu]) {
      y[s.mu] = 0;
      s.fac = g.bcf[s.mu];
    }
  }
  s.L = lex_index(g, y);
  return s;
}

// The link of path p: U_mu(x) forward, U_mu(x - mu) (at the source site) backward.
__device__ inline void path_link(const NetGeom& g, const void* gauge, const int* x, const PathSrc& ps,
                                 qq::Su3<float>& u) {
  int y[4];
  lex_coords(g, ps.back ? ps.L : lex_index(g, x), y);
  const int par = (y[0] + y[1] + y[2] + y[3]) & 1;
  qq::LinkIO<qq::P32, 12>::load(gauge, g.vh, par, ps.mu, lex_index(g, y) >> 1, u);
}

__device__ inline void transport3(const qq::Su3<float>& u, bool back, float fac, const float2* v, float2* t) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const float2 e = back ? make_float2(u.e[b][a].re, -u.e[b][a].im) : make_float2(u.e[a][b].re, u.e[a][b].im);
      cmacf(s, e, v[b]);
    }
    t[a] = make_float2(fac * s.x, fac * s.y);
  }
}

// out = layer(w) in; w: [9][COUT][CIN] complex.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kNetThreads) ptc_kernel(NetGeom g, const void* gauge, const float2* __restrict__ in,
                                                          float2* __restrict__ out, const float2* __restrict__ w) {
  __shared__ float2 sw[9 * COUT * CIN];
  for (int i = threadIdx.x; i < 9 * COUT * CIN; i += blockDim.x) sw[i] = w[i];
  __syncthreads();
  const int L = blockIdx.x * blockDim.x + threadIdx.x;
  if (L >= g.V) return;
  int x[4];
  lex_coords(g, L, x);
  float2 acc[COUT][3];
#pragma unroll
  for (int co = 0; co < COUT; ++co)
#pragma unroll
    for (int a = 0; a < 3; ++a) acc[co][a] = make_float2(0.f, 0.f);
  for (int p = 0; p < 9; ++p) {
    const PathSrc ps = path_src(g, x, L, p);
    if (ps.fac == 0.0f) continue;
    qq::Su3<float> u;
    if (p > 0) path_link(g, gauge, x, ps, u);
    for (int ci = 0; ci < CIN; ++ci) {
      float2 v[3], t[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) v[a] = in[(size_t)(ci * 3 + a) * g.V + ps.L];
      if (p == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) t[a] = v[a];
      } else {
        transport3(u, ps.back, ps.fac, v, t);
      }
#pragma unroll
      for (int co = 0; co < COUT; ++co) {
        const float2 wc = sw[(p * COUT + co) * CIN + ci];
#pragma unroll
        for (int a = 0; a < 3; ++a) cmacf(acc[co][a], wc, t[a]);
      }
    }
  }
#pragma unroll
  for (int co = 0; co < COUT; ++co)
#pragma unroll
    for (int a = 0; a < 3; ++a) out[(size_t)(co * 3 + a) * g.V + L] = acc[co][a];
}

// Per-block partial of grad[p][co][ci] = sum_x sum_a delta_co(x)_a conj((T_p f_ci)(x)_a),
// in FP64: partial[(block * 9 * COUT + p * COUT + co) * CIN + ci] (complex).
template <int CIN, int COUT>
__global__ void __launch_bounds__(kNetThreads) ptc_wgrad_kernel(NetGeom g, const void* gauge,
                                                                const float2* __restrict__ delta,
                                                                const float2* __restrict__ fin, double2* partial) {
  __shared__ double2 red[kNetThreads / 32][COUT];
  const int L = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = L < g.V;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x[4] = {0, 0, 0, 0};
  if (act) lex_coords(g, L, x);
  float2 d[COUT][3];
#pragma unroll
  for (int co = 0; co < COUT; ++co)
#pragma unroll
    for (int a = 0; a < 3; ++a) d[co][a] = act ? delta[(size_t)(co * 3 + a) * g.V + L] : make_float2(0.f, 0.f);
  for (int p = 0; p < 9; ++p) {
    PathSrc ps{L, 0.0f, 0, 0};
    qq::Su3<float> u;
    if (act) {
      ps = path_src(g, x, L, p);
      if (p > 0 && ps.fac != 0.0f) path_link(g, gauge, x, ps, u);
    }
    for (int ci = 0; ci < CIN; ++ci) {
      float2 t[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      if (act && ps.fac != 0.0f) {
        float2 v[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) v[a] = fin[(size_t)(ci * 3 + a) * g.V + ps.L];
        if (p == 0) {
#pragma unroll
          for (int a = 0; a < 3; ++a) t[a] = v[a];
        } else {
          transport3(u, ps.back, ps.fac, v, t);
        }
      }
#pragma unroll
      for (int co = 0; co < COUT; ++co) {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {  // d conj(t)
          re += (double)d[co][a].x * t[a].x + (double)d[co][a].y * t[a].y;
          im += (double)d[co][a].y * t[a].x - (double)d[co][a].x * t[a].y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          re += __shfl_down_sync(0xffffffffu, re, o);
          im += __shfl_down_sync(0xffffffffu, im, o);
        }
        if (lane == 0) red[warp][co] = make_double2(re, im);
      }
      __syncthreads();
      if (threadIdx.x < COUT) {
        double2 s = red[0][threadIdx.x];
        for (int wi = 1; wi < kNetThreads / 32; ++wi) {
          s.x += red[wi][threadIdx.x].x;
          s.y += red[wi][threadIdx.x].y;
        }
        partial[((size_t)blockIdx.x * 9 * COUT + (size_t)p * COUT + threadIdx.x) * CIN + ci] = s;
      }
      __syncthreads();
    }
  }
}

// grad[e] (+)= sum over blocks of partial[block][e], fixed order.
__global__ void net_grad_sum_kernel(const double2* partial, int nblocks, int ne, double2* grad, int accumulate) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double2 s = make_double2(0.0, 0.0);
  for (int b = 0; b < nblocks; ++b) {
    const double2 v = partial[(size_t)b * ne + e];
    s.x += v.x;
    s.y += v.y;
  }
  if (accumulate) {
    s.x += grad[e].x;
    s.y += grad[e].y;
  }
  grad[e] = s;
}

// even-site FP64 spinor (checkerboard index) -> 4-channel net field (odd sites untouched)
__global__ void net_embed_kernel(qq::Geom gg, NetGeom g, qq::Spinor in, float2* out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= gg.vh) return;
  int x[4];
  qq::site_coords(gg, 0, s, x);
  const int L = lex_index(g, x);
  qq::cplx<double> v[12];
  qq::SpinorIO<qq::P64>::load(in.data, in.norm, gg.vh, s, v);
#pragma unroll
  for (int q = 0; q < 12; ++q) out[(size_t)q * g.V + L] = make_float2((float)v[q].re, (float)v[q].im);
}

// 4-channel net field -> even-site FP64 spinor
__global__ void net_extract_kernel(qq::Geom gg, NetGeom g, const float2* in, qq::Spinor out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= gg.vh) return;
  int x[4];
  qq::site_coords(gg, 0, s, x);
  const int L = lex_index(g, x);
  qq::cplx<double> v[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    const float2 t = in[(size_t)q * g.V + L];
    v[q] = {(double)t.x, (double)t.y};
  }
  qq::SpinorIO<qq::P64>::store(out.data, out.norm, gg.vh, s, v);
}

// delta = scale (out - target) on even sites, 0 on odd; partial[block] = sum |out - target|^2
// over even sites (FP64).
__global__ void __launch_bounds__(kNetThreads) net_residual_kernel(NetGeom g, const float2* out, const float2* target,
                                                                   float2* delta, double scale, double* partial) {
  __shared__ double red[kNetThreads / 32];
  const int L = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  if (L < g.V) {
    int x[4];
    lex_coords(g, L, x);
    const bool even = ((x[0] + x[1] + x[2] + x[3]) & 1) == 0;
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      const size_t i = (size_t)q * g.V + L;
      float2 r = make_float2(0.f, 0.f);
      if (even) {
        r = make_float2(out[i].x - target[i].x, out[i].y - target[i].y);
        s += (double)r.x * r.x + (double)r.y * r.y;
      }
      delta[i] = make_float2((float)(scale * r.x), (float)(scale * r.y));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int wi = 0; wi < kNetThreads / 32; ++wi) t += red[wi];
    partial[blockIdx.x] = t;
  }
}

// Gaussian even-site FP64 field (counter-based hash, Box-Muller), unit variance per real.
__device__ inline double u01(unsigned long long k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return ((double)(k >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
__global__ void net_gauss_kernel(int vh, unsigned long long seed, qq::Spinor out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= vh) return;
  qq::cplx<double> v[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    const unsigned long long k = (seed * 0x9e3779b97f4a7c15ULL) ^ (((unsigned long long)s * 12 + q) * 2654435761ULL);
    const double r = sqrt(-2.0 * log(u01(2 * k + 1))), th = 6.283185307179586 * u01(2 * k + 2);
    v[q] = {r * cos(th), r * sin(th)};
  }
  qq::SpinorIO<qq::P64>::store(out.data, out.norm, vh, s, v);
}

template <int CIN, int COUT>
cudaError_t launch_ptc(const NetGeom& g, const void* gauge, const float2* in, float2* out, const float2* w,
                       cudaStream_t st) {
  ptc_kernel<CIN, COUT><<<(g.V + kNetThreads - 1) / kNetThreads, kNetThreads, 0, st>>>(g, gauge, in, out, w);
  return cudaGetLastError();
}
template <int CIN, int COUT>
cudaError_t launch_wgrad(const NetGeom& g, const void* gauge, const float2* delta, const float2* fin, double2* part,
                         cudaStream_t st) {
  ptc_wgrad_kernel<CIN, COUT><<<(g.V + kNetThreads - 1) / kNetThreads, kNetThreads, 0, st>>>(g, gauge, delta, fin,
                                                                                              part);
  return cudaGetLastError();
}

#define QQ_NET_DISPATCH(FN, CI, CO, ...)                                        \
  switch (CI * 100 + CO) {                                                      \
    case 404: return FN<4, 4>(__VA_ARGS__);                                     \
    case 408: return FN<4, 8>(__VA_ARGS__);                                     \
    case 416: return FN<4, 16>(__VA_ARGS__);                                    \
    case 804: return FN<8, 4>(__VA_ARGS__);                                     \
    case 808: return FN<8, 8>(__VA_ARGS__);                                     \
    case 816: return FN<8, 16>(__VA_ARGS__);                                    \
    case 1604: return FN<16, 4>(__VA_ARGS__);                                   \
    case 1608: return FN<16, 8>(__VA_ARGS__);                                   \
    case 1616: return FN<16, 16>(__VA_ARGS__);                                  \
    default: return cudaErrorInvalidValue;                                      \
  }

cudaError_t ptc(int ci, int co, const NetGeom& g, const void* gauge, const float2* in, float2* out, const float2* w,
                cudaStream_t st) {
  qq::count_launch();
  QQ_NET_DISPATCH(launch_ptc, ci, co, g, gauge, in, out, w, st)
}
cudaError_t wgrad(int ci, int co, const NetGeom& g, const void* gauge, const float2* delta, const float2* fin,
                  double2* part, cudaStream_t st) {
  qq::count_launch();
  QQ_NET_DISPATCH(launch_wgrad, ci, co, g, gauge, delta, fin, part, st)
}

}  // namespace qqnet

using namespace qqnet;

// ---------------------------------------------------------------------------
// The network handle
// ---------------------------------------------------------------------------
struct qq_net {
  int nl = 0;
  int ch[kNetMaxLayers + 1] = {};
  std::vector<std::complex<double>> w;  // [layer][9][co][ci], FP64 master copy
  std::vector<size_t> off;              // first weight of each layer
  DevBuf wf, wa;                        // FP32 weights and adjoint weights on the device
  DevBuf acts[kNetMaxLayers + 1];       // activations (acts[0]: the embedded input), kept
  int wdev = -1;                        // device of wf / wa / acts
  bool dirty = true;
  std::vector<double> am, av;           // Adam moments (real, imaginary interleaved)
  int at = 0;
  size_t nw() const { return w.size(); }
};

namespace qq {

namespace {

NetGeom net_geom(qq_ctx* c) {
  NetGeom g;
  for (int mu = 0; mu < 4; ++mu) {
    g.n[mu] = c->g.n[mu];
    g.bcf[mu] = (float)c->g.bc[mu];
  }
  g.V = 2 * c->g.vh;
  g.vh = c->g.vh;
  return g;
}

size_t net_field_bytes(qq_ctx* c, int channels) { return (size_t)channels * 3 * 2 * c->g.vh * sizeof(float2); }

// FP32 weights and adjoint weights of every layer on the context's device.
int net_upload(qq_ctx* c, qq_net* net) {
  if (!net->dirty && net->wdev == c->device) return QQ_OK;
  if (net->wdev != c->device)  // buffers of another device: release them
    for (DevBuf& b : net->acts)
      if (b.p) {
        cudaFree(b.p);
        b.p = nullptr;
        b.bytes = 0;
      }
  std::vector<float2> wf(net->nw()), wa(net->nw());
  for (int l = 0; l < net->nl; ++l) {
    const int ci = net->ch[l], co = net->ch[l + 1];
    const std::complex<double>* W = net->w.data() + net->off[l];
    float2* F = wf.data() + net->off[l];
    float2* A = wa.data() + net->off[l];  // adjoint: [9][ci][co]
    for (int p = 0; p < 9; ++p)
      for (int o = 0; o < co; ++o)
        for (int i = 0; i < ci; ++i) {
          const std::complex<double> v = W[((size_t)p * co + o) * ci + i];
          F[((size_t)p * co + o) * ci + i] = make_float2((float)v.real(), (float)v.imag());
          const int pa = p == 0 ? 0 : ((p - 1) & 1) ? p - 1 : p + 1;  // mu+ <-> mu-
          A[((size_t)pa * ci + i) * co + o] = make_float2((float)v.real(), (float)-v.imag());
        }
  }
  QQ_CK(net->wf.alloc(sizeof(float2) * wf.size()));
  QQ_CK(net->wa.alloc(sizeof(float2) * wa.size()));
  QQ_CK(cudaMemcpyAsync(net->wf.p, wf.data(), sizeof(float2) * wf.size(), cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaMemcpyAsync(net->wa.p, wa.data(), sizeof(float2) * wa.size(), cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  net->wdev = c->device;
  net->dirty = false;
  return QQ_OK;
}

// acts[l + 1] = layer l applied to (l == 0 ? input : acts[l]); acts[0] is not used.
int net_forward(qq_ctx* c, qq_net* net, const float2* input, DevBuf* acts) {
  const NetGeom g = net_geom(c);
  for (int l = 0; l < net->nl; ++l) {
    QQ_CK(acts[l + 1].alloc(net_field_bytes(c, net->ch[l + 1])));
    QQ_CK(ptc(net->ch[l], net->ch[l + 1], g, c->gauge32.p, l == 0 ? input : acts[l].as<float2>(),
              acts[l + 1].as<float2>(), net->wf.as<float2>() + net->off[l], c->st));
  }
  return QQ_OK;
}

}  // namespace

// z = N(v) for even-site FP64 fields (the preconditioner of flexible GMRES).  The
// activation buffers live in the network handle, so repeated applications allocate
// nothing.
int net_apply_field(qq_ctx* c, qq_net* net, Spinor out, Spinor in) {
  QQ_TRY(net_upload(c, net));
  const NetGeom g = net_geom(c);
  DevBuf* acts = net->acts;
  QQ_CK(acts[0].alloc(net_field_bytes(c, 4)));
  QQ_CK(cudaMemsetAsync(acts[0].p, 0, acts[0].bytes, c->st));
  const int nblk = (c->g.vh + 127) / 128;
  count_launch(2);
  net_embed_kernel<<<nblk, 128, 0, c->st>>>(c->g, g, in, acts[0].as<float2>());
  QQ_CK(cudaGetLastError());
  QQ_TRY(net_forward(c, net, acts[0].as<float2>(), acts));
  net_extract_kernel<<<nblk, 128, 0, c->st>>>(c->g, g, acts[net->nl].as<float2>(), out);
  QQ_CK(cudaGetLastError());
  return QQ_OK;
}

namespace {

// Loss and gradient (accumulated into grad, complex [nw]) over pairs of embedded net
// fields B[i], X[i]; returns the loss.
int net_loss_grad(qq_ctx* c, qq_net* net, const std::vector<DevBuf>& B, const std::vector<DevBuf>& X,
                  const std::vector<double>& xnorm2, DevBuf& grad, double* loss) {
  QQ_TRY(net_upload(c, net));
  const NetGeom g = net_geom(c);
  const int S = (int)B.size();
  const int nblk = (g.V + kNetThreads - 1) / kNetThreads;
  int maxc = 4;
  for (int l = 0; l <= net->nl; ++l) maxc = std::max(maxc, net->ch[l]);
  DevBuf part, lpart, d0, d1;
  QQ_CK(part.alloc(sizeof(double2) * (size_t)nblk * 9 * maxc * maxc));
  QQ_CK(lpart.alloc(sizeof(double) * nblk));
  QQ_CK(d0.alloc(net_field_bytes(c, maxc)));
  QQ_CK(d1.alloc(net_field_bytes(c, maxc)));
  QQ_CK(grad.alloc(sizeof(double2) * net->nw()));
  QQ_CK(cudaMemsetAsync(grad.p, 0, grad.bytes, c->st));
  std::vector<double> lp(nblk);
  DevBuf* acts = net->acts;
  double total = 0.0;
  for (int i = 0; i < S; ++i) {
    QQ_TRY(net_forward(c, net, B[i].as<float2>(), acts));
    const double scale = 1.0 / ((double)S * xnorm2[i]);
    count_launch();
    net_residual_kernel<<<nblk, kNetThreads, 0, c->st>>>(g, acts[net->nl].as<float2>(), X[i].as<float2>(),
                                                         d0.as<float2>(), scale, lpart.as<double>());
    QQ_CK(cudaGetLastError());
    QQ_CK(cudaMemcpyAsync(lp.data(), lpart.p, sizeof(double) * nblk, cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    double li = 0.0;
    for (double v : lp) li += v;
    total += li / ((double)S * xnorm2[i]);
    DevBuf* dcur = &d0;
    DevBuf* dnext = &d1;
    for (int l = net->nl - 1; l >= 0; --l) {
      const int ci = net->ch[l], co = net->ch[l + 1];
      const int ne = 9 * co * ci;
      const float2* fin = l == 0 ? B[i].as<float2>() : acts[l].as<float2>();
      QQ_CK(wgrad(ci, co, g, c->gauge32.p, dcur->as<float2>(), fin, part.as<double2>(), c->st));
      count_launch();
      net_grad_sum_kernel<<<(ne + 127) / 128, 128, 0, c->st>>>(part.as<double2>(), nblk, ne,
                                                              grad.as<double2>() + net->off[l], 1);
      QQ_CK(cudaGetLastError());
      if (l > 0) {
        QQ_CK(ptc(co, ci, g, c->gauge32.p, dcur->as<float2>(), dnext->as<float2>(), net->wa.as<float2>() + net->off[l],
                  c->st));
        std::swap(dcur, dnext);
      }
    }
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  *loss = total;
  return QQ_OK;
}

// Even-site reference half vectors -> embedded net fields (and |x|^2 of each); out
// holds n buffers.
int net_embed_refs(qq_ctx* c, int n, const double* refs, std::vector<DevBuf>& out, std::vector<double>* norm2) {
  const NetGeom g = net_geom(c);
  const size_t nv = c->ref_doubles();
  Tmp t(c, P64);
  if (norm2) norm2->resize(n);
  const int nblk = (c->g.vh + 127) / 128;
  for (int i = 0; i < n; ++i) {
    const double* d = nullptr;
    QQ_TRY(stage_in(c, 1, refs + (size_t)i * nv, nv, &d));
    QQ_TRY(ref_to_field(c, d, 0, t.sp()));
    if (norm2) QQ_TRY(norm2_host(c, t.sp(), &(*norm2)[i]));
    QQ_CK(out[i].alloc(net_field_bytes(c, 4)));
    QQ_CK(cudaMemsetAsync(out[i].p, 0, out[i].bytes, c->st));
    count_launch();
    net_embed_kernel<<<nblk, 128, 0, c->st>>>(c->g, g, t.sp(), out[i].as<float2>());
    QQ_CK(cudaGetLastError());
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

int net_check(qq_ctx* c, const qq_net* net) {
  if (!c || !net) return set_error(QQ_BAD_ARG, "null context or network");
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  QQ_CK(cudaSetDevice(c->device));
  return QQ_OK;
}

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_net_create(int nlayers, const int* channels, unsigned long long seed, double scale,
                             qq_net** out) {
  if (!channels || !out) return set_error(QQ_BAD_ARG, "null argument");
  if (nlayers < 1 || nlayers > kNetMaxLayers) return set_error(QQ_BAD_ARG, "nlayers must be 1..6");
  if (channels[0] != 4 || channels[nlayers] != 4)
    return set_error(QQ_BAD_ARG, "the first and last channel counts must be 4 (the spins)");
  for (int l = 0; l <= nlayers; ++l)
    if (channels[l] != 4 && channels[l] != 8 && channels[l] != 16)
      return set_error(QQ_BAD_ARG, "channel counts must be 4, 8 or 16");
  auto* net = new qq_net();
  net->nl = nlayers;
  size_t n = 0;
  for (int l = 0; l <= nlayers; ++l) net->ch[l] = channels[l];
  for (int l = 0; l < nlayers; ++l) {
    net->off.push_back(n);
    n += (size_t)9 * channels[l] * channels[l + 1];
  }
  net->w.assign(n, 0.0);
  // Start near scale * identity: path 0 passes channel i to channel i (the first four
  // channels of every layer; the product of the layers' factors is `scale`), every
  // other weight small and random.
  const double per = std::pow(std::fabs(scale) > 0 ? std::fabs(scale) : 1.0, 1.0 / nlayers);
  unsigned long long st = seed * 0x9e3779b97f4a7c15ULL + 1;
  auto rnd = [&]() {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return ((double)(st >> 11) / 9007199254740992.0) - 0.5;
  };
  for (int l = 0; l < nlayers; ++l) {
    const int ci = channels[l], co = channels[l + 1];
    std::complex<double>* W = net->w.data() + net->off[l];
    for (int p = 0; p < 9; ++p)
      for (int o = 0; o < co; ++o)
        for (int i = 0; i < ci; ++i) W[((size_t)p * co + o) * ci + i] = 0.02 * per * std::complex<double>(rnd(), rnd());
    for (int i = 0; i < 4; ++i) W[(size_t)i * ci + i] += (l == 0 && scale < 0) ? -per : per;
  }
  net->am.assign(2 * n, 0.0);
  net->av.assign(2 * n, 0.0);
  *out = net;
  return QQ_OK;
}

extern "C" int qq_net_destroy(qq_net* net) {
  delete net;
  return QQ_OK;
}

extern "C" int qq_net_nweights(const qq_net* net) { return net ? (int)net->nw() : 0; }

extern "C" int qq_net_get_weights(const qq_net* net, double* w) {
  if (!net || !w) return set_error(QQ_BAD_ARG, "null argument");
  for (size_t i = 0; i < net->nw(); ++i) {
    w[2 * i] = net->w[i].real();
    w[2 * i + 1] = net->w[i].imag();
  }
  return QQ_OK;
}

extern "C" int qq_net_set_weights(qq_net* net, const double* w) {
  if (!net || !w) return set_error(QQ_BAD_ARG, "null argument");
  for (size_t i = 0; i < net->nw(); ++i) net->w[i] = {w[2 * i], w[2 * i + 1]};
  net->dirty = true;
  return QQ_OK;
}

extern "C" int qq_net_apply(qq_ctx* c, qq_net* net, const double* in, double* out) {
  QQ_TRY(net_check(c, net));
  if (!in || !out) return set_error(QQ_BAD_ARG, "null array");
  Tmp a(c, P64), b(c, P64);
  const double* d = nullptr;
  QQ_TRY(stage_in(c, 1, in, c->ref_doubles(), &d));
  QQ_TRY(ref_to_field(c, d, 0, a.sp()));
  QQ_TRY(net_apply_field(c, net, b.sp(), a.sp()));
  double* o = nullptr;
  QQ_TRY(stage_out_begin(c, 2, out, c->ref_doubles(), &o));
  QQ_TRY(field_to_ref(c, b.sp(), 0, o));
  QQ_TRY(stage_out_end(c, 2, out, c->ref_doubles(), o));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

extern "C" int qq_net_grad(qq_ctx* c, qq_net* net, int nsamples, const double* b, const double* x, double* loss,
                           double* grad) {
  QQ_TRY(net_check(c, net));
  if (nsamples < 1 || !b || !x || !loss || !grad) return set_error(QQ_BAD_ARG, "bad arguments");
  std::vector<DevBuf> B(nsamples), X(nsamples);
  std::vector<double> xn2;
  QQ_TRY(net_embed_refs(c, nsamples, b, B, nullptr));
  QQ_TRY(net_embed_refs(c, nsamples, x, X, &xn2));
  for (double v : xn2)
    if (!(v > 0.0)) return set_error(QQ_BAD_ARG, "a target vector is zero");
  DevBuf g;
  QQ_TRY(net_loss_grad(c, net, B, X, xn2, g, loss));
  QQ_CK(cudaMemcpy(grad, g.p, sizeof(double2) * net->nw(), cudaMemcpyDeviceToHost));
  return QQ_OK;
}

namespace qq {
namespace {
int adam_steps(qq_ctx* c, qq_net* net, const std::vector<DevBuf>& B, const std::vector<DevBuf>& X,
               const std::vector<double>& xn2, int nsteps, double lr, double* losses);
}  // namespace
}  // namespace qq

extern "C" int qq_net_train(qq_ctx* c, qq_net* net, const double kappa[2], int nsamples, int nsteps, double lr,
                            unsigned long long seed, double* losses) {
  QQ_TRY(net_check(c, net));
  if (!kappa || nsamples < 1 || nsteps < 0 || !(lr > 0.0)) return set_error(QQ_BAD_ARG, "bad arguments");
  // pairs (b = A x, x) with Gaussian x on the even sites
  const NetGeom g = net_geom(c);
  std::vector<DevBuf> B(nsamples), X(nsamples);
  std::vector<double> xn2(nsamples);
  Tmp xf(c, P64), bf(c, P64), tmp(c, P64);
  const int nblk = (c->g.vh + 127) / 128;
  for (int i = 0; i < nsamples; ++i) {
    count_launch();
    net_gauss_kernel<<<nblk, 128, 0, c->st>>>(c->g.vh, seed * 1000003ULL + (unsigned long long)i, xf.sp());
    QQ_CK(cudaGetLastError());
    QQ_TRY(op_dbletm(c, bf.sp(), xf.sp(), tmp.sp(), 0, kappa));
    QQ_TRY(norm2_host(c, xf.sp(), &xn2[i]));
    for (auto* pr : {&B[i], &X[i]}) {
      QQ_CK(pr->alloc(net_field_bytes(c, 4)));
      QQ_CK(cudaMemsetAsync(pr->p, 0, pr->bytes, c->st));
    }
    count_launch(2);
    net_embed_kernel<<<nblk, 128, 0, c->st>>>(c->g, g, bf.sp(), B[i].as<float2>());
    net_embed_kernel<<<nblk, 128, 0, c->st>>>(c->g, g, xf.sp(), X[i].as<float2>());
    QQ_CK(cudaGetLastError());
  }
  return adam_steps(c, net, B, X, xn2, nsteps, lr, losses);
}

extern "C" int qq_net_train_pairs(qq_ctx* c, qq_net* net, int nsamples, const double* b, const double* x, int nsteps,
                                  double lr, double* losses) {
  QQ_TRY(net_check(c, net));
  if (nsamples < 1 || !b || !x || nsteps < 0 || !(lr > 0.0)) return set_error(QQ_BAD_ARG, "bad arguments");
  std::vector<DevBuf> B(nsamples), X(nsamples);
  std::vector<double> xn2;
  QQ_TRY(net_embed_refs(c, nsamples, b, B, nullptr));
  QQ_TRY(net_embed_refs(c, nsamples, x, X, &xn2));
  for (double v : xn2)
    if (!(v > 0.0)) return set_error(QQ_BAD_ARG, "a target vector is zero");
  return adam_steps(c, net, B, X, xn2, nsteps, lr, losses);
}

namespace qq {
namespace {
// nsteps Adam steps (learning rate lr) on the loss of net_loss_grad over the embedded
// pairs (B[i], X[i]); losses[step] (may be null) = the loss before each step.
int adam_steps(qq_ctx* c, qq_net* net, const std::vector<DevBuf>& B, const std::vector<DevBuf>& X,
               const std::vector<double>& xn2, int nsteps, double lr, double* losses) {
  const size_t n = net->nw();
  std::vector<double2> gh(n);
  constexpr double b1 = 0.9, b2 = 0.999, eps = 1e-12;
  for (int step = 0; step < nsteps; ++step) {
    DevBuf gd;
    double loss = 0.0;
    QQ_TRY(net_loss_grad(c, net, B, X, xn2, gd, &loss));
    if (!std::isfinite(loss)) return set_error(QQ_NAN, "NaN loss in network training");
    if (losses) losses[step] = loss;
    QQ_CK(cudaMemcpy(gh.data(), gd.p, sizeof(double2) * n, cudaMemcpyDeviceToHost));
    ++net->at;
    const double c1 = 1.0 - std::pow(b1, net->at), c2 = 1.0 - std::pow(b2, net->at);
    for (size_t i = 0; i < n; ++i) {
      const double gr[2] = {2.0 * gh[i].x, 2.0 * gh[i].y};  // dl/dRe W, dl/dIm W
      double upd[2];
      for (int k = 0; k < 2; ++k) {
        double& m = net->am[2 * i + k];
        double& v = net->av[2 * i + k];
        m = b1 * m + (1.0 - b1) * gr[k];
        v = b2 * v + (1.0 - b2) * gr[k] * gr[k];
        upd[k] = lr * (m / c1) / (std::sqrt(v / c2) + eps);
      }
      net->w[i] -= std::complex<double>(upd[0], upd[1]);
    }
    net->dirty = true;
  }
  return QQ_OK;
}
}  // namespace
}  // namespace qq

// Flexible GMRES(m) (k = 0) or flexible GMRES-DR(m, k) preconditioned by the network
// (or unpreconditioned when net is null); when two consecutive cycles each gain less
// than a factor 2, plain FP64 GMRES-DR(m, max(k, m/3)) takes over from the current x
// to the same overall tolerance.
static int flexible_solve(qq_ctx* c, qq_net* net, const double* phi, double* x, int m, int k, double resmax,
                          int max_cycles, const double kappa[2], qq_solve_info* info) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  QQ_CK(cudaSetDevice(c->device));
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  if (!phi || !x || !kappa) return set_error(QQ_BAD_ARG, "null argument");
  if (m < 2 || m > 127 || k < 0 || k >= m || max_cycles < 1 || !(resmax > 0.0))
    return set_error(QQ_BAD_ARG, "bad FGMRES arguments");
  if (net) QQ_TRY(net_check(c, net));
  Tmp fphi(c, P64), fx(c, P64);
  const size_t nv = c->ref_doubles();
  const double* d = nullptr;
  QQ_TRY(stage_in(c, 1, phi, nv, &d));
  QQ_TRY(ref_to_field(c, d, 0, fphi.sp()));
  QQ_TRY(stage_in(c, 2, x, nv, &d));
  QQ_TRY(ref_to_field(c, d, 0, fx.sp()));
  QQ_CK(cudaEventRecord(c->ev0, c->st));
  auto M = [&](Spinor z, Spinor v) -> int { return net ? net_apply_field(c, net, z, v) : copy_field(c, z, v); };
  SolveStats s;
  bool stalled = false;
  int status = k == 0 ? fgmres_fp64(c, fphi.sp(), fx.sp(), m, resmax, max_cycles, kappa, M, &s, &stalled)
                      : fgmresdr_fp64(c, fphi.sp(), fx.sp(), m, k, resmax, max_cycles, kappa, M, &s, &stalled);
  int fallback = 0;
  if (status == QQ_NOT_CONVERGED && stalled && s.true_rel > 0.0) {
    fallback = 1;
    const double r0 = s.true_rel;  // relative to the original initial residual
    SolveStats s2;
    status = gmresdr_fp64(c, fphi.sp(), fx.sp(), m, std::max(std::max(1, k), m / 3), resmax / r0, 0, kappa,
                          nullptr, &s2);
    s.itercount += s2.itercount;
    const int mvp0 = s.mvp;
    s.mvp += s2.mvp;
    s.ncycles += s2.ncycles;
    for (size_t i = 0; i < s2.hist.size(); ++i) {
      s.hist.push_back(s2.hist[i] * r0);
      s.hist_mvp.push_back(mvp0 + s2.hist_mvp[i]);
    }
    s.true_rel = s2.true_rel * r0;
    s.ritz = s2.ritz;
  }
  if (status != QQ_OK && status != QQ_NOT_CONVERGED) return status;
  QQ_CK(cudaEventRecord(c->ev1, c->st));
  QQ_CK(cudaEventSynchronize(c->ev1));
  float ms = 0.f;
  QQ_CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  double* o = nullptr;
  QQ_TRY(stage_out_begin(c, 2, x, nv, &o));
  QQ_TRY(field_to_ref(c, fx.sp(), 0, o));
  QQ_TRY(stage_out_end(c, 2, x, nv, o));
  QQ_CK(cudaStreamSynchronize(c->st));
  fill_info(info, status, s, ms * 1e-3);
  if (info) info->fallback = fallback;
  return status;
}

extern "C" int qq_fgmres(qq_ctx* c, qq_net* net, const double* phi, double* x, int m, double resmax, int max_cycles,
                         const double kappa[2], qq_solve_info* info) {
  return flexible_solve(c, net, phi, x, m, 0, resmax, max_cycles, kappa, info);
}

extern "C" int qq_fgmresdr(qq_ctx* c, qq_net* net, const double* phi, double* x, const int GMRES[2], double resmax,
                           int max_cycles, const double kappa[2], qq_solve_info* info) {
  if (!GMRES) return set_error(QQ_BAD_ARG, "null GMRES");
  if (GMRES[1] < 1) return set_error(QQ_BAD_ARG, "FGMRES-DR needs k >= 1");
  return flexible_solve(c, net, phi, x, GMRES[0], GMRES[1], resmax, max_cycles, kappa, info);
}
