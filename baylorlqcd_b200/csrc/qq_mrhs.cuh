// Batched (multi right-hand side) BiCGStab building blocks.
//
// One launch updates every active right-hand side (blockIdx.y = RHS slot); each RHS
// keeps its own complex scalars in device memory, so an iteration needs no host round
// trip.  Reductions are deterministic: per-block partials, then one block per RHS sums
// them in a fixed order inside the scalar kernel that consumes them.
#pragma once
#include "qq_blas.cuh"

namespace qq {

constexpr int kMaxBatch = 32;

// per-RHS scalar slots (doubles) in S[rhs * kScal + slot]
enum ScalSlot : int {
  SC_RHO = 0,      // complex rho
  SC_ALPHA = 2,    // complex alpha
  SC_OMEGA = 4,    // complex omega
  SC_BETA = 6,     // complex beta
  SC_R2 = 8,       // ||r||^2 (iterated residual)
  SC_TT = 9,       // ||t||^2
  kScal = 16,
};

enum BiOp : int {
  OP_DOT_RHAT_R = 0,  // red: <rhat, r>
  OP_P_UPDATE = 1,    // p = r + beta (p - omega v)
  OP_DOT_RHAT_V = 2,  // red: <rhat, v>
  OP_S_UPDATE = 3,    // r = r - alpha v
  OP_DOTS_T = 4,      // red: <t, r>, ||t||^2
  OP_XR_UPDATE = 5,   // x += alpha p + omega r ; r -= omega t ; red: ||r||^2
};

struct BatchArgs {
  int vh;
  int n;                       // active right-hand sides
  Spinor r[kMaxBatch], rhat[kMaxBatch], p[kMaxBatch], v[kMaxBatch], t[kMaxBatch], x[kMaxBatch];
  int slot[kMaxBatch];         // scalar slot of each active RHS
  double* S;                   // scalar array
  double* partial;             // [rhs][kRedBlocks][3]
};

template <class R>
__device__ inline cplx<R> cmuld(cplx<double> a, cplx<R> b) {
  return {(R)(a.re * b.re - a.im * b.im), (R)(a.re * b.im + a.im * b.re)};
}

// x, r, p, ... of one precision P (P32 or P16; P64 for testing)
template <int P, int OP>
__global__ void __launch_bounds__(kRedThreads) bicg_kernel(BatchArgs A) {
  using IO = SpinorIO<P>;
  using R = typename IO::R;
  const int k = blockIdx.y;
  const double* S = A.S + (size_t)A.slot[k] * kScal;
  double acc[3] = {0.0, 0.0, 0.0};
  cplx<double> alpha{S[SC_ALPHA], S[SC_ALPHA + 1]}, omega{S[SC_OMEGA], S[SC_OMEGA + 1]},
      beta{S[SC_BETA], S[SC_BETA + 1]};
  const cplx<double> bo = {beta.re * omega.re - beta.im * omega.im, beta.re * omega.im + beta.im * omega.re};
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < A.vh; s += gridDim.x * blockDim.x) {
    cplx<R> a[12], b[12], c[12];
    if (OP == OP_DOT_RHAT_R || OP == OP_DOT_RHAT_V) {
      IO::load(A.rhat[k].data, A.rhat[k].norm, A.vh, s, a);
      if (OP == OP_DOT_RHAT_R)
        IO::load(A.r[k].data, A.r[k].norm, A.vh, s, b);
      else
        IO::load(A.v[k].data, A.v[k].norm, A.vh, s, b);
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        acc[0] += (double)a[q].re * b[q].re + (double)a[q].im * b[q].im;
        acc[1] += (double)a[q].re * b[q].im - (double)a[q].im * b[q].re;
      }
    } else if (OP == OP_P_UPDATE) {
      IO::load(A.r[k].data, A.r[k].norm, A.vh, s, a);
      IO::load(A.p[k].data, A.p[k].norm, A.vh, s, b);
      IO::load(A.v[k].data, A.v[k].norm, A.vh, s, c);
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        const cplx<R> t1 = cmuld(beta, b[q]);
        const cplx<R> t2 = cmuld(bo, c[q]);
        a[q] = csub(cadd(a[q], t1), t2);
      }
      IO::store(A.p[k].data, A.p[k].norm, A.vh, s, a);
    } else if (OP == OP_S_UPDATE) {
      IO::load(A.r[k].data, A.r[k].norm, A.vh, s, a);
      IO::load(A.v[k].data, A.v[k].norm, A.vh, s, b);
#pragma unroll
      for (int q = 0; q < 12; ++q) a[q] = csub(a[q], cmuld(alpha, b[q]));
      IO::store(A.r[k].data, A.r[k].norm, A.vh, s, a);
    } else if (OP == OP_DOTS_T) {
      IO::load(A.t[k].data, A.t[k].norm, A.vh, s, a);
      IO::load(A.r[k].data, A.r[k].norm, A.vh, s, b);
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        acc[0] += (double)a[q].re * b[q].re + (double)a[q].im * b[q].im;
        acc[1] += (double)a[q].re * b[q].im - (double)a[q].im * b[q].re;
        acc[2] += (double)a[q].re * a[q].re + (double)a[q].im * a[q].im;
      }
    } else {  // OP_XR_UPDATE
      IO::load(A.x[k].data, A.x[k].norm, A.vh, s, a);
      IO::load(A.p[k].data, A.p[k].norm, A.vh, s, b);
      IO::load(A.r[k].data, A.r[k].norm, A.vh, s, c);
#pragma unroll
      for (int q = 0; q < 12; ++q) a[q] = cadd(a[q], cadd(cmuld(alpha, b[q]), cmuld(omega, c[q])));
      IO::store(A.x[k].data, A.x[k].norm, A.vh, s, a);
      IO::load(A.t[k].data, A.t[k].norm, A.vh, s, b);
#pragma unroll
      for (int q = 0; q < 12; ++q) c[q] = csub(c[q], cmuld(omega, b[q]));
      IO::store(A.r[k].data, A.r[k].norm, A.vh, s, c);
      if (P == P16) IO::load(A.r[k].data, A.r[k].norm, A.vh, s, c);  // reduce what was stored
#pragma unroll
      for (int q = 0; q < 12; ++q) acc[0] += (double)c[q].re * c[q].re + (double)c[q].im * c[q].im;
    }
  }
  if (OP == OP_DOT_RHAT_R || OP == OP_DOT_RHAT_V || OP == OP_DOTS_T || OP == OP_XR_UPDATE) {
    __shared__ double red[3][kRedThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      double v = acc[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      double sum = 0.0;
      for (int w = 0; w < kRedThreads / 32; ++w) sum += red[threadIdx.x][w];
      A.partial[((size_t)k * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = sum;
    }
  }
}

enum ScalStep : int {
  ST_BETA = 0,   // rho' = <rhat,r>; beta = (rho'/rho)(alpha/omega); rho = rho'
  ST_ALPHA = 1,  // alpha = rho / <rhat, v>
  ST_OMEGA = 2,  // omega = <t, r> / ||t||^2
  ST_R2 = 3,     // ||r||^2
};

// one block per RHS: sum the partials (fixed order) and update the scalars
static __global__ void bicg_scalar_kernel(double* S, const int* slots, const double* partial, int nblocks,
                                   int step) {
  const int k = blockIdx.x;
  __shared__ double red[3][256];
  double a[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int q = 0; q < 3; ++q) a[q] += partial[((size_t)k * nblocks + b) * 3 + q];
  for (int q = 0; q < 3; ++q) red[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double* s = S + (size_t)slots[k] * kScal;
  const double d0 = red[0][0], d1 = red[1][0], d2 = red[2][0];
  auto cdiv = [](double ar, double ai, double br, double bi, double* cr, double* ci) {
    const double den = br * br + bi * bi;
    *cr = (ar * br + ai * bi) / den;
    *ci = (ai * br - ar * bi) / den;
  };
  if (step == ST_BETA) {
    double qr, qi, pr, pi;
    cdiv(d0, d1, s[SC_RHO], s[SC_RHO + 1], &qr, &qi);               // rho'/rho
    cdiv(s[SC_ALPHA], s[SC_ALPHA + 1], s[SC_OMEGA], s[SC_OMEGA + 1], &pr, &pi);  // alpha/omega
    s[SC_BETA] = qr * pr - qi * pi;
    s[SC_BETA + 1] = qr * pi + qi * pr;
    s[SC_RHO] = d0;
    s[SC_RHO + 1] = d1;
  } else if (step == ST_ALPHA) {
    cdiv(s[SC_RHO], s[SC_RHO + 1], d0, d1, &s[SC_ALPHA], &s[SC_ALPHA + 1]);
  } else if (step == ST_OMEGA) {
    s[SC_OMEGA] = d0 / d2;
    s[SC_OMEGA + 1] = d1 / d2;
    s[SC_TT] = d2;
  } else {
    s[SC_R2] = d0;
  }
}

}  // namespace qq
