// Batched (multi right-hand side) BiCGStab building blocks on RHS-interleaved block
// fields: a block of nb right-hand sides is one spinor field of vh * nb "sites",
// element (plane q, site s, rhs r) at q * (vh * nb) + s * nb + r, so a warp reads
// contiguous 16-byte runs across right-hand sides and sites.
//
// One launch updates every right-hand side of the block; each keeps its own complex
// scalars in device memory, so an iteration needs no host round trip.  Reductions are
// deterministic: per-block partials per right-hand side, then one block per RHS sums
// them in a fixed order inside the scalar kernel that consumes them.
#pragma once
#include "qq_blas.cuh"

namespace qq {

// per-RHS scalar slots (doubles) in S[rhs * kScal + slot]
enum ScalSlot : int {
  SC_RHO = 0,      // complex rho
  SC_ALPHA = 2,    // complex alpha
  SC_OMEGA = 4,    // complex omega
  SC_BETA = 6,     // complex beta
  SC_R2 = 8,       // ||r||^2 (iterated residual)
  SC_TT = 9,       // ||t||^2
  SC_RMAX = 10,    // ||r|| at the last reliable update
  SC_BN = 11,      // ||b||
  SC_ITS = 12,     // iterations done
  SC_T2 = 13,      // ||b - A x||^2 of the last reliable update (FP64)
  SC_TRUE = 14,    // ||b - A x|| / ||b|| of the last reliable update
  SC_NUPD = 15,    // reliable updates done
  SC_RHATN = 16,   // ||rhat|| (the shadow residual; replaced only at a restart)
  SC_CHK_R = 17,   // progress anchor: the FP64 true ||b - A x|| that last fell 10x
  SC_CHK_ITS = 18, // iterations done when the anchor was set
  SC_FAIL = 19,    // why the right-hand side was stopped (FailCode), 0 while it runs
  SC_NRST = 20,    // restarts after a breakdown so far
  kScal = 21,
};

// Control words after the scalar slots: bit k of ACTIVE / PENDING / DONE / INSERT /
// NAN / FAIL / RESTART = right-hand side k iterates / awaits its reliable update or
// convergence test / is finished (converged or stopped) / is re-inserted / stopped on a
// non-finite value / stopped without converging (reason in its SC_FAIL) / restarts with
// its re-inserted residual as the shadow residual; ITER counts the iterations of the
// graph-driven loop.
enum CtlWord : int {
  CTL_ACTIVE = 0,
  CTL_PENDING = 1,
  CTL_DONE = 2,
  CTL_INSERT = 3,
  CTL_ITER = 4,
  CTL_NAN = 5,
  CTL_FAIL = 6,
  CTL_RESTART = 7,
  kCtlWords = 8
};

// Why the batched BiCGStab stopped a right-hand side short of its tolerance; the
// caller hands such a right-hand side to plain FP64 GMRES-DR (qq_solve_info.fallback).
enum FailCode : int {
  FAIL_NONE = 0,
  FAIL_NAN = 1,        // a non-finite scalar or residual
  FAIL_BREAKDOWN = 2,  // rho = <rhat, r>, <rhat, v>, ||t|| or omega = <t, s> / ||t||^2 vanished
                       // again after kMaxRestarts restarts
  FAIL_STALL = 3,      // the FP64 true residual did not fall 10x within the stall window
  FAIL_MAXITER = 4,    // the iteration limit ran out (set by the host)
};

// Relative size below which a BiCGStab inner product counts as a breakdown:
// |<rhat, r>| <= kBreakEps ||rhat|| ||r||, and the same for omega.  Only a degenerate
// (numerically zero) product trips it; slow progress is the stall window's business.
constexpr double kBreakEps = 1e-12;

// Restarts a right-hand side may take after a breakdown before it stops for good.  A
// restart is a reliable update after which the shadow residual becomes the re-inserted
// FP64 residual (rho = ||r||^2, beta = 0, so the next search direction is r).  The
// usual shadow residual rhat = r0 is one spin-colour component at one site for a point
// source: every <rhat, .> is then a single component, which 16-bit storage against the
// site's norm (or an exact FP32 cancellation) can make exactly zero while the Krylov
// space is fine; the residual a few iterations on is spread over the lattice.
constexpr int kMaxRestarts = 8;

enum BiOp : int {
  OP_DOT_RHAT_R = 0,  // red: <rhat, r>
  OP_P_UPDATE = 1,    // p = r + beta (p - omega v)
  OP_DOT_RHAT_V = 2,  // red: <rhat, v>
  OP_S_UPDATE = 3,    // r = r - alpha v
  OP_DOTS_T = 4,      // red: <t, r>, ||t||^2
  OP_XR_UPDATE = 5,   // x += alpha p + omega r ; r -= omega t ; red: ||r||^2, <rhat, r>
};

struct BlockBiArgs {
  int vh;                      // sites per parity
  int nb;                      // right-hand sides in the block
  const unsigned* active;      // device word, bit r set: right-hand side r iterates
  Spinor r, rhat, p, v, t, x;  // block fields
  int slot[kMaxBatch];         // scalar slot of each right-hand side
  double* S;                   // scalar array
  double* partial;             // [rhs][gridDim.x][3]
  double* partial2;            // [rhs][kFoldChunks][3]: first-stage sums of long partial lists
};

// Per-block partial lists longer than this (the fused dot products of the hop kernel,
// one entry per hop block) are first folded into kFoldChunks sums per right-hand side
// by a grid of blocks, so the one-block-per-RHS scalar step sums few numbers.
constexpr int kFoldChunks = 256;

template <class R>
__device__ inline cplx<R> cmuld(cplx<double> a, cplx<R> b) {
  return {(R)(a.re * b.re - a.im * b.im), (R)(a.re * b.im + a.im * b.re)};
}

// blockDim.x is a multiple of nb and so is the grid stride, hence every thread keeps
// one right-hand side k = threadIdx.x % nb for its whole loop.
template <int P, int OP>
__global__ void __launch_bounds__(kRedThreads) bicg_block_kernel(BlockBiArgs A) {
  using IO = SpinorIO<P>;
  using R = typename IO::R;
  const int k = threadIdx.x % A.nb;
  const bool act = (*A.active >> k) & 1u;
  const double* S = A.S + (size_t)A.slot[k] * kScal;
  double acc[3] = {0.0, 0.0, 0.0};
  const cplx<double> alpha{S[SC_ALPHA], S[SC_ALPHA + 1]}, omega{S[SC_OMEGA], S[SC_OMEGA + 1]},
      beta{S[SC_BETA], S[SC_BETA + 1]};
  const cplx<double> bo = {beta.re * omega.re - beta.im * omega.im, beta.re * omega.im + beta.im * omega.re};
  const int n = A.vh * A.nb;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    cplx<R> a[12], b[12], c[12];
    if (OP == OP_DOT_RHAT_R || OP == OP_DOT_RHAT_V) {
      IO::load(A.rhat.data, A.rhat.norm, n, s, a);
      if (OP == OP_DOT_RHAT_R)
        IO::load(A.r.data, A.r.norm, n, s, b);
      else
        IO::load(A.v.data, A.v.norm, n, s, b);
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        acc[0] += (double)a[q].re * b[q].re + (double)a[q].im * b[q].im;
        acc[1] += (double)a[q].re * b[q].im - (double)a[q].im * b[q].re;
      }
    } else if (OP == OP_P_UPDATE) {
      if (!act) continue;
      IO::load(A.r.data, A.r.norm, n, s, a);
      IO::load(A.p.data, A.p.norm, n, s, b);
      IO::load(A.v.data, A.v.norm, n, s, c);
#pragma unroll
      for (int q = 0; q < 12; ++q) a[q] = csub(cadd(a[q], cmuld(beta, b[q])), cmuld(bo, c[q]));
      IO::store(A.p.data, A.p.norm, n, s, a);
    } else if (OP == OP_S_UPDATE) {
      if (!act) continue;
      IO::load(A.r.data, A.r.norm, n, s, a);
      IO::load(A.v.data, A.v.norm, n, s, b);
#pragma unroll
      for (int q = 0; q < 12; ++q) a[q] = csub(a[q], cmuld(alpha, b[q]));
      IO::store(A.r.data, A.r.norm, n, s, a);
    } else if (OP == OP_DOTS_T) {
      IO::load(A.t.data, A.t.norm, n, s, a);
      IO::load(A.r.data, A.r.norm, n, s, b);
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        acc[0] += (double)a[q].re * b[q].re + (double)a[q].im * b[q].im;
        acc[1] += (double)a[q].re * b[q].im - (double)a[q].im * b[q].re;
        acc[2] += (double)a[q].re * a[q].re + (double)a[q].im * a[q].im;
      }
    } else {  // OP_XR_UPDATE
      // every operand is loaded before the first store, so the loads overlap
      cplx<R> d[12];
      IO::load(A.r.data, A.r.norm, n, s, c);
      IO::load(A.rhat.data, A.rhat.norm, n, s, d);
      if (act) {
        IO::load(A.x.data, A.x.norm, n, s, a);
        IO::load(A.p.data, A.p.norm, n, s, b);
#pragma unroll
        for (int q = 0; q < 12; ++q) a[q] = cadd(a[q], cadd(cmuld(alpha, b[q]), cmuld(omega, c[q])));
        IO::load(A.t.data, A.t.norm, n, s, b);
        IO::store(A.x.data, A.x.norm, n, s, a);
#pragma unroll
        for (int q = 0; q < 12; ++q) c[q] = csub(c[q], cmuld(omega, b[q]));
        IO::store(A.r.data, A.r.norm, n, s, c);
        if (has_norm(P)) IO::load(A.r.data, A.r.norm, n, s, c);  // reduce what was stored
      }
      // ||r||^2 and, fused, the next iteration's rho' = <rhat, r>
#pragma unroll
      for (int q = 0; q < 12; ++q) b[q] = d[q];
#pragma unroll
      for (int q = 0; q < 12; ++q) {
        acc[0] += (double)c[q].re * c[q].re + (double)c[q].im * c[q].im;
        acc[1] += (double)b[q].re * c[q].re + (double)b[q].im * c[q].im;
        acc[2] += (double)b[q].re * c[q].im - (double)b[q].im * c[q].re;
      }
    }
  }
  if (OP == OP_DOT_RHAT_R || OP == OP_DOT_RHAT_V || OP == OP_DOTS_T || OP == OP_XR_UPDATE) {
    __shared__ double red[3][kRedThreads];
#pragma unroll
    for (int q = 0; q < 3; ++q) red[q][threadIdx.x] = acc[q];
    __syncthreads();
    if (threadIdx.x < A.nb) {
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
      for (int j = threadIdx.x; j < blockDim.x; j += A.nb) {
        s0 += red[0][j];
        s1 += red[1][j];
        s2 += red[2][j];
      }
      double* dst = A.partial + ((size_t)threadIdx.x * gridDim.x + blockIdx.x) * 3;
      dst[0] = s0;
      dst[1] = s1;
      dst[2] = s2;
    }
  }
}

enum ScalStep : int {
  ST_BETA = 0,   // rho' = <rhat,r>; beta = (rho'/rho)(alpha/omega); rho = rho'
  ST_ALPHA = 1,  // alpha = rho / <rhat, v>
  ST_OMEGA = 2,  // omega = <t, r> / ||t||^2
  ST_R2 = 3,     // ||r||^2, then (still iterating) ST_BETA on the fused <rhat, r>
};

// Right-hand side k stops for good, short of its tolerance, for reason `code`: it
// leaves the active mask and counts as finished for the loop; the host reads CTL_FAIL
// and SC_FAIL and solves it again with the fallback method.
__device__ inline void bicg_fail(double* s, unsigned* ctl, int k, int code) {
  const unsigned bit = 1u << k;
  s[SC_FAIL] = (double)code;
  atomicAnd(&ctl[CTL_ACTIVE], ~bit);
  atomicAnd(&ctl[CTL_PENDING], ~bit);
  atomicAnd(&ctl[CTL_INSERT], ~bit);
  atomicOr(&ctl[CTL_FAIL], bit);
  atomicOr(&ctl[CTL_DONE], bit);
  if (code == FAIL_NAN) atomicOr(&ctl[CTL_NAN], bit);
}

// A breakdown of right-hand side k: it restarts (goes pending with the restart mark;
// its reliable update then replaces the shadow residual) while it has restarts left,
// else it stops.
__device__ inline void bicg_breakdown(double* s, unsigned* ctl, int k) {
  if (s[SC_NRST] < (double)kMaxRestarts) {
    const unsigned bit = 1u << k;
    s[SC_NRST] += 1.0;
    atomicOr(&ctl[CTL_RESTART], bit);
    atomicAnd(&ctl[CTL_ACTIVE], ~bit);
    atomicOr(&ctl[CTL_PENDING], bit);
    return;
  }
  bicg_fail(s, ctl, k, FAIL_BREAKDOWN);
}

// rho' = <rhat, r> arrived: beta = (rho'/rho)(alpha/omega), rho = rho' -- or a stop on a
// non-finite or vanishing rho' (rnorm = ||r||).
__device__ inline void bicg_beta(double* s, unsigned* ctl, int k, double d0, double d1, double rnorm) {
  const double rho = sqrt(d0 * d0 + d1 * d1);
  if (!isfinite(rho)) return bicg_fail(s, ctl, k, FAIL_NAN);
  if (rho <= kBreakEps * s[SC_RHATN] * rnorm) return bicg_breakdown(s, ctl, k);
  auto cdiv = [](double ar, double ai, double br, double bi, double* cr, double* ci) {
    const double den = br * br + bi * bi;
    *cr = (ar * br + ai * bi) / den;
    *ci = (ai * br - ar * bi) / den;
  };
  double qr, qi, pr, pi;
  cdiv(d0, d1, s[SC_RHO], s[SC_RHO + 1], &qr, &qi);                           // rho'/rho
  cdiv(s[SC_ALPHA], s[SC_ALPHA + 1], s[SC_OMEGA], s[SC_OMEGA + 1], &pr, &pi);  // alpha/omega
  s[SC_BETA] = qr * pr - qi * pi;
  s[SC_BETA + 1] = qr * pi + qi * pr;
  s[SC_RHO] = d0;
  s[SC_RHO + 1] = d1;
  if (!isfinite(s[SC_BETA]) || !isfinite(s[SC_BETA + 1])) bicg_fail(s, ctl, k, FAIL_NAN);
}

// First stage of a long per-block reduction: block (p, k) sums right-hand side k's
// partials of hop blocks p*chunk .. (p+1)*chunk-1 in a fixed order into
// partial2[(k * P + p) * 3 + q].
static __global__ void __launch_bounds__(256) partial_fold_kernel(const double* partial, int nblocks,
                                                                  double* partial2, int P) {
  const int p = blockIdx.x, k = blockIdx.y;
  const int chunk = (nblocks + P - 1) / P;
  const int b0 = p * chunk, b1 = min(nblocks, b0 + chunk);
  double a[3] = {0.0, 0.0, 0.0};
  for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x)
    for (int q = 0; q < 3; ++q) a[q] += partial[((size_t)k * nblocks + b) * 3 + q];
  __shared__ double red[3][256];
  for (int q = 0; q < 3; ++q) red[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; ++q) partial2[((size_t)k * P + p) * 3 + q] = red[q][0];
}

// One block per right-hand side: sum the partials (fixed order), update the scalars.
// At ST_R2 it also counts the iteration and, when ||r|| has dropped below delta times
// its value at the last reliable update or below half_tol ||b||, takes the right-hand
// side out of the active mask and marks it pending, so the iteration needs no host
// round trip until the host next looks.
// A right-hand side stops (bicg_fail) when a scalar is not finite, when BiCGStab breaks
// down (<rhat, r>, <rhat, v>, ||t|| or <t, s> numerically zero), or when `window` > 0
// iterations have passed since its FP64 true residual last fell 10x (stagnation; the
// anchor is moved by reliable_decide_kernel).
static __global__ void bicg_scalar_kernel(double* S, const int* slots, const double* partial,
                                          int nblocks, int step, unsigned* ctl, double delta,
                                          double half_tol, int window) {
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
  if (threadIdx.x != 0 || !((ctl[CTL_ACTIVE] >> k) & 1u)) return;
  double* s = S + (size_t)slots[k] * kScal;
  const double d0 = red[0][0], d1 = red[1][0], d2 = red[2][0];
  auto cdiv = [](double ar, double ai, double br, double bi, double* cr, double* ci) {
    const double den = br * br + bi * bi;
    *cr = (ar * br + ai * bi) / den;
    *ci = (ai * br - ar * bi) / den;
  };
  const double rnorm = sqrt(s[SC_R2]);  // ||r|| of the previous iteration (or update)
  if (step == ST_BETA) {
    bicg_beta(s, ctl, k, d0, d1, rnorm);
  } else if (step == ST_ALPHA) {
    const double den = sqrt(d0 * d0 + d1 * d1);
    if (!isfinite(den)) return bicg_fail(s, ctl, k, FAIL_NAN);
    if (!(den > 0.0)) return bicg_breakdown(s, ctl, k);
    cdiv(s[SC_RHO], s[SC_RHO + 1], d0, d1, &s[SC_ALPHA], &s[SC_ALPHA + 1]);
    if (!isfinite(s[SC_ALPHA]) || !isfinite(s[SC_ALPHA + 1])) return bicg_fail(s, ctl, k, FAIL_NAN);
  } else if (step == ST_OMEGA) {
    if (!isfinite(d0) || !isfinite(d1) || !isfinite(d2)) return bicg_fail(s, ctl, k, FAIL_NAN);
    if (!(d2 > 0.0) || sqrt(d0 * d0 + d1 * d1) <= kBreakEps * sqrt(d2) * rnorm)
      return bicg_breakdown(s, ctl, k);
    s[SC_OMEGA] = d0 / d2;
    s[SC_OMEGA + 1] = d1 / d2;
    s[SC_TT] = d2;
  } else {
    s[SC_R2] = d0;
    s[SC_ITS] += 1.0;
    const double rn = sqrt(d0);
    if (!isfinite(rn)) return bicg_fail(s, ctl, k, FAIL_NAN);
    if (rn < delta * s[SC_RMAX] || rn < half_tol * s[SC_BN]) {
      atomicAnd(&ctl[CTL_ACTIVE], ~(1u << k));
      atomicOr(&ctl[CTL_PENDING], 1u << k);
    } else if (window > 0 && s[SC_ITS] - s[SC_CHK_ITS] >= (double)window) {
      bicg_fail(s, ctl, k, FAIL_STALL);
    } else {  // the next iteration's beta from the fused <rhat, r>
      bicg_beta(s, ctl, k, d1, d2, rn);
    }
  }
}

// <rhat, r> of right-hand side k's slot of two block fields, per-block partials (re,
// im, 0) at partial[block * 3]; skipped unless bit k of *pred (the insert mask) is set.
template <int P>
__global__ void __launch_bounds__(kRedThreads) slot_dot_kernel(int vh, int nb, int k, Spinor a, Spinor b,
                                                              const unsigned* pred, double* partial) {
  using IO = SpinorIO<P>;
  if (pred && !((*pred >> k) & 1u)) return;
  const int n = vh * nb;
  double re = 0.0, im = 0.0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < vh; s += gridDim.x * blockDim.x) {
    cplx<typename IO::R> x[12], y[12];
    IO::load(a.data, a.norm, n, s * nb + k, x);
    IO::load(b.data, b.norm, n, s * nb + k, y);
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      re += (double)x[q].re * y[q].re + (double)x[q].im * y[q].im;
      im += (double)x[q].re * y[q].im - (double)x[q].im * y[q].re;
    }
  }
  __shared__ double red[2][kRedThreads];
  red[0][threadIdx.x] = re;
  red[1][threadIdx.x] = im;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[blockIdx.x * 3] = red[0][0];
    partial[blockIdx.x * 3 + 1] = red[1][0];
    partial[blockIdx.x * 3 + 2] = 0.0;
  }
}

// After right-hand side k's residual was re-inserted (bit k of the insert mask, or
// unconditionally when `always`): rho' = <rhat, r> from slot_dot_kernel's partials
// (fixed-order sum), then beta and rho as at ST_BETA -- or, at a restart (rhat was set
// to the same residual), rho = ||r||^2 and beta = 0.  One block of 256 threads.
static __global__ void reliable_rho_kernel(double* S, const int* slots, unsigned* ctl, int k,
                                           const double* partial, int nblocks, int always) {
  if (!always && !((ctl[CTL_INSERT] >> k) & 1u)) return;
  __shared__ double red[2][256];
  double a0 = 0.0, a1 = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    a0 += partial[b * 3];
    a1 += partial[b * 3 + 1];
  }
  red[0][threadIdx.x] = a0;
  red[1][threadIdx.x] = a1;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[0][threadIdx.x] += red[0][threadIdx.x + o];
      red[1][threadIdx.x] += red[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  double* s = S + (size_t)slots[k] * kScal;
  const unsigned bit = 1u << k;
  if (ctl[CTL_RESTART] & bit) {  // rhat was set to this residual: rho = ||r||^2, p = r next
    atomicAnd(&ctl[CTL_RESTART], ~bit);
    const double rho = red[0][0];
    if (!isfinite(rho)) return bicg_fail(s, ctl, k, FAIL_NAN);
    if (!(rho > 0.0)) return bicg_fail(s, ctl, k, FAIL_BREAKDOWN);
    s[SC_RHO] = rho;
    s[SC_RHO + 1] = 0.0;
    s[SC_BETA] = s[SC_BETA + 1] = 0.0;
    s[SC_RHATN] = sqrt(rho);
    return;
  }
  bicg_beta(s, ctl, k, red[0][0], red[1][0], sqrt(s[SC_R2]));
}

// End of right-hand side k's reliable update, after ||b - A x||^2 has landed in
// S[SC_T2]: record the true residual, move the progress anchor when it has fallen 10x,
// decide convergence, and either mark k done or arm the re-insertion of the FP64
// residual (rmax = ||r||).  One thread.
// Every decision is also appended to right-hand side k's history: hist[k * hmax + j] =
// the j-th true relative residual, hist_its[k * hmax + j] = the iterations done then.
static __global__ void reliable_decide_kernel(double* S, const int* slots, unsigned* ctl, int k,
                                              double tol, double* hist, int* hist_its, int hmax) {
  double* s = S + (size_t)slots[k] * kScal;
  const double rn = sqrt(s[SC_T2]);
  const double rel = rn / s[SC_BN];
  s[SC_TRUE] = rel;
  const int j = (int)s[SC_NUPD];
  if (j < hmax) {
    hist[(size_t)k * hmax + j] = rel;
    hist_its[(size_t)k * hmax + j] = (int)s[SC_ITS];
  }
  s[SC_NUPD] += 1.0;
  const unsigned bit = 1u << k;
  if (rn < 0.1 * s[SC_CHK_R]) {
    s[SC_CHK_R] = rn;
    s[SC_CHK_ITS] = s[SC_ITS];
  }
  if (!isfinite(rel)) {
    atomicAnd(&ctl[CTL_INSERT], ~bit);
    atomicAnd(&ctl[CTL_RESTART], ~bit);
    bicg_fail(s, ctl, k, FAIL_NAN);
    return;
  }
  if (!(rel > tol)) {  // converged
    atomicOr(&ctl[CTL_DONE], bit);
    atomicAnd(&ctl[CTL_INSERT], ~bit);
    atomicAnd(&ctl[CTL_RESTART], ~bit);
  } else {
    s[SC_RMAX] = rn;
    s[SC_R2] = s[SC_T2];
    atomicOr(&ctl[CTL_INSERT], bit);
  }
  atomicAnd(&ctl[CTL_PENDING], ~bit);
}

// After the (predicated) re-insertion: k iterates again unless it converged.
static __global__ void reliable_resume_kernel(unsigned* ctl, int k) {
  const unsigned bit = 1u << k;
  if (ctl[CTL_INSERT] & bit) {
    atomicAnd(&ctl[CTL_INSERT], ~bit);
    atomicOr(&ctl[CTL_ACTIVE], bit);
  }
}

// Conditions of the graph-driven loop (CUDA graph conditional nodes).
struct CondHandles {
  cudaGraphConditionalHandle h[kMaxBatch];
};

// IF node k (right-hand side k's reliable update) runs when k is pending.
static __global__ void reliable_conds_kernel(const unsigned* ctl, CondHandles hs, int nb) {
  const int k = threadIdx.x;
  if (k < nb) {
    const unsigned pend = ctl[CTL_PENDING] & ~ctl[CTL_DONE];
    cudaGraphSetConditional(hs.h[k], (pend >> k) & 1u);
  }
}

// WHILE node: another iteration while a right-hand side of `all` can still move and
// fewer than maxiter iterations have run.
static __global__ void loop_cond_kernel(unsigned* ctl, unsigned all, unsigned maxiter,
                                        cudaGraphConditionalHandle h) {
  const unsigned n = ctl[CTL_ITER] + 1u;
  ctl[CTL_ITER] = n;
  const unsigned live = (ctl[CTL_ACTIVE] | ctl[CTL_PENDING]) & ~ctl[CTL_DONE] & all;
  cudaGraphSetConditional(h, live != 0u && n < maxiter ? 1u : 0u);
}

// Slot k of a block field <-> a separate FP64 field.
//   mode 0: block[k] = x (rounded to the block precision)   mode 1: x += block[k]
//   mode 2: block[k] = 0
// When `pred` is given the kernel does nothing unless bit k of *pred is set.
template <int P>
__global__ void block_slot_kernel(int vh, int nb, int k, Spinor blockf, Spinor x, int mode,
                                  const unsigned* pred) {
  using RB = typename SpinorIO<P>::R;
  if (pred && !((*pred >> k) & 1u)) return;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < vh; s += gridDim.x * blockDim.x) {
    const int e = s * nb + k, n = vh * nb;
    cplx<RB> b[12];
    if (mode == 2) {
#pragma unroll
      for (int q = 0; q < 12; ++q) b[q] = {(RB)0, (RB)0};
      SpinorIO<P>::store(blockf.data, blockf.norm, n, e, b);
    } else if (mode == 0) {
      cplx<double> v[12];
      SpinorIO<P64>::load(x.data, x.norm, vh, s, v);
#pragma unroll
      for (int q = 0; q < 12; ++q) b[q] = {(RB)v[q].re, (RB)v[q].im};
      SpinorIO<P>::store(blockf.data, blockf.norm, n, e, b);
    } else {
      cplx<double> v[12];
      SpinorIO<P64>::load(x.data, x.norm, vh, s, v);
      SpinorIO<P>::load(blockf.data, blockf.norm, n, e, b);
#pragma unroll
      for (int q = 0; q < 12; ++q) v[q] = {v[q].re + (double)b[q].re, v[q].im + (double)b[q].im};
      SpinorIO<P64>::store(x.data, x.norm, vh, s, v);
    }
  }
}

}  // namespace qq
