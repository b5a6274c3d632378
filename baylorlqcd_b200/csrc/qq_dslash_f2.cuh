// Wilson hopping term for FP32 spinors with packed FP32x2 arithmetic (sm_100).
//
// SpinorIO<P32> stores spin pairs: plane q < 3 is colour q of spins (0, 1), plane
// q >= 3 colour q - 3 of spins (2, 3), as (a.re, b.re, a.im, b.im).  One 16-byte load
// therefore gives the pair of real parts and the pair of imaginary parts of a spin
// pair in adjacent registers.  A hop acts on a half spinor whose two rows (h0, h1) are
// built from the spin pairs (0, 1) and (2, 3) and are multiplied by the same SU(3)
// link, so every step of the hop -- projection, the link product and the
// reconstruction -- runs on (h0, h1) pairs with __ffma2_rn / __fmul2_rn: one packed
// instruction does the work of two scalar ones, and the link's entries are broadcast
// into pairs once per direction and shared by the RPT right-hand sides of the thread.
// The projector decompositions and sign patterns are those of project() /
// reconstruct_acc() in qq_dslash.cuh, regrouped by spin pair.
#pragma once
#include "qq_dslash.cuh"

namespace qq {

__device__ inline float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ inline float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ inline float2 f2swap(float2 a) { return make_float2(a.y, a.x); }
__device__ inline float2 f2bc(float a) { return make_float2(a, a); }

// Spinor as spin pairs: p[0..2] = spins (0,1) colour c, p[3..5] = spins (2,3); re and im pairs.
struct Pair12 {
  float2 re[6], im[6];
};

__device__ inline void load_pairs(const float4* f, int n, int idx, Pair12& p) {
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const float4 t = __ldg(f + (size_t)q * n + idx);
    p.re[q] = make_float2(t.x, t.y);
    p.im[q] = make_float2(t.z, t.w);
  }
}
__device__ inline void store_pairs(float4* f, int n, int idx, const Pair12& p) {
#pragma unroll
  for (int q = 0; q < 6; ++q) f[(size_t)q * n + idx] = make_float4(p.re[q].x, p.re[q].y, p.im[q].x, p.im[q].y);
}

// Matrix M (= U forward, U^+ backward) as broadcast pairs.
struct LinkPairs {
  float2 r[3][3], i[3][3];
};

template <bool FWD>
__device__ inline void link_pairs(const Su3<float>& u, LinkPairs& m) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const cplx<float> e = FWD ? u.e[a][b] : u.e[b][a];
      m.r[a][b] = f2bc(e.re);
      m.i[a][b] = f2bc(FWD ? e.im : -e.im);
    }
}

// (h0, h1) = projection of psi for direction MU and sign S (unscaled; MU = 3 omits its 2)
template <int MU, int S>
__device__ inline void project2(const Pair12& p, float2* hre, float2* him) {
  constexpr float s = (float)S;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (MU == 0) {
      hre[c] = f2fma(f2bc(s), f2swap(p.re[3 + c]), p.re[c]);
      him[c] = f2fma(f2bc(s), f2swap(p.im[3 + c]), p.im[c]);
    } else if (MU == 1) {
      hre[c] = f2fma(make_float2(s, -s), f2swap(p.im[3 + c]), p.re[c]);
      him[c] = f2fma(make_float2(-s, s), f2swap(p.re[3 + c]), p.im[c]);
    } else if (MU == 2) {
      hre[c] = f2fma(make_float2(s, -s), p.re[3 + c], p.re[c]);
      him[c] = f2fma(make_float2(s, -s), p.im[3 + c], p.im[c]);
    } else {
      hre[c] = S < 0 ? p.re[3 + c] : p.re[c];
      him[c] = S < 0 ? p.im[3 + c] : p.im[c];
    }
  }
}

// w = M h on both rows at once
__device__ inline void matvec2(const LinkPairs& m, const float2* hre, const float2* him, float2* wre,
                               float2* wim) {
  float2 nhim[3];
#pragma unroll
  for (int b = 0; b < 3; ++b) nhim[b] = f2mul(f2bc(-1.0f), him[b]);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float2 xr = f2mul(m.r[a][0], hre[0]);
    float2 xi = f2mul(m.r[a][0], him[0]);
    xr = f2fma(m.i[a][0], nhim[0], xr);
    xi = f2fma(m.i[a][0], hre[0], xi);
#pragma unroll
    for (int b = 1; b < 3; ++b) {
      xr = f2fma(m.r[a][b], hre[b], xr);
      xr = f2fma(m.i[a][b], nhim[b], xr);
      xi = f2fma(m.r[a][b], him[b], xi);
      xi = f2fma(m.i[a][b], hre[b], xi);
    }
    wre[a] = xr;
    wim[a] = xi;
  }
}

// acc += k * reconstruct(w) for direction MU and sign S
template <int MU, int S>
__device__ inline void recon2(Pair12& acc, float k, const float2* wre, const float2* wim) {
  const float ks = k * (float)S;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (MU == 3) {
      const int q = S < 0 ? 3 + c : c;
      acc.re[q] = f2fma(f2bc(k), wre[c], acc.re[q]);
      acc.im[q] = f2fma(f2bc(k), wim[c], acc.im[q]);
      continue;
    }
    acc.re[c] = f2fma(f2bc(k), wre[c], acc.re[c]);
    acc.im[c] = f2fma(f2bc(k), wim[c], acc.im[c]);
    if (MU == 0) {
      acc.re[3 + c] = f2fma(f2bc(ks), f2swap(wre[c]), acc.re[3 + c]);
      acc.im[3 + c] = f2fma(f2bc(ks), f2swap(wim[c]), acc.im[3 + c]);
    } else if (MU == 1) {
      acc.re[3 + c] = f2fma(make_float2(ks, -ks), f2swap(wim[c]), acc.re[3 + c]);
      acc.im[3 + c] = f2fma(make_float2(-ks, ks), f2swap(wre[c]), acc.im[3 + c]);
    } else {
      acc.re[3 + c] = f2fma(make_float2(ks, -ks), wre[c], acc.re[3 + c]);
      acc.im[3 + c] = f2fma(make_float2(ks, -ks), wim[c], acc.im[3 + c]);
    }
  }
}

// One direction's hops (forward or backward) for the thread's RPT right-hand sides.
template <int MU, bool FWD, int RPT>
__device__ inline void hop2(const HopArgs& a, int s, int r0, int G, const int* x, Pair12* acc) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  float sgn = 1.0f;
  if (FWD) {
    y[MU] += 1;
    if (y[MU] == a.g.n[MU]) {
      y[MU] = 0;
      sgn = a.g.bcf[MU];
    }
  } else {
    y[MU] -= 1;
    if (y[MU] < 0) {
      y[MU] = a.g.n[MU] - 1;
      sgn = a.g.bcf[MU];
    }
  }
  if (sgn == 0.0f) return;
  const int sy = site_index(a.g, y);
  const float twice = MU == 3 ? 2.0f : 1.0f;
  const float cm = twice * sgn * (FWD ? a.c.fmf[MU] : a.c.bmf[MU]);
  const float cp = twice * sgn * (FWD ? a.c.fpf[MU] : a.c.bpf[MU]);
  Su3<float> u;
  if (FWD)
    LinkIO<P32, 12>::load(a.gauge, a.g.vh, a.pout, MU, s, u);
  else
    LinkIO<P32, 12>::load(a.gauge, a.g.vh, 1 - a.pout, MU, sy, u);
  LinkPairs m;
  link_pairs<FWD>(u, m);
  const int n = a.vh_of();
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int r = r0 + k * G;
    Pair12 p;
    load_pairs(static_cast<const float4*>(a.in_base(r)), n, a.idx_of(sy, r), p);
    float2 hre[3], him[3], wre[3], wim[3];
    if (cm != 0.0f) {
      project2<MU, -1>(p, hre, him);
      matvec2(m, hre, him, wre, wim);
      recon2<MU, -1>(acc[k], cm, wre, wim);
    }
    if (cp != 0.0f) {
      project2<MU, +1>(p, hre, him);
      matvec2(m, hre, him, wre, wim);
      recon2<MU, +1>(acc[k], cp, wre, wim);
    }
  }
}

// Epilogue and store; g is the EPI_DBLE operand at (s, r), read by the caller.  Returns
// what was stored.
template <int EPI>
__device__ inline Pair12 finish2_g(const HopArgs& a, int s, int r, const Pair12& acc, const Pair12& g) {
  Pair12 o;
  if (EPI == EPI_STORE) {
    o = acc;
  } else if (EPI == EPI_TWIST) {
    const float t = a.af;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o.re[c] = f2fma(f2bc(-t), acc.re[3 + c], acc.re[c]);
      o.im[c] = f2fma(f2bc(-t), acc.im[3 + c], acc.im[c]);
      o.re[3 + c] = f2fma(f2bc(t), acc.re[c], acc.re[3 + c]);
      o.im[3 + c] = f2fma(f2bc(t), acc.im[c], acc.im[3 + c]);
    }
  } else {
    const float2 f1 = f2bc(a.f1f), f2 = f2bc(a.f2f), nf2 = f2bc(-a.f2f), nf3 = f2bc(-a.f3f);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o.re[c] = f2fma(nf3, acc.re[c], f2fma(f2, g.re[3 + c], f2mul(f1, g.re[c])));
      o.im[c] = f2fma(nf3, acc.im[c], f2fma(f2, g.im[3 + c], f2mul(f1, g.im[c])));
      o.re[3 + c] = f2fma(nf3, acc.re[3 + c], f2fma(nf2, g.re[c], f2mul(f1, g.re[3 + c])));
      o.im[3 + c] = f2fma(nf3, acc.im[3 + c], f2fma(nf2, g.im[c], f2mul(f1, g.im[3 + c])));
    }
  }
  store_pairs(static_cast<float4*>(a.blk ? a.out[0] : a.out[r]), a.vh_of(), a.idx_of(s, r), o);
  return o;
}

template <int EPI>
__device__ inline void finish2(const HopArgs& a, int s, int r, const Pair12& acc) {
  Pair12 g;
  if (EPI == EPI_DBLE)
    load_pairs(static_cast<const float4*>(a.blk ? a.aux[0] : a.aux[r]), a.vh_of(), a.idx_of(s, r), g);
  finish2_g<EPI>(a, s, r, acc, g);
}

// ---------------------------------------------------------------------------
// Software-pipelined variant (one RHS per thread): the loads of the next hop (its
// link and neighbour spinor, 9 x 16 bytes) are issued before the current hop is
// computed, so every warp keeps two hops of loads in flight instead of one.
// ---------------------------------------------------------------------------
struct HopLoad {
  float4 u[3];
  float4 p[6];
  float sgn;
};

template <int MU, bool FWD>
__device__ inline void hop_issue(const HopArgs& a, int s, int r, const int* x, HopLoad& L) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  L.sgn = 1.0f;
  if (FWD) {
    y[MU] += 1;
    if (y[MU] == a.g.n[MU]) {
      y[MU] = 0;
      L.sgn = a.g.bcf[MU];
    }
  } else {
    y[MU] -= 1;
    if (y[MU] < 0) {
      y[MU] = a.g.n[MU] - 1;
      L.sgn = a.g.bcf[MU];
    }
  }
  const int sy = site_index(a.g, y);
  const float4* gl = static_cast<const float4*>(a.gauge) +
                     (size_t)((FWD ? a.pout : 1 - a.pout) * 4 + MU) * 3 * a.g.vh + (FWD ? s : sy);
#pragma unroll
  for (int q = 0; q < 3; ++q) L.u[q] = __ldg(gl + (size_t)q * a.g.vh);
  const float4* f = static_cast<const float4*>(a.in_base(r));
  const int n = a.vh_of(), idx = a.idx_of(sy, r);
#pragma unroll
  for (int q = 0; q < 6; ++q) L.p[q] = __ldg(f + (size_t)q * n + idx);
}

template <int MU, bool FWD>
__device__ inline void hop_issue_spinor(const HopArgs& a, int s, int r, const int* x, HopLoad& L) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  L.sgn = 1.0f;
  if (FWD) {
    y[MU] += 1;
    if (y[MU] == a.g.n[MU]) {
      y[MU] = 0;
      L.sgn = a.g.bcf[MU];
    }
  } else {
    y[MU] -= 1;
    if (y[MU] < 0) {
      y[MU] = a.g.n[MU] - 1;
      L.sgn = a.g.bcf[MU];
    }
  }
  const int sy = site_index(a.g, y);
  const float4* f = static_cast<const float4*>(a.in_base(r));
  const int n = a.vh_of(), idx = a.idx_of(sy, r);
#pragma unroll
  for (int q = 0; q < 6; ++q) L.p[q] = __ldg(f + (size_t)q * n + idx);
  (void)s;
}

template <int MU, bool FWD>
__device__ inline void hop_consume(const HopArgs& a, const HopLoad& L, Pair12& acc) {
  if (L.sgn == 0.0f) return;
  const float twice = MU == 3 ? 2.0f : 1.0f;
  const float cm = twice * L.sgn * (FWD ? a.c.fmf[MU] : a.c.bmf[MU]);
  const float cp = twice * L.sgn * (FWD ? a.c.fpf[MU] : a.c.bpf[MU]);
  Su3<float> u;  // the layout of LinkIO<P32, 12>
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int c0 = 2 * q, c1 = 2 * q + 1;
    u.e[c0 / 3][c0 % 3] = {L.u[q].x, L.u[q].y};
    u.e[c1 / 3][c1 % 3] = {L.u[q].z, L.u[q].w};
  }
  reconstruct_row3(u);
  LinkPairs m;
  link_pairs<FWD>(u, m);
  Pair12 p;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    p.re[q] = make_float2(L.p[q].x, L.p[q].y);
    p.im[q] = make_float2(L.p[q].z, L.p[q].w);
  }
  float2 hre[3], him[3], wre[3], wim[3];
  if (cm != 0.0f) {
    project2<MU, -1>(p, hre, him);
    matvec2(m, hre, him, wre, wim);
    recon2<MU, -1>(acc, cm, wre, wim);
  }
  if (cp != 0.0f) {
    project2<MU, +1>(p, hre, him);
    matvec2(m, hre, him, wre, wim);
    recon2<MU, +1>(acc, cp, wre, wim);
  }
}

template <int EPI>
__global__ void __launch_bounds__(128) hop_f2p_kernel(HopArgs a) {
  const int G = a.nrhs;
  const int tx = threadIdx.x;
  const int sl = a.div_nrhs.div(tx);
  const int r = tx - sl * G;
  const int s = blockIdx.x * a.per_block + sl;
  if (s >= a.g.vh || sl >= a.per_block) return;
  Pair12 acc;
#pragma unroll
  for (int q = 0; q < 6; ++q) acc.re[q] = acc.im[q] = make_float2(0.0f, 0.0f);
  int x[4];
  site_coords(a.g, a.pout, s, x);
  HopLoad A, B;
  hop_issue<0, true>(a, s, r, x, A);
  hop_issue<0, false>(a, s, r, x, B);
  hop_consume<0, true>(a, A, acc);
  hop_issue<1, true>(a, s, r, x, A);
  hop_consume<0, false>(a, B, acc);
  hop_issue<1, false>(a, s, r, x, B);
  hop_consume<1, true>(a, A, acc);
  hop_issue<2, true>(a, s, r, x, A);
  hop_consume<1, false>(a, B, acc);
  hop_issue<2, false>(a, s, r, x, B);
  hop_consume<2, true>(a, A, acc);
  hop_issue<3, true>(a, s, r, x, A);
  hop_consume<2, false>(a, B, acc);
  hop_issue<3, false>(a, s, r, x, B);
  hop_consume<3, true>(a, A, acc);
  hop_consume<3, false>(a, B, acc);
  finish2<EPI>(a, s, r, acc);
}

// ---------------------------------------------------------------------------
// Link-staged variant for block fields (one RHS per thread, loads a hop ahead).  All
// nrhs threads of a site use the same 8 links; loading them per thread sends nrhs
// copies of every link through L1 (the largest share of the kernel's L1 traffic at
// 12 RHS).  Here the block first copies the links of its sites -- 8 hops x 3 vectors
// per site, 6 KiB at most -- into shared memory, one 16-byte vector per thread, and
// after one barrier every thread reads them as shared-memory broadcasts.
// ---------------------------------------------------------------------------
constexpr int kLinkStageSites = 16;  // sites per block at most (nrhs >= 8)

template <int EPI>
__global__ void __launch_bounds__(128) hop_f2s_kernel(HopArgs a) {
  __shared__ float4 slink[kLinkStageSites * 8 * 3];  // [site][hop][vector]
  const int G = a.nrhs;
  const int tx = threadIdx.x;
  const int s0 = blockIdx.x * a.per_block;
  // stage: entry k = (site, hop, vector); hop = 2 mu + (0 forward, 1 backward)
  for (int k = tx; k < a.per_block * 24; k += blockDim.x) {
    const int sl = k / 24, h = (k / 3) % 8, q = k % 3, mu = h >> 1;
    const int ss = s0 + sl;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ss < a.g.vh) {
      int x[4];
      site_coords(a.g, a.pout, ss, x);
      int site = ss, par = a.pout;
      if (h & 1) {  // backward hop: U_mu(x - mu) on the other parity
        x[mu] = x[mu] == 0 ? a.g.n[mu] - 1 : x[mu] - 1;
        site = site_index(a.g, x);
        par = 1 - a.pout;
      }
      const float4* gl = static_cast<const float4*>(a.gauge) + (size_t)(par * 4 + mu) * 3 * a.g.vh;
      v = __ldg(gl + (size_t)q * a.g.vh + site);
    }
    slink[k] = v;
  }
  __syncthreads();
  const int sl = a.div_nrhs.div(tx);
  const int r = tx - sl * G;
  const int s = s0 + sl;
  if (s >= a.g.vh || sl >= a.per_block) return;
  Pair12 acc;
#pragma unroll
  for (int q = 0; q < 6; ++q) acc.re[q] = acc.im[q] = make_float2(0.0f, 0.0f);
  int x[4];
  site_coords(a.g, a.pout, s, x);
  const float4* sl_link = slink + sl * 24;
  HopLoad A, B;
#define QQ_STAGED_ISSUE(MU, FWD, L)                              \
  hop_issue_spinor<MU, FWD>(a, s, r, x, L);                      \
  _Pragma("unroll") for (int q = 0; q < 3; ++q) L.u[q] = sl_link[(2 * MU + (FWD ? 0 : 1)) * 3 + q];
  QQ_STAGED_ISSUE(0, true, A);
  QQ_STAGED_ISSUE(0, false, B);
  hop_consume<0, true>(a, A, acc);
  QQ_STAGED_ISSUE(1, true, A);
  hop_consume<0, false>(a, B, acc);
  QQ_STAGED_ISSUE(1, false, B);
  hop_consume<1, true>(a, A, acc);
  QQ_STAGED_ISSUE(2, true, A);
  hop_consume<1, false>(a, B, acc);
  QQ_STAGED_ISSUE(2, false, B);
  hop_consume<2, true>(a, A, acc);
  QQ_STAGED_ISSUE(3, true, A);
  hop_consume<2, false>(a, B, acc);
  QQ_STAGED_ISSUE(3, false, B);
  hop_consume<3, true>(a, A, acc);
  hop_consume<3, false>(a, B, acc);
#undef QQ_STAGED_ISSUE
  finish2<EPI>(a, s, r, acc);
}

// ---------------------------------------------------------------------------
// Copy-ring variant for block fields.  The kernels above hold a hop's operands in
// registers: a thread issues the loads, waits a full L2 round trip, computes and only
// then issues the next hop, and at 96+ registers too few warps are resident to cover
// that wait (the hop is bound by bytes in flight per SM, not by bandwidth or
// arithmetic).  Here every thread keeps the neighbour spinors of its next D hops in
// flight as cp.async copies into its own slots of a shared-memory ring, which holds no
// registers.  The EPI_DBLE operand travels through the ring as a ninth stage.  A
// thread reads only its own ring slots, so the ring needs no barrier: the hardware
// wait on the thread's own copy groups orders it.
// Everything the nrhs threads of a site would otherwise repeat is done once per block:
// the neighbour indices and boundary signs of its sites' 8 hops (a table, before any
// copy is issued) and their 8 hop matrices (U forward, U^+ backward, third row rebuilt
// from the recon-12 rows) in shared memory.  That leaves the threads with the spin
// projection, the matrix product and the reconstruction.
// Measured alternatives: matrices stored as broadcast pairs (9 shared loads per hop,
// more registers) and 2-3 right-hand sides per thread (160+ registers, 3 blocks per
// SM) were both slower.
// Shared memory: neighbour table [site][hop] (int) and signs [site][hop] (float), raw
// recon-12 rows [site][hop][3] and matrices [site][hop][5] (18 floats in 5 16-byte
// entries, one entry of padding per site so that a warp reading three sites'
// matrices hits distinct banks), then the ring [stage][rhs][6 planes][thread]
// (conflict free: a warp reads consecutive entries).
// ---------------------------------------------------------------------------
constexpr int kF2aMatStride = 8 * 5 + 1;  // 16-byte entries per site

// MB = 1 keeps every matrix entry pre-broadcast, (re, re, im, im) in one 16-byte entry,
// 9 per hop: the SU(3) product reads a row's three entries just before it needs them
// and uses their halves as packed operands, with no broadcast instructions.
__host__ __device__ constexpr int f2a_mat_stride(int mb) { return mb ? 8 * 9 + 1 : kF2aMatStride; }

inline size_t f2a_smem_bytes(int per_block, int threads, int depth, int rpt, int mb = 0) {
  return (size_t)per_block * 8 * 8 + (size_t)16 * per_block * (24 + f2a_mat_stride(mb)) +
         (size_t)16 * depth * rpt * 6 * threads;
}

// w = M h with M's rows read from pre-broadcast shared entries e = (re, re, im, im).
__device__ inline void matvec2_rows(const float4* mp, const float2* hre, const float2* him, float2* wre,
                                    float2* wim) {
  float2 nhim[3];
#pragma unroll
  for (int b = 0; b < 3; ++b) nhim[b] = f2mul(f2bc(-1.0f), him[b]);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float4 e = mp[3 * a];
    float2 xr = f2mul(make_float2(e.x, e.y), hre[0]);
    float2 xi = f2mul(make_float2(e.x, e.y), him[0]);
    xr = f2fma(make_float2(e.z, e.w), nhim[0], xr);
    xi = f2fma(make_float2(e.z, e.w), hre[0], xi);
#pragma unroll
    for (int b = 1; b < 3; ++b) {
      e = mp[3 * a + b];
      xr = f2fma(make_float2(e.x, e.y), hre[b], xr);
      xr = f2fma(make_float2(e.z, e.w), nhim[b], xr);
      xi = f2fma(make_float2(e.x, e.y), him[b], xi);
      xi = f2fma(make_float2(e.z, e.w), hre[b], xi);
    }
    wre[a] = xr;
    wim[a] = xi;
  }
}

struct F2aShared {
  int* nbr;       // [site][hop] neighbour site index
  float* sgn;     // [site][hop] boundary factor of the hop (0 = no hop)
  float4* raw;    // [site][hop][3] recon-12 rows as stored
  float4* mat;    // [site][kF2aMatStride] hop matrices, 18 floats per hop
  float4* ring;   // [stage][rhs][6][thread]
};

// The fused dot product's operand is the EPI_DBLE operand itself (the <t, s> step of
// BiCGStab): stage 8 serves both, and stage 9 is not loaded.
__device__ inline bool f2a_dot_is_aux(const HopArgs& a) { return a.blk && a.dot_op == a.aux[0]; }

// Stage H (hops 0-7, 8 = the EPI_DBLE operand, 9 = the fused dot product's operand)
// into ring slot H % D; always one group.  Thread j of a site holds right-hand sides
// j, j + G, ..., j + (RPT - 1) G.
template <int H, int D, int EPI, int RPT>
__device__ inline void f2a_issue(const HopArgs& a, const F2aShared& sh, int s, int sl, int j, int G, int T,
                                 int tx, bool act) {
  if constexpr (H < 8 || (H >= 8 && H <= 9 && EPI == EPI_DBLE)) {
    if (act && (H != 9 || (a.dot_mode && !f2a_dot_is_aux(a)))) {
      const int site = H < 8 ? sh.nbr[sl * 8 + H] : s;
      const int n = a.vh_of();
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        const int r = j + k * G;
        const void* base = H < 8 ? a.in_base(r) : H == 8 ? (a.blk ? a.aux[0] : a.aux[r]) : a.dot_op;
        const float4* f = static_cast<const float4*>(base) + a.idx_of(site, r);
        float4* dst = sh.ring + ((H % D) * RPT + k) * 6 * T + tx;
#pragma unroll
        for (int q = 0; q < 6; ++q) cp_async16(dst + q * T, f + (size_t)q * n);
      }
    }
  }
  cp_async_commit();
}

template <int H, int D, int EPI, int RPT, int MB>
__device__ inline void f2a_run(const HopArgs& a, const F2aShared& sh, int s, int sl, int j, int G, int T,
                               int tx, Pair12* acc) {
  if constexpr (H < 8) {
    constexpr int MU = H >> 1;
    constexpr bool FWD = !(H & 1);
    cp_async_wait<D - 1>();  // stage H has landed; stages H+1 .. H+D-1 may be in flight
    const float sgn = sh.sgn[sl * 8 + H];
    if (sgn != 0.0f) {
      const float twice = MU == 3 ? 2.0f : 1.0f;
      const float cm = twice * sgn * (FWD ? a.c.fmf[MU] : a.c.bmf[MU]);
      const float cp = twice * sgn * (FWD ? a.c.fpf[MU] : a.c.bpf[MU]);
      const float4* mp = sh.mat + sl * f2a_mat_stride(MB) + H * (MB ? 9 : 5);
      LinkPairs m;
      if constexpr (MB == 0) {  // 18 floats in 5 entries, broadcast into pairs
        float me[20];
#pragma unroll
        for (int e = 0; e < 5; ++e) {
          const float4 t = mp[e];
          me[4 * e] = t.x;
          me[4 * e + 1] = t.y;
          me[4 * e + 2] = t.z;
          me[4 * e + 3] = t.w;
        }
#pragma unroll
        for (int e = 0; e < 9; ++e) {
          m.r[e / 3][e % 3] = f2bc(me[2 * e]);
          m.i[e / 3][e % 3] = f2bc(me[2 * e + 1]);
        }
      }
#pragma unroll
      for (int k = 0; k < RPT; ++k) {
        Pair12 p;
        const float4* src = sh.ring + ((H % D) * RPT + k) * 6 * T + tx;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const float4 t = src[q * T];
          p.re[q] = make_float2(t.x, t.y);
          p.im[q] = make_float2(t.z, t.w);
        }
        float2 hre[3], him[3], wre[3], wim[3];
        if (cm != 0.0f) {
          project2<MU, -1>(p, hre, him);
          if constexpr (MB == 1)
            matvec2_rows(mp, hre, him, wre, wim);
          else
            matvec2(m, hre, him, wre, wim);
          recon2<MU, -1>(acc[k], cm, wre, wim);
        }
        if (cp != 0.0f) {
          project2<MU, +1>(p, hre, him);
          if constexpr (MB == 1)
            matvec2_rows(mp, hre, him, wre, wim);
          else
            matvec2(m, hre, him, wre, wim);
          recon2<MU, +1>(acc[k], cp, wre, wim);
        }
      }
    }
    f2a_issue<H + D, D, EPI, RPT>(a, sh, s, sl, j, G, T, tx, true);
    f2a_run<H + 1, D, EPI, RPT, MB>(a, sh, s, sl, j, G, T, tx, acc);
  }
}

// Thread layout: threadIdx.x = (site-in-block) * G + j, G = nrhs / RPT threads per site.
// MINB: resident blocks per SM the register allocation is capped for (4: none; 5 and 6
// trade a few spilled registers for 25-50% more resident warps).
// MB: hop-matrix layout (0: 5 packed entries per hop, 1: 9 pre-broadcast entries).
template <int EPI, int D, int RPT, int MINB, int MB = 0>
__global__ void __launch_bounds__(128, MINB) hop_f2a_kernel(HopArgs a) {
  extern __shared__ float4 f2a_smem[];
  const int T = blockDim.x, per = a.per_block, tx = threadIdx.x;
  const int G = a.nrhs / RPT;
  F2aShared sh;
  sh.raw = f2a_smem;
  sh.mat = sh.raw + per * 24;
  sh.ring = sh.mat + per * f2a_mat_stride(MB);
  sh.nbr = reinterpret_cast<int*>(sh.ring + D * RPT * 6 * T);
  sh.sgn = reinterpret_cast<float*>(sh.nbr + per * 8);
  const int s0 = blockIdx.x * per;
  // 1. per (site, hop): neighbour index and sign; copy of the link's recon-12 rows
  for (int k = tx; k < per * 8; k += T) {
    const int sl = k >> 3, h = k & 7, mu = h >> 1;
    const int ss = min(s0 + sl, a.g.vh - 1);  // sites past the end: any valid site, never read
    int x[4];
    site_coords(a.g, a.pout, ss, x);
    const int back = h & 1;
    int y[4] = {x[0], x[1], x[2], x[3]};
    float sg = 1.0f;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      if (d != mu) continue;
      y[d] += back ? -1 : 1;
      if (y[d] < 0 || y[d] == a.g.n[d]) {
        y[d] = y[d] < 0 ? a.g.n[d] - 1 : 0;
        sg = a.g.bcf[d];
      }
    }
    const int sy = site_index(a.g, y);
    sh.nbr[k] = sy;
    sh.sgn[k] = sg;
    // forward hop: U_mu(x) on the output parity; backward: U_mu(x - mu) on the other
    const int lsite = back ? sy : ss, par = back ? 1 - a.pout : a.pout;
    const float4* gl = static_cast<const float4*>(a.gauge) + (size_t)(par * 4 + mu) * 3 * a.g.vh + lsite;
#pragma unroll
    for (int q = 0; q < 3; ++q) cp_async16(sh.raw + k * 3 + q, gl + (size_t)q * a.g.vh);
  }
  cp_async_commit();
  __syncthreads();  // the neighbour table
  const int sl = a.div_nrhs.div(tx);
  const int j = tx - sl * G;
  const int s = s0 + sl;
  const bool act = s < a.g.vh;
  f2a_issue<0, D, EPI, RPT>(a, sh, s, sl, j, G, T, tx, act);
  if constexpr (D > 1) f2a_issue<1, D, EPI, RPT>(a, sh, s, sl, j, G, T, tx, act);
  if constexpr (D > 2) f2a_issue<2, D, EPI, RPT>(a, sh, s, sl, j, G, T, tx, act);
  if constexpr (D > 3) f2a_issue<3, D, EPI, RPT>(a, sh, s, sl, j, G, T, tx, act);
  cp_async_wait<D>();  // the link rows (the oldest group) have landed ...
  __syncthreads();     // ... for every thread of the block
  // 2. hop matrices: M = U (forward) or U^+ (backward), 18 floats (re, im) row-major
  for (int k = tx; k < per * 8; k += T) {
    Su3<float> u;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float4 t = sh.raw[k * 3 + q];
      const int c0 = 2 * q, c1 = 2 * q + 1;
      u.e[c0 / 3][c0 % 3] = {t.x, t.y};
      u.e[c1 / 3][c1 % 3] = {t.z, t.w};
    }
    reconstruct_row3(u);
    float v[20];
    const bool back = k & 1;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      const int i = e / 3, c = e % 3;
      v[2 * e] = back ? u.e[c][i].re : u.e[i][c].re;
      v[2 * e + 1] = back ? -u.e[c][i].im : u.e[i][c].im;
    }
    v[18] = v[19] = 0.0f;
    if constexpr (MB == 1) {
      float4* dst = sh.mat + (k >> 3) * f2a_mat_stride(1) + (k & 7) * 9;
#pragma unroll
      for (int e = 0; e < 9; ++e) dst[e] = make_float4(v[2 * e], v[2 * e], v[2 * e + 1], v[2 * e + 1]);
    } else {
      float4* dst = sh.mat + (k >> 3) * kF2aMatStride + (k & 7) * 5;
#pragma unroll
      for (int e = 0; e < 5; ++e) dst[e] = make_float4(v[4 * e], v[4 * e + 1], v[4 * e + 2], v[4 * e + 3]);
    }
  }
  __syncthreads();
  double dsum[3] = {0.0, 0.0, 0.0};  // this thread's share of the fused dot products
  if (act) {
    Pair12 acc[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k)
#pragma unroll
      for (int q = 0; q < 6; ++q) acc[k].re[q] = acc[k].im[q] = make_float2(0.0f, 0.0f);
    f2a_run<0, D, EPI, RPT, MB>(a, sh, s, sl, j, G, T, tx, acc);
    if constexpr (EPI == EPI_DBLE) cp_async_wait<D - 2>();  // stages 8 and 9 (D >= 2)
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      Pair12 g;
      if constexpr (EPI == EPI_DBLE) {
        const float4* src = sh.ring + ((8 % D) * RPT + k) * 6 * T + tx;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const float4 t = src[q * T];
          g.re[q] = make_float2(t.x, t.y);
          g.im[q] = make_float2(t.z, t.w);
        }
      }
      const Pair12 o = finish2_g<EPI>(a, s, j + k * G, acc[k], g);
      if (a.dot_mode) {
        Pair12 w;
        const float4* wsrc = sh.ring + (((f2a_dot_is_aux(a) ? 8 : 9) % D) * RPT + k) * 6 * T + tx;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const float4 t = wsrc[q * T];
          w.re[q] = make_float2(t.x, t.y);
          w.im[q] = make_float2(t.z, t.w);
        }
        // conj(w) o (mode 1), else conj(o) w and |o|^2: the thread's 12 products are
        // summed in packed FP32, the block and grid sums in FP64
        const float sg = a.dot_mode == 1 ? 1.0f : -1.0f;  // im part flips with the order
        float2 dre = make_float2(0.f, 0.f), dim = make_float2(0.f, 0.f), dnn = make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          dre = f2fma(w.re[q], o.re[q], f2fma(w.im[q], o.im[q], dre));
          dim = f2fma(w.re[q], o.im[q], f2fma(f2bc(-1.0f), f2mul(w.im[q], o.re[q]), dim));
          dnn = f2fma(o.re[q], o.re[q], f2fma(o.im[q], o.im[q], dnn));
        }
        dsum[0] += (double)dre.x + (double)dre.y;
        dsum[1] += sg * ((double)dim.x + (double)dim.y);
        dsum[2] += (double)dnn.x + (double)dnn.y;
      }
    }
  }
  if (a.dot_mode) {  // per right-hand side over the block's sites, fixed order
    // the partial sums reuse the start of the ring (3 KB, smaller than one stage), once
    // every thread is done reading its own ring slots
    double(*dred)[128] = reinterpret_cast<double(*)[128]>(sh.ring);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 3; ++q) dred[q][tx] = dsum[q];
    __syncthreads();
    if (RPT == 1 && tx < a.nrhs) {
      double t0 = 0.0, t1 = 0.0, t2 = 0.0;
      for (int site = 0; site < per; ++site) {
        t0 += dred[0][site * G + tx];
        t1 += dred[1][site * G + tx];
        t2 += dred[2][site * G + tx];
      }
      double* dst = a.dot_part + ((size_t)tx * gridDim.x + blockIdx.x) * 3;
      dst[0] = t0;
      dst[1] = t1;
      dst[2] = t2;
    }
  }
}

// Thread layout as hop_mrhs_kernel: threadIdx.x = (site-in-block) * G + j, G = nrhs / RPT.
template <int RPT, int EPI>
__global__ void __launch_bounds__(128) hop_f2_kernel(HopArgs a) {
  const int G = a.nrhs / RPT;
  const int tx = threadIdx.x;
  const int sl = a.div_nrhs.div(tx);  // divides by G for this kernel
  const int j = tx - sl * G;
  const int s = blockIdx.x * a.per_block + sl;
  if (s >= a.g.vh || sl >= a.per_block) return;
  Pair12 acc[RPT];
#pragma unroll
  for (int k = 0; k < RPT; ++k)
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[k].re[q] = acc[k].im[q] = make_float2(0.0f, 0.0f);
  int x[4];
  site_coords(a.g, a.pout, s, x);
  hop2<0, true, RPT>(a, s, j, G, x, acc);
  hop2<0, false, RPT>(a, s, j, G, x, acc);
  hop2<1, true, RPT>(a, s, j, G, x, acc);
  hop2<1, false, RPT>(a, s, j, G, x, acc);
  hop2<2, true, RPT>(a, s, j, G, x, acc);
  hop2<2, false, RPT>(a, s, j, G, x, acc);
  hop2<3, true, RPT>(a, s, j, G, x, acc);
  hop2<3, false, RPT>(a, s, j, G, x, acc);
#pragma unroll
  for (int k = 0; k < RPT; ++k) finish2<EPI>(a, s, j + k * G, acc[k]);
}

}  // namespace qq
