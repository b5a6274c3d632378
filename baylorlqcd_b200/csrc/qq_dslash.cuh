// Wilson hopping term H_eo / H_oe (the reference's Hsingle, Q/diracops.f90:554-599,
// with mulbac :950-1159 and mulfor :1163-1391) for the B200.
//
// A thread owns one (output site, right-hand side, direction group).  For each of its
// directions it gathers the two neighbour spinors with the periodic / antiperiodic /
// fixed boundary factor folded into the hop coefficient (the MPI halo exchange of
// setvector/slidevector becomes in-kernel neighbour indexing), spin-projects them
// with (1 -/+ gamma_mu) in the reference gamma basis (so only two colour vectors are
// multiplied by the link), multiplies by U or U^dagger and accumulates in registers.
// The right-hand sides of a site occupy adjacent lanes, so each link load is one
// broadcast transaction for the whole RHS block; splitting the 8 hops over 2 or 4
// direction groups multiplies the resident warps on small lattices.  The epilogue
// fuses the twisted-mass / Schur-complement axpys of Hdouble (:264-346) and Hdbletm
// (:435-550).
#pragma once
#include "qq_fields.cuh"

namespace qq {

enum Epilogue : int {
  EPI_STORE = 0,  // out = H in
  EPI_TWIST = 1,  // out = (1 - i a gamma5) H in           (Hdbletm :483-490)
  EPI_DBLE = 2,   // out = f1*g + f2*J(g) - f3 * H in      (Hdbletm :496-514, Hdouble :340-343)
};

constexpr int kMaxRhs = 8;     // right-hand sides per launch, separate fields
constexpr int kMaxBatch = 32;  // right-hand sides per launch, one block field
constexpr int kShapeMrhs = 200;  // kernel-shape code base of hop_mrhs_kernel (200 + RPT)
constexpr int kShapeF2 = 300;    // kernel-shape code base of hop_f2_kernel (300 + RPT)
constexpr int kShapeMax = kShapeF2 + 11;  // the largest kernel-shape code

struct HopArgs {
  Geom g;
  HopCoef c;
  int pout;                    // output parity (0 = gblclr 1, 1 = gblclr 2)
  int nrhs;
  int per_block;               // sites per thread block (set by the launcher)
  FastDiv div_nrhs;            // thread -> (site, rhs) split without integer division
  int blk;                     // 1: in/out/aux[0] are RHS-interleaved block fields of nrhs
                               //    right-hand sides: element (plane q, site s, rhs r) at
                               //    q * (vh * nrhs) + s * nrhs + r
  __device__ const void* in_base(int r) const { return blk ? in[0] : in[r]; }
  __device__ const float* in_nrm(int r) const { return blk ? in_norm[0] : in_norm[r]; }
  __device__ int vh_of() const { return blk ? g.vh * nrhs : g.vh; }
  __device__ int idx_of(int s, int r) const { return blk ? s * nrhs + r : s; }
  const void* gauge;
  const void* in[kMaxRhs];
  const float* in_norm[kMaxRhs];
  void* out[kMaxRhs];
  float* out_norm[kMaxRhs];
  const void* aux[kMaxRhs];    // g of EPI_DBLE (same precision as out)
  const float* aux_norm[kMaxRhs];
  double a;                    // EPI_TWIST: 2 kappa mu
  double f1, f2, f3;           // EPI_DBLE factors
  float af, f1f, f2f, f3f;     // float copies (set by the launcher)
  // Optional dot products of the output with a block field of the same layout, fused
  // into the copy-ring kernel's epilogue (hop_f2a_kernel only): dot_mode 1 gives
  // sum conj(dot_op) out, 2 gives sum conj(out) dot_op and sum |out|^2, as per-block
  // partials dot_part[(rhs * gridDim.x + block) * 3 + q].
  const void* dot_op;
  double* dot_part;
  int dot_mode;
};

template <class R>
__device__ inline void matvec(const Su3<R>& u, const cplx<R>* h, cplx<R>* w) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cplx<R> t = cmul(u.e[a][0], h[0]);
    t = cadd(t, cmul(u.e[a][1], h[1]));
    t = cadd(t, cmul(u.e[a][2], h[2]));
    w[a] = t;
  }
}
template <class R>
__device__ inline void matvec_dag(const Su3<R>& u, const cplx<R>* h, cplx<R>* w) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cplx<R> t = cmulconj(u.e[0][a], h[0]);
    t = cadd(t, cmulconj(u.e[1][a], h[1]));
    t = cadd(t, cmulconj(u.e[2][a], h[2]));
    w[a] = t;
  }
}

// Half-spinor projection (1 + S gamma_MU) psi = reconstruct(h0, h1), MU = 0..3 for
// gamma_1..gamma_4 of Q/diracops.f90:61-71; S = -1 or +1.
template <int MU, int S, class R>
__device__ inline void project(const cplx<R>* psi, R coef, cplx<R>* h) {
  const R s = (R)S;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    cplx<R> h0, h1;
    if (MU == 0) {
      h0 = cadd(psi[0 + c], cscale(s, psi[9 + c]));
      h1 = cadd(psi[3 + c], cscale(s, psi[6 + c]));
    } else if (MU == 1) {
      h0 = csub(psi[0 + c], cscale(s, ctimesi(psi[9 + c])));
      h1 = cadd(psi[3 + c], cscale(s, ctimesi(psi[6 + c])));
    } else if (MU == 2) {
      h0 = cadd(psi[0 + c], cscale(s, psi[6 + c]));
      h1 = csub(psi[3 + c], cscale(s, psi[9 + c]));
    } else {
      if (S < 0) {
        h0 = cscale((R)2, psi[6 + c]);
        h1 = cscale((R)2, psi[9 + c]);
      } else {
        h0 = cscale((R)2, psi[0 + c]);
        h1 = cscale((R)2, psi[3 + c]);
      }
    }
    h[c] = cscale(coef, h0);
    h[3 + c] = cscale(coef, h1);
  }
}

template <int MU, int S, class R>
__device__ inline void reconstruct_acc(cplx<R>* acc, const cplx<R>* w) {
  const R s = (R)S;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const cplx<R> w0 = w[c], w1 = w[3 + c];
    if (MU == 3) {
      if (S < 0) {
        acc[6 + c] = cadd(acc[6 + c], w0);
        acc[9 + c] = cadd(acc[9 + c], w1);
      } else {
        acc[0 + c] = cadd(acc[0 + c], w0);
        acc[3 + c] = cadd(acc[3 + c], w1);
      }
      continue;
    }
    acc[0 + c] = cadd(acc[0 + c], w0);
    acc[3 + c] = cadd(acc[3 + c], w1);
    if (MU == 0) {
      acc[6 + c] = cadd(acc[6 + c], cscale(s, w1));
      acc[9 + c] = cadd(acc[9 + c], cscale(s, w0));
    } else if (MU == 1) {
      acc[6 + c] = csub(acc[6 + c], cscale(s, ctimesi(w1)));
      acc[9 + c] = cadd(acc[9 + c], cscale(s, ctimesi(w0)));
    } else {
      acc[6 + c] = cadd(acc[6 + c], cscale(s, w0));
      acc[9 + c] = csub(acc[9 + c], cscale(s, w1));
    }
  }
}

// One hop (forward or backward in direction MU) of right-hand side r at output site s.
template <int SP, int LP, int RECON, int MU, bool FWD, class R>
__device__ inline void hop(const HopArgs& a, int s, int r, const int* x, cplx<R>* acc) {
  using SIO = SpinorIO<SP>;
  using LIO = LinkIO<LP, RECON>;
  int y[4] = {x[0], x[1], x[2], x[3]};
  constexpr bool kF = sizeof(R) == 4;
  const R bcr = kF ? (R)a.g.bcf[MU] : (R)a.g.bcd[MU];  // same type: no conversion
  R sgn = (R)1;
  if (FWD) {
    y[MU] += 1;
    if (y[MU] == a.g.n[MU]) {
      y[MU] = 0;
      sgn = bcr;
    }
  } else {
    y[MU] -= 1;
    if (y[MU] < 0) {
      y[MU] = a.g.n[MU] - 1;
      sgn = bcr;
    }
  }
  if (sgn == (R)0) return;
  const int sy = site_index(a.g, y);
  const R cm = sgn * (kF ? (R)(FWD ? a.c.fmf[MU] : a.c.bmf[MU]) : (R)(FWD ? a.c.fm[MU] : a.c.bm[MU]));
  const R cp = sgn * (kF ? (R)(FWD ? a.c.fpf[MU] : a.c.bpf[MU]) : (R)(FWD ? a.c.fp[MU] : a.c.bp[MU]));
  // All right-hand sides of a site sit in adjacent lanes: this load is one
  // broadcast transaction for them, so the link crosses HBM once per RHS block.
  Su3<R> u;
  if (FWD)
    LIO::load(a.gauge, a.g.vh, a.pout, MU, s, u);
  else
    LIO::load(a.gauge, a.g.vh, 1 - a.pout, MU, sy, u);
  cplx<R> psi[12];
  SIO::load(a.in_base(r), a.in_nrm(r), a.vh_of(), a.idx_of(sy, r), psi);
  cplx<R> h[6], w[6];
  if (cm != (R)0) {
    project<MU, -1>(psi, cm, h);
    if (FWD) {
      matvec(u, h, w);
      matvec(u, h + 3, w + 3);
    } else {
      matvec_dag(u, h, w);
      matvec_dag(u, h + 3, w + 3);
    }
    reconstruct_acc<MU, -1>(acc, w);
  }
  if (cp != (R)0) {
    project<MU, +1>(psi, cp, h);
    if (FWD) {
      matvec(u, h, w);
      matvec(u, h + 3, w + 3);
    } else {
      matvec_dag(u, h, w);
      matvec_dag(u, h + 3, w + 3);
    }
    reconstruct_acc<MU, +1>(acc, w);
  }
}

// Epilogue of one (site, right-hand side): combine the accumulated hopping term with
// the twist / Schur-complement factors and store.
template <int SP, int EPI, class R>
__device__ inline void hop_finish(const HopArgs& a, int s, int r, const cplx<R>* acc) {
  using SIO = SpinorIO<SP>;
  constexpr bool kF = sizeof(R) == 4;
  cplx<R> o[12];
  if (EPI == EPI_STORE) {
#pragma unroll
    for (int c = 0; c < 12; ++c) o[c] = acc[c];
  } else if (EPI == EPI_TWIST) {
    const R t = kF ? (R)a.af : (R)a.a;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o[0 + c] = csub(acc[0 + c], cscale(t, acc[6 + c]));
      o[3 + c] = csub(acc[3 + c], cscale(t, acc[9 + c]));
      o[6 + c] = cadd(acc[6 + c], cscale(t, acc[0 + c]));
      o[9 + c] = cadd(acc[9 + c], cscale(t, acc[3 + c]));
    }
  } else {
    cplx<R> gg[12];
    SIO::load(a.blk ? a.aux[0] : a.aux[r], a.blk ? a.aux_norm[0] : a.aux_norm[r], a.vh_of(),
              a.idx_of(s, r), gg);
    const R f1 = kF ? (R)a.f1f : (R)a.f1, f2 = kF ? (R)a.f2f : (R)a.f2, f3 = kF ? (R)a.f3f : (R)a.f3;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o[0 + c] = csub(cadd(cscale(f1, gg[0 + c]), cscale(f2, gg[6 + c])), cscale(f3, acc[0 + c]));
      o[3 + c] = csub(cadd(cscale(f1, gg[3 + c]), cscale(f2, gg[9 + c])), cscale(f3, acc[3 + c]));
      o[6 + c] = csub(csub(cscale(f1, gg[6 + c]), cscale(f2, gg[0 + c])), cscale(f3, acc[6 + c]));
      o[9 + c] = csub(csub(cscale(f1, gg[9 + c]), cscale(f2, gg[3 + c])), cscale(f3, acc[9 + c]));
    }
  }
  SIO::store(a.blk ? a.out[0] : a.out[r], a.blk ? a.out_norm[0] : a.out_norm[r], a.vh_of(),
             a.idx_of(s, r), o);
}

// ---------------------------------------------------------------------------
// Several right-hand sides per thread (block fields only).  A thread owns one site
// and the RPT right-hand sides r0, r0 + G, ..., r0 + (RPT-1) G of the block
// (G = nrhs / RPT threads per site, so each plane load of a warp still covers whole
// 32-byte sectors).  Per direction it computes the neighbour index and boundary
// factor and loads and rebuilds the link once, then applies them to its RPT spinors:
// the index arithmetic, link loads and recon-12 reconstruction that dominate the
// instruction count of the one-RHS-per-thread kernel are shared RPT ways.
// ---------------------------------------------------------------------------
template <int SP, int LP, int RECON, int MU, bool FWD, int RPT, class R>
__device__ inline void hop_multi(const HopArgs& a, int s, int r0, int G, const int* x,
                                 cplx<R> (*acc)[12]) {
  using SIO = SpinorIO<SP>;
  using LIO = LinkIO<LP, RECON>;
  constexpr bool kF = sizeof(R) == 4;
  int y[4] = {x[0], x[1], x[2], x[3]};
  R sgn = (R)1;
  const R bcr = kF ? (R)a.g.bcf[MU] : (R)a.g.bcd[MU];
  if (FWD) {
    y[MU] += 1;
    if (y[MU] == a.g.n[MU]) {
      y[MU] = 0;
      sgn = bcr;
    }
  } else {
    y[MU] -= 1;
    if (y[MU] < 0) {
      y[MU] = a.g.n[MU] - 1;
      sgn = bcr;
    }
  }
  if (sgn == (R)0) return;
  const int sy = site_index(a.g, y);
  const R cm = sgn * (kF ? (R)(FWD ? a.c.fmf[MU] : a.c.bmf[MU]) : (R)(FWD ? a.c.fm[MU] : a.c.bm[MU]));
  const R cp = sgn * (kF ? (R)(FWD ? a.c.fpf[MU] : a.c.bpf[MU]) : (R)(FWD ? a.c.fp[MU] : a.c.bp[MU]));
  Su3<R> u;
  if (FWD)
    LIO::load(a.gauge, a.g.vh, a.pout, MU, s, u);
  else
    LIO::load(a.gauge, a.g.vh, 1 - a.pout, MU, sy, u);
  const int n = a.g.vh * a.nrhs;
  const int base = sy * a.nrhs + r0;
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    cplx<R> psi[12];
    SIO::load(a.in[0], a.in_norm[0], n, base + k * G, psi);
    cplx<R> h[6], w[6];
    if (cm != (R)0) {
      project<MU, -1>(psi, cm, h);
      if (FWD) {
        matvec(u, h, w);
        matvec(u, h + 3, w + 3);
      } else {
        matvec_dag(u, h, w);
        matvec_dag(u, h + 3, w + 3);
      }
      reconstruct_acc<MU, -1>(acc[k], w);
    }
    if (cp != (R)0) {
      project<MU, +1>(psi, cp, h);
      if (FWD) {
        matvec(u, h, w);
        matvec(u, h + 3, w + 3);
      } else {
        matvec_dag(u, h, w);
        matvec_dag(u, h + 3, w + 3);
      }
      reconstruct_acc<MU, +1>(acc[k], w);
    }
  }
}

// Thread layout: threadIdx.x = (site-in-block) * G + j, G = nrhs / RPT; the thread
// handles right-hand sides j, j + G, ..., j + (RPT - 1) G of its site.
template <int SP, int LP, int RECON, int RPT, int EPI>
__global__ void __launch_bounds__(128) hop_mrhs_kernel(HopArgs a) {
  using SIO = SpinorIO<SP>;
  using R = typename SIO::R;
  const int G = a.nrhs / RPT;
  const int tx = threadIdx.x;
  const int sl = a.div_nrhs.div(tx);  // div_nrhs divides by G for this kernel
  const int j = tx - sl * G;
  const int s = blockIdx.x * a.per_block + sl;
  if (s >= a.g.vh || sl >= a.per_block) return;
  cplx<R> acc[RPT][12];
#pragma unroll
  for (int k = 0; k < RPT; ++k)
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[k][c] = {(R)0, (R)0};
  int x[4];
  site_coords(a.g, a.pout, s, x);
  hop_multi<SP, LP, RECON, 0, true, RPT>(a, s, j, G, x, acc);
  hop_multi<SP, LP, RECON, 0, false, RPT>(a, s, j, G, x, acc);
  hop_multi<SP, LP, RECON, 1, true, RPT>(a, s, j, G, x, acc);
  hop_multi<SP, LP, RECON, 1, false, RPT>(a, s, j, G, x, acc);
  hop_multi<SP, LP, RECON, 2, true, RPT>(a, s, j, G, x, acc);
  hop_multi<SP, LP, RECON, 2, false, RPT>(a, s, j, G, x, acc);
  hop_multi<SP, LP, RECON, 3, true, RPT>(a, s, j, G, x, acc);
  hop_multi<SP, LP, RECON, 3, false, RPT>(a, s, j, G, x, acc);
#pragma unroll
  for (int k = 0; k < RPT; ++k) hop_finish<SP, EPI>(a, s, j + k * G, acc[k]);
}

// Thread layout: threadIdx.x = (site-in-block) * nrhs + rhs, threadIdx.y = direction
// group (TPS groups; group t applies the directions mu with mu % TPS == t).  With
// TPS > 1 the partial sums meet in shared memory and group 0 runs the epilogue.
template <int SP, int LP, int RECON, int TPS, int EPI>
__global__ void __launch_bounds__(128) hop_kernel(HopArgs a) {
  using SIO = SpinorIO<SP>;
  using R = typename SIO::R;
  static_assert(sizeof(typename LinkIO<LP, RECON>::R) == sizeof(R), "link/spinor precision");
  const int nrhs = a.nrhs;
  const int per_block = a.per_block;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int sl = a.div_nrhs.div(tx);
  const int r = tx - sl * nrhs;
  const int s = blockIdx.x * per_block + sl;
  const bool active = s < a.g.vh && sl < per_block;
  cplx<R> acc[12];
#pragma unroll
  for (int c = 0; c < 12; ++c) acc[c] = {(R)0, (R)0};
  int x[4] = {0, 0, 0, 0};
  if (active) {
    site_coords(a.g, a.pout, s, x);
    if (TPS == 1 || ty == 0) {
      hop<SP, LP, RECON, 0, true>(a, s, r, x, acc);
      hop<SP, LP, RECON, 0, false>(a, s, r, x, acc);
    }
    if (TPS == 1 || ty == (1 % TPS)) {
      hop<SP, LP, RECON, 1, true>(a, s, r, x, acc);
      hop<SP, LP, RECON, 1, false>(a, s, r, x, acc);
    }
    if (TPS == 1 || ty == (2 % TPS)) {
      hop<SP, LP, RECON, 2, true>(a, s, r, x, acc);
      hop<SP, LP, RECON, 2, false>(a, s, r, x, acc);
    }
    if (TPS == 1 || ty == (3 % TPS)) {
      hop<SP, LP, RECON, 3, true>(a, s, r, x, acc);
      hop<SP, LP, RECON, 3, false>(a, s, r, x, acc);
    }
  }
  if (TPS > 1) {
    __shared__ cplx<R> red[TPS > 1 ? 128 : 1][12];
    const int slot = ty * blockDim.x + tx;
    if (ty > 0) {
#pragma unroll
      for (int c = 0; c < 12; ++c) red[slot][c] = acc[c];
    }
    __syncthreads();
    if (ty > 0) return;
#pragma unroll
    for (int g = 1; g < TPS; ++g)
#pragma unroll
      for (int c = 0; c < 12; ++c) acc[c] = cadd(acc[c], red[g * blockDim.x + tx][c]);
  }
  if (!active) return;
  hop_finish<SP, EPI>(a, s, r, acc);
}

// ---------------------------------------------------------------------------
// Staged variant.  A thread first issues asynchronous global->shared copies
// (cp.async, 16 bytes each) of everything its 8 hops read -- the neighbour spinors
// and the links -- into its own shared-memory slots, in two commit groups (hops 0-3
// and 4-7).  It then waits for the first group (a hardware wait on its own copies,
// no spin loop, no block barrier since no thread reads another's slots), computes
// those hops from shared memory while the second group lands, and so on.  All the
// loads of a site are in flight at once, independent of register pressure, which is
// what keeps HBM busy when the lattice is too small for many resident warps.
// Slot layout: [hop][16-byte element][thread], so every warp access is conflict free.
// ---------------------------------------------------------------------------
__device__ inline void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ inline void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
// The "memory" clobbers keep the compiler from moving shared-memory accesses across
// the copies and the waits.
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int SP>
struct SlotSpinor;
template <>
struct SlotSpinor<P64> {
  __device__ static inline void load(const uint4* slot, int T, cplx<double>* v) {
#pragma unroll
    for (int c = 0; c < 12; ++c) {
      const double2 t = *reinterpret_cast<const double2*>(slot + c * T);
      v[c] = {t.x, t.y};
    }
  }
};
template <>
struct SlotSpinor<P32> {  // the spin-paired planes of SpinorIO<P32>
  __device__ static inline void load(const uint4* slot, int T, cplx<float>* v) {
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const float4 t = *reinterpret_cast<const float4*>(slot + q * T);
      const int a = p32_first(q);
      v[a] = {t.x, t.z};
      v[a + 3] = {t.y, t.w};
    }
  }
};
template <>
struct SlotSpinor<P16> {
  // slots 0..2: the halves; slot 3: the site norm in its first 4 bytes
  __device__ static inline void load(const uint4* slot, int T, cplx<float>* v) {
    const float nrm = *reinterpret_cast<const float*>(slot + 3 * T);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const uint4 t = slot[q * T];
      const __half2* h = reinterpret_cast<const __half2*>(&t);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float2 f = __half22float2(h[k]);
        v[4 * q + k] = {f.x * nrm, f.y * nrm};
      }
    }
  }
};

template <>
struct SlotSpinor<PB16> {  // as SlotSpinor<P16>, bfloat16 values
  __device__ static inline void load(const uint4* slot, int T, cplx<float>* v) {
    const float nrm = *reinterpret_cast<const float*>(slot + 3 * T);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const uint4 t = slot[q * T];
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&t);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float2 f = __bfloat1622float2(h[k]);
        v[4 * q + k] = {f.x * nrm, f.y * nrm};
      }
    }
  }
};

template <int LP, int RECON>
__device__ inline void slot_link(const uint4* slot, int T, Su3<typename LinkIO<LP, RECON>::R>& u) {
  if (LP == P64) {
    constexpr int n = RECON == 18 ? 9 : 6;
#pragma unroll
    for (int q = 0; q < n; ++q) {
      const double2 t = *reinterpret_cast<const double2*>(slot + q * T);
      reinterpret_cast<Su3<double>&>(u).e[q / 3][q % 3] = {t.x, t.y};
    }
    if (RECON == 12) reconstruct_row3(reinterpret_cast<Su3<double>&>(u));
  } else {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const float4 t = *reinterpret_cast<const float4*>(slot + q * T);
      const int c0 = 2 * q, c1 = 2 * q + 1;
      reinterpret_cast<Su3<float>&>(u).e[c0 / 3][c0 % 3] = {t.x, t.y};
      reinterpret_cast<Su3<float>&>(u).e[c1 / 3][c1 % 3] = {t.z, t.w};
    }
    reconstruct_row3(reinterpret_cast<Su3<float>&>(u));
  }
}

// Neighbour of x in direction MU (forward or backward) and its boundary factor.
template <int MU, bool FWD>
__device__ inline int neighbour(const Geom& g, const int* x, int* sgn) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  *sgn = 1;
  if (FWD) {
    y[MU] += 1;
    if (y[MU] == g.n[MU]) {
      y[MU] = 0;
      *sgn = g.bc[MU];
    }
  } else {
    y[MU] -= 1;
    if (y[MU] < 0) {
      y[MU] = g.n[MU] - 1;
      *sgn = g.bc[MU];
    }
  }
  return site_index(g, y);
}

template <int SP, int LP, int RECON>
struct StageShape {
  static constexpr int SQ = SpinorIO<SP>::planes + (has_norm(SP) ? 1 : 0);  // + norm slot
  static constexpr int LQ = LinkIO<LP, RECON>::planes;
  static constexpr int NQ = SQ + LQ;
};

template <int SP, int LP, int RECON, int MU, bool FWD>
__device__ inline void stage_hop(const HopArgs& a, uint4* slots, int T, int s, int r,
                                 const int* x) {
  using Sh = StageShape<SP, LP, RECON>;
  constexpr int H = 2 * MU + (FWD ? 0 : 1);
  int sgn;
  const int sy = neighbour<MU, FWD>(a.g, x, &sgn);
  if (sgn == 0) return;
  uint4* dst = slots + (size_t)H * Sh::NQ * T;
  const uint4* sp = static_cast<const uint4*>(a.in_base(r));
  const int vhe = a.vh_of(), iy = a.idx_of(sy, r);
#pragma unroll
  for (int q = 0; q < SpinorIO<SP>::planes; ++q) cp_async16(dst + q * T, sp + (size_t)q * vhe + iy);
  if (has_norm(SP)) cp_async4(dst + SpinorIO<SP>::planes * T, a.in_nrm(r) + iy);
  const int lp = FWD ? a.pout : 1 - a.pout;
  const int ls = FWD ? s : sy;
  const uint4* lk = static_cast<const uint4*>(a.gauge) + (size_t)(lp * 4 + MU) * Sh::LQ * a.g.vh;
#pragma unroll
  for (int q = 0; q < Sh::LQ; ++q) cp_async16(dst + (Sh::SQ + q) * T, lk + (size_t)q * a.g.vh + ls);
}

template <int SP, int LP, int RECON, int MU, bool FWD, class R>
__device__ inline void apply_hop(const HopArgs& a, const uint4* slots, int T, const int* x,
                                 cplx<R>* acc) {
  using Sh = StageShape<SP, LP, RECON>;
  constexpr int H = 2 * MU + (FWD ? 0 : 1);
  int isgn;
  (void)neighbour<MU, FWD>(a.g, x, &isgn);
  if (isgn == 0) return;
  const R sgn = (R)isgn;
  const R cm = sgn * (R)(FWD ? a.c.fm[MU] : a.c.bm[MU]);
  const R cp = sgn * (R)(FWD ? a.c.fp[MU] : a.c.bp[MU]);
  const uint4* src = slots + (size_t)H * Sh::NQ * T;
  cplx<R> psi[12];
  SlotSpinor<SP>::load(src, T, psi);
  Su3<R> u;
  slot_link<LP, RECON>(src + Sh::SQ * T, T, u);
  cplx<R> h[6], w[6];
  if (cm != (R)0) {
    project<MU, -1>(psi, cm, h);
    if (FWD) {
      matvec(u, h, w);
      matvec(u, h + 3, w + 3);
    } else {
      matvec_dag(u, h, w);
      matvec_dag(u, h + 3, w + 3);
    }
    reconstruct_acc<MU, -1>(acc, w);
  }
  if (cp != (R)0) {
    project<MU, +1>(psi, cp, h);
    if (FWD) {
      matvec(u, h, w);
      matvec(u, h + 3, w + 3);
    } else {
      matvec_dag(u, h, w);
      matvec_dag(u, h + 3, w + 3);
    }
    reconstruct_acc<MU, +1>(acc, w);
  }
}

template <int SP, class R>
__device__ inline void hop_epilogue(const HopArgs& a, int EPI, int s, int r, const cplx<R>* acc) {
  using SIO = SpinorIO<SP>;
  cplx<R> o[12];
  if (EPI == EPI_STORE) {
#pragma unroll
    for (int c = 0; c < 12; ++c) o[c] = acc[c];
  } else if (EPI == EPI_TWIST) {
    const R t = (R)a.a;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o[0 + c] = csub(acc[0 + c], cscale(t, acc[6 + c]));
      o[3 + c] = csub(acc[3 + c], cscale(t, acc[9 + c]));
      o[6 + c] = cadd(acc[6 + c], cscale(t, acc[0 + c]));
      o[9 + c] = cadd(acc[9 + c], cscale(t, acc[3 + c]));
    }
  } else {
    cplx<R> gg[12];
    SIO::load(a.blk ? a.aux[0] : a.aux[r], a.blk ? a.aux_norm[0] : a.aux_norm[r], a.vh_of(),
              a.idx_of(s, r), gg);
    const R f1 = (R)a.f1, f2 = (R)a.f2, f3 = (R)a.f3;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o[0 + c] = csub(cadd(cscale(f1, gg[0 + c]), cscale(f2, gg[6 + c])), cscale(f3, acc[0 + c]));
      o[3 + c] = csub(cadd(cscale(f1, gg[3 + c]), cscale(f2, gg[9 + c])), cscale(f3, acc[3 + c]));
      o[6 + c] = csub(csub(cscale(f1, gg[6 + c]), cscale(f2, gg[0 + c])), cscale(f3, acc[6 + c]));
      o[9 + c] = csub(csub(cscale(f1, gg[9 + c]), cscale(f2, gg[3 + c])), cscale(f3, acc[9 + c]));
    }
  }
  SIO::store(a.blk ? a.out[0] : a.out[r], a.blk ? a.out_norm[0] : a.out_norm[r], a.vh_of(),
             a.idx_of(s, r), o);
}

// blockDim.x = T threads = (T / nrhs) sites x nrhs right-hand sides; dynamic shared
// memory = 8 * NQ * T * 16 bytes.
template <int SP, int LP, int RECON, int EPI>
__global__ void __launch_bounds__(128) hop_staged_kernel(HopArgs a) {
  using R = typename SpinorIO<SP>::R;
  extern __shared__ uint4 slots[];
  const int T = blockDim.x;
  const int nrhs = a.nrhs;
  const int per_block = a.per_block;
  const int tid = threadIdx.x;
  const int sl = a.div_nrhs.div(tid);
  const int r = tid - sl * nrhs;
  const int s = blockIdx.x * per_block + sl;
  if (s >= a.g.vh || sl >= per_block) return;
  uint4* my = slots + tid;
  int x[4];
  site_coords(a.g, a.pout, s, x);
  stage_hop<SP, LP, RECON, 0, true>(a, my, T, s, r, x);
  stage_hop<SP, LP, RECON, 0, false>(a, my, T, s, r, x);
  stage_hop<SP, LP, RECON, 1, true>(a, my, T, s, r, x);
  stage_hop<SP, LP, RECON, 1, false>(a, my, T, s, r, x);
  cp_async_commit();
  stage_hop<SP, LP, RECON, 2, true>(a, my, T, s, r, x);
  stage_hop<SP, LP, RECON, 2, false>(a, my, T, s, r, x);
  stage_hop<SP, LP, RECON, 3, true>(a, my, T, s, r, x);
  stage_hop<SP, LP, RECON, 3, false>(a, my, T, s, r, x);
  cp_async_commit();
  cplx<R> acc[12];
#pragma unroll
  for (int c = 0; c < 12; ++c) acc[c] = {(R)0, (R)0};
  cp_async_wait<1>();
  apply_hop<SP, LP, RECON, 0, true>(a, my, T, x, acc);
  apply_hop<SP, LP, RECON, 0, false>(a, my, T, x, acc);
  apply_hop<SP, LP, RECON, 1, true>(a, my, T, x, acc);
  apply_hop<SP, LP, RECON, 1, false>(a, my, T, x, acc);
  cp_async_wait<0>();
  apply_hop<SP, LP, RECON, 2, true>(a, my, T, x, acc);
  apply_hop<SP, LP, RECON, 2, false>(a, my, T, x, acc);
  apply_hop<SP, LP, RECON, 3, true>(a, my, T, x, acc);
  apply_hop<SP, LP, RECON, 3, false>(a, my, T, x, acc);
  hop_epilogue<SP, R>(a, EPI, s, r, acc);
}

template <int SP, int LP, int RECON>
inline size_t staged_smem_bytes(int T) {
  return (size_t)8 * StageShape<SP, LP, RECON>::NQ * T * 16;
}

// Block shape of hop_kernel for TPS direction groups and nrhs right-hand sides.
// Sites per block: as many as fit in 128 / tps threads, reduced to a whole number of
// warps when that keeps at least half of them (12 RHS: 8 sites = 96 threads, not 120).
inline int hop_sites_per_block(int tps, int nrhs) {
  const int bx_max = 128 / tps;
  int per_block = bx_max / nrhs;
  for (int p = per_block; p >= (per_block + 1) / 2; --p)
    if ((p * nrhs) % 32 == 0) return p;
  return per_block;
}
inline void hop_block_shape(int tps, int nrhs, int vh, dim3* blk, dim3* grd) {
  const int per_block = hop_sites_per_block(tps, nrhs);
  *blk = dim3(per_block * nrhs, tps);
  *grd = dim3((vh + per_block - 1) / per_block);
}

// Host-side helper: the hop coefficients of Hsingle for action coefficients
// c1[mu] = coact(3,1,mu), c2[mu] = coact(3,2,mu) and dagger flag idag.
inline HopCoef make_hopcoef(const double* c1, const double* c2, int idag) {
  HopCoef h;
  for (int mu = 0; mu < 4; ++mu) {
    const double a = 0.5 * (c1[mu] + c2[mu]), b = 0.5 * (c1[mu] - c2[mu]);
    // forward hop: (c1 - c2 gamma) for idag=0, (c1 + c2 gamma) for idag=1
    h.fm[mu] = idag ? b : a;
    h.fp[mu] = idag ? a : b;
    // backward hop: (c1 + c2 gamma) for idag=0, (c1 - c2 gamma) for idag=1
    h.bm[mu] = idag ? a : b;
    h.bp[mu] = idag ? b : a;
    h.fmf[mu] = (float)h.fm[mu];
    h.fpf[mu] = (float)h.fp[mu];
    h.bmf[mu] = (float)h.bm[mu];
    h.bpf[mu] = (float)h.bp[mu];
  }
  return h;
}

}  // namespace qq
