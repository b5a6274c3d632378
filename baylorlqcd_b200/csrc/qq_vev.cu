// Perturbative vacuum expectation values of the loop operators (qq_twvev): twvev,
// Q/vevbleft.f90:757-2536, on the GPU.
//
// The reference expands the twisted-mass propagator in the hopping parameter for every
// unit source e(x, colour, spin): order n comes from order n-1 by GammaMultiply
// (:8163-8873: rotate by the twist angle, hop to the 8 neighbours with r -/+ gamma_mu),
// called at every site of the diamond shells |b|_1 = md it enumerates (:1168-1450).
// Only a few sites of each order are ever read: the shell sites of the next order, and
// x with its 8 neighbours at the end (:1583-1800).  The reference's zeroing (:2037-2227)
// covers every site its hops write, so the sources are independent.
//
// Here every (site, colour, spin) source is one task, run by one warp; one block takes
// the 12 tasks of a site at a time, its warps sharing a shared-memory copy of the links
// the site's program touches (about 280 links, loaded once per site):
//   * The host builds one gather program per lattice shape.  Level n holds the distinct
//     lattice offsets its order is read at ("slots", offsets wrapped onto the lattice,
//     so two shell offsets that meet on a small lattice share a slot).  Each target
//     slot of level n has the list of (source slot of level n-1, direction, number of
//     times the reference's shells call GammaMultiply at that source).  Hops into
//     offsets nothing reads are dropped, as their values never reach an operator.
//   * The warp keeps the orders in shared memory (one slot = 12 complex FP64, padded to
//     13 so lane-strided 16-byte loads hit distinct banks) already multiplied by the
//     rotation R, which is both what the next order's GammaMultiply rotates first and
//     the rotation the reference applies to the read sites at the end.
//   * Each lane gathers one target slot: per incoming hop, the projection (r +- gamma)
//     has rank 2, so two SU(3) products give all four spins.
//   * The operators of :1700-2025 are written in closed form (point-split J_1..J_4,
//     psibar psi, psibar gamma5 psi, and the momentum factors ffac / fas of :955-985);
//     each lane owns a few of the 140 (level, momentum, operator, slice) sums and adds
//     every task's contribution in task order.
//   * Blocks own a fixed range of sites of one time slice; a second kernel adds the
//     warp partials in a fixed order.  Results are deterministic.
// The test suite checks this against the CPU restatement of the reference's loops
// (which is itself checked against an independent full-lattice expansion).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "qq_ctx.h"

namespace qq {
namespace {

constexpr int kVevStride = 13;     // double2 per slot (12 used)
constexpr int kVevEntries = 140;   // 2 levels x 5 momenta x (12 ops at t + 2 at t - 1)
constexpr int kVevQ = 20;          // closed-form operator values per task
constexpr int kVevMaxSlot = 1023;  // slot index field of an edge

struct VevArgs {
  int n[4];
  int vh;
  const void* gauge;
  const char4* off;       // slot offsets of all levels
  const uint32_t* edge;   // src slot | right << 10 | mu << 11 | multiplicity << 13 | link slot << 21
  const int* lpk;         // link slots: offset x | y << 7 | z << 14 | t << 21 | mu << 28
  const double* mfac;     // [nx ny nz][k 0..3][ffac, fas1, fas2, fas3]
  double* part;           // [block][warp][kVevEntries]
  const int* meta;        // per-level tables, VevMeta layout
  const double* xk;       // (kappa cos(delta))^n, n = 0..6
  int sacc, tacc, qbase;  // slot bases of S[2][9], T[2] and Q within a warp's region
  const uint32_t* item;   // work items: target slot | first edge << 10 | edge count << 26
  const int* titem;       // per level: ns[n] + 1 item offsets (targets' item ranges)
  int nlink, gbytes, ngroup;  // link slots; bytes of a group's region; groups per block
  int scr;                // slot base of the work-item scratch within a group's region
  int nlev;               // 4 (nsub = 4) or 6
  int twist, fixbc;
  double cosd, sind, r;
  int sps, spc, chunks;   // sites per slice, sites per block, blocks per slice
};
constexpr int kLinkStride = 10;  // double2 per cached link (9 used)
constexpr int kVevGroupLanes = 128;  // threads running one task
constexpr int kVevMaxGroups = 3;     // tasks in flight per block (a divisor of the 12 of a site)

// Per-level integer tables in device memory (read with runtime level indices):
// base[7] | ns[7] | rbase[7] | buf[7] | fr9[3][9] (slots of x, x-x, x+x, x-y, x+y, x-z,
// x+z, x-t, x+t in levels 1, 3, 5) | fr0[3] (slot of x in levels 2, 4, 6) | flk[8]
// (link slots of U_mu(x) and U_mu(x - mu), mu = 0..3) | ibase[7], nitems[7] (work items
// of each level) | tbase[7] (offset of each level's item ranges in titem).
enum VevMeta {
  kMBase = 0, kMNs = 7, kMRbase = 14, kMBuf = 21, kMFr9 = 28, kMFr0 = 55, kMFlk = 58,
  kMIbase = 66, kMNitems = 73, kMTbase = 80, kMSize = 87
};

__device__ inline cplx<double> ld(const double2* p) {
  const double2 v = *p;
  return {v.x, v.y};
}
__device__ inline void st(double2* p, cplx<double> v) { *p = make_double2(v.re, v.im); }
__device__ inline cplx<double> cscale(double a, cplx<double> v) { return {a * v.re, a * v.im}; }
__device__ inline cplx<double> cmuli(double a, cplx<double> v) { return {-a * v.im, a * v.re}; }  // i a v

__device__ inline void cached_link(const double2* lk, int l, Su3<double>& u) {
  const double2* p = lk + (size_t)l * kLinkStride;
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const double2 t = p[q];
    u.e[q / 3][q % 3] = {t.x, t.y};
  }
}

__device__ inline void wrap_add(const VevArgs& A, const int* x, char4 o, int* c) {
  const int v0 = x[0] + o.x, v1 = x[1] + o.y, v2 = x[2] + o.z, v3 = x[3] + o.w;
  c[0] = v0 >= A.n[0] ? v0 - A.n[0] : v0;
  c[1] = v1 >= A.n[1] ? v1 - A.n[1] : v1;
  c[2] = v2 >= A.n[2] ? v2 - A.n[2] : v2;
  c[3] = v3 >= A.n[3] ? v3 - A.n[3] : v3;
}

// u.e[a][b] with a runtime index a (selects, so u stays in registers)
__device__ inline cplx<double> urow(const Su3<double>& u, int a, int b) {
  return a == 0 ? u.e[0][b] : (a == 1 ? u.e[1][b] : u.e[2][b]);
}
__device__ inline cplx<double> ucol(const Su3<double>& u, int b, int a) {
  return a == 0 ? u.e[b][0] : (a == 1 ? u.e[b][1] : u.e[b][2]);
}

// y = W h: W = U (left hop) or U^+ (right hop)
__device__ inline void su3_apply(const Su3<double>& u, bool dag, const cplx<double>* h, cplx<double>* y) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cplx<double> t{0.0, 0.0};
#pragma unroll
    for (int b = 0; b < 3; ++b) t = cadd(t, dag ? cmulconj(u.e[b][a], h[b]) : cmul(u.e[a][b], h[b]));
    y[a] = t;
  }
}

// One hop of a work item: y0 = W h0, y1 = W h1 with W = U (hop to -mu) or U^+ (hop to
// +mu), the link read element by element from the block's link cache.
__device__ inline void su3_pair(const double2* lk, bool dag, const cplx<double>* h0, const cplx<double>* h1,
                                cplx<double>* y0, cplx<double>* y1) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    y0[a] = {0.0, 0.0};
    y1[a] = {0.0, 0.0};
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double2 e = lk[3 * a + b];  // U[a][b]
      const cplx<double> u{e.x, e.y};
      if (dag) {  // (U^+)[b][a] = conj(U[a][b]) acts on h[a] into y[b]
        y0[b] = cadd(y0[b], cmulconj(u, h0[a]));
        y1[b] = cadd(y1[b], cmulconj(u, h1[a]));
      } else {
        y0[a] = cadd(y0[a], cmul(u, h0[b]));
        y1[a] = cadd(y1[a], cmul(u, h1[b]));
      }
    }
}

__device__ inline void group_sync(int grp) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(kVevGroupLanes) : "memory");
}

template <int RECON>
__global__ void __launch_bounds__(kVevMaxGroups * kVevGroupLanes) vev_sites_kernel(VevArgs A) {
  extern __shared__ double2 smem[];
  const double2* lk = smem;  // link cache [nlink][kLinkStride]
  const int grp = threadIdx.x / kVevGroupLanes, lane = threadIdx.x % kVevGroupLanes;
  double2* sm = smem + (size_t)A.nlink * kLinkStride + (size_t)grp * (A.gbytes / sizeof(double2));
  double2* scr = sm + (size_t)A.scr * kVevStride;  // work-item partial sums
  const int slice = blockIdx.x / A.chunks, chunk = blockIdx.x % A.chunks;
  const int sp0 = chunk * A.spc, sp1 = min(A.sps, sp0 + A.spc);
  const double r = A.r;
  double accE[2] = {0.0, 0.0};
  for (int sp = sp0; sp < sp1; ++sp) {
    const int x[4] = {sp % A.n[0], (sp / A.n[0]) % A.n[1], sp / (A.n[0] * A.n[1]), slice};
    __syncthreads();  // the previous site's links are no longer read
    for (int l = threadIdx.x; l < A.nlink; l += blockDim.x) {
      const int w = __ldg(A.lpk + l);
      const int mu = (w >> 28) & 3;
      int c[4];
      wrap_add(A, x, make_char4((char)(w & 127), (char)((w >> 7) & 127), (char)((w >> 14) & 127),
                                (char)((w >> 21) & 127)), c);
      const int L = c[0] + A.n[0] * (c[1] + A.n[1] * (c[2] + A.n[2] * c[3]));
      const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
      Su3<double> u;
      LinkIO<P64, RECON>::load(A.gauge, A.vh, par, mu, L >> 1, u);
#pragma unroll
      for (int qd = 0; qd < 9; ++qd)
        smem[(size_t)l * kLinkStride + qd] = make_double2(u.e[qd / 3][qd % 3].re, u.e[qd / 3][qd % 3].im);
    }
    __syncthreads();
    for (int task = grp; task < 12; task += A.ngroup) {
      const int id = task / 3, ic = task % 3;
      // level 0: R (cos(delta) e(x, ic, id))
      if (lane < 12) {
        const int d = lane / 3, c = lane % 3;
        double v = 0.0;
        if (c == ic) {
          if (d == id) v = A.cosd * A.cosd;
          else if (d == (id ^ 2)) v = (id < 2 ? A.sind : -A.sind) * A.cosd;
        }
        sm[(size_t)__ldg(A.meta + kMBuf) * kVevStride + lane] = make_double2(v, 0.0);
      }
      group_sync(grp);
      for (int n = 1; n <= A.nlev; ++n) {
        const double2* src = sm + (size_t)__ldg(A.meta + kMBuf + n - 1) * kVevStride;
        double2* dst = sm + (size_t)__ldg(A.meta + kMBuf + n) * kVevStride;
        const int ns = __ldg(A.meta + kMNs + n), bp = __ldg(A.meta + kMBase + n - 1);
        const int ni = __ldg(A.meta + kMNitems + n);
        // work items: up to K hops into one target, partial sum to the scratch slot
        if (lane < ni) {
          const uint32_t it = __ldg(A.item + __ldg(A.meta + kMIbase + n) + lane);
          const int e0 = (it >> 10) & 0xFFFF, e1 = e0 + (int)(it >> 26);
          cplx<double> acc[4][3];
#pragma unroll
          for (int d = 0; d < 4; ++d)
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[d][c] = {0.0, 0.0};
          for (int k = e0; k < e1; ++k) {
            const uint32_t e = __ldg(A.edge + k);
            const int sj = e & 1023, mu = (e >> 11) & 3;
            const bool right = (e >> 10) & 1;
            if (mu == 3 && A.fixbc) {
              const int st = x[3] + A.off[bp + sj].w;
              const int sct = st >= A.n[3] ? st - A.n[3] : st;
              if (right ? sct == A.n[3] - 1 : sct == 0) continue;
            }
            const double mult = (double)((e >> 13) & 255);
            const double2* sv = src + (size_t)sj * kVevStride;
            const double sg = right ? 1.0 : -1.0, sr = sg * r;
            cplx<double> h0[3], h1[3], y0[3], y1[3];
            if (mu == 0) {  // (gamma_1 v)_d = v_{3-d}
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                h0[c] = cadd(cscale(r, ld(sv + c)), cscale(sg, ld(sv + 9 + c)));
                h1[c] = cadd(cscale(r, ld(sv + 3 + c)), cscale(sg, ld(sv + 6 + c)));
              }
            } else if (mu == 1) {  // gamma_2 v = (-i v3, i v2, -i v1, i v0)
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                h0[c] = cadd(cscale(r, ld(sv + c)), cmuli(-sg, ld(sv + 9 + c)));
                h1[c] = cadd(cscale(r, ld(sv + 3 + c)), cmuli(sg, ld(sv + 6 + c)));
              }
            } else if (mu == 2) {  // gamma_3 v = (v2, -v3, v0, -v1)
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                h0[c] = cadd(cscale(r, ld(sv + c)), cscale(sg, ld(sv + 6 + c)));
                h1[c] = csub(cscale(r, ld(sv + 3 + c)), cscale(sg, ld(sv + 9 + c)));
              }
            } else {  // gamma_4 = diag(1, 1, -1, -1): (r + sg gamma_4) keeps spins 0,1 (r = sg) or 2,3
              const int o = (r == sg) ? 0 : 6;
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                h0[c] = cscale(2.0 * r, ld(sv + o + c));
                h1[c] = cscale(2.0 * r, ld(sv + o + 3 + c));
              }
            }
            su3_pair(lk + (size_t)(e >> 21) * kLinkStride, right, h0, h1, y0, y1);
            if (mult != 1.0)
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                y0[c] = cscale(mult, y0[c]);
                y1[c] = cscale(mult, y1[c]);
              }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              if (mu == 3) {
                if (r == sg) {
                  acc[0][c] = cadd(acc[0][c], y0[c]);
                  acc[1][c] = cadd(acc[1][c], y1[c]);
                } else {
                  acc[2][c] = cadd(acc[2][c], y0[c]);
                  acc[3][c] = cadd(acc[3][c], y1[c]);
                }
              } else {
                acc[0][c] = cadd(acc[0][c], y0[c]);
                acc[1][c] = cadd(acc[1][c], y1[c]);
                if (mu == 0) {
                  acc[2][c] = cadd(acc[2][c], cscale(sr, y1[c]));
                  acc[3][c] = cadd(acc[3][c], cscale(sr, y0[c]));
                } else if (mu == 1) {
                  acc[2][c] = cadd(acc[2][c], cmuli(-sr, y1[c]));
                  acc[3][c] = cadd(acc[3][c], cmuli(sr, y0[c]));
                } else {
                  acc[2][c] = cadd(acc[2][c], cscale(sr, y0[c]));
                  acc[3][c] = cadd(acc[3][c], cscale(-sr, y1[c]));
                }
              }
            }
          }
          double2* pv = scr + (size_t)lane * kVevStride;
#pragma unroll
          for (int d = 0; d < 4; ++d)
#pragma unroll
            for (int c = 0; c < 3; ++c) st(pv + 3 * d + c, acc[d][c]);
        }
        group_sync(grp);
        // combine: each target adds its items in order, then R
        if (lane < ns) {
          const int* tr = A.titem + __ldg(A.meta + kMTbase + n);
          const int i0 = __ldg(tr + lane), i1 = __ldg(tr + lane + 1);
          cplx<double> acc[4][3];
#pragma unroll
          for (int d = 0; d < 4; ++d)
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[d][c] = {0.0, 0.0};
          for (int i = i0; i < i1; ++i) {
            const double2* pv = scr + (size_t)i * kVevStride;
#pragma unroll
            for (int d = 0; d < 4; ++d)
#pragma unroll
              for (int c = 0; c < 3; ++c) acc[d][c] = cadd(acc[d][c], ld(pv + 3 * d + c));
          }
          double2* dv = dst + (size_t)lane * kVevStride;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            st(dv + c, csub(cscale(A.cosd, acc[0][c]), cscale(A.sind, acc[2][c])));
            st(dv + 3 + c, csub(cscale(A.cosd, acc[1][c]), cscale(A.sind, acc[3][c])));
            st(dv + 6 + c, cadd(cscale(A.cosd, acc[2][c]), cscale(A.sind, acc[0][c])));
            st(dv + 9 + c, cadd(cscale(A.cosd, acc[3][c]), cscale(A.sind, acc[1][c])));
          }
        }
        group_sync(grp);
        // fold the read sites into S (odd orders) and T (even orders)
        const double xkn = __ldg(A.xk + n);
        if (n & 1) {
          const int which = n >> 1;  // 0, 1, 2 for orders 1, 3, 5
          const bool use = n == 5 || n == 3 || A.twist;
          if (use && lane < 9 * 12) {
            const int site = lane / 12, comp = lane % 12;
            const int isb = n == 5 ? 1 : 0;
            double2* s = sm + (size_t)(A.sacc + isb * 9 + site) * kVevStride + comp;
            const cplx<double> v =
                cscale(xkn, ld(dst + (size_t)__ldg(A.meta + kMFr9 + which * 9 + site) * kVevStride + comp));
            const bool first = n == 5 || n == 1 || !A.twist;
            st(s, first ? v : cadd(ld(s), v));
          }
        } else {
          const int which = (n >> 1) - 1;  // 0, 1, 2 for orders 2, 4, 6
          const bool use = n == 6 || n == 4 || A.twist;
          if (use && lane < 12) {
            const int isb = n == 6 ? 1 : 0;
            double2* s = sm + (size_t)(A.tacc + isb) * kVevStride + lane;
            const cplx<double> v = cscale(xkn, ld(dst + (size_t)__ldg(A.meta + kMFr0 + which) * kVevStride + lane));
            const bool first = n == 6 || n == 2 || !A.twist;
            st(s, first ? v : cadd(ld(s), v));
          }
        }
        group_sync(grp);
      }
      // closed-form operators: lane = isb * 10 + (rho(x), rho(x-t), J1(x), J1(x-x), J2(x),
      // J2(x-y), J3(x), J3(x-z), psibar psi, psibar gamma5 psi)
      const int nq = A.nlev == 6 ? 20 : 10;
      if (lane < nq) {
        const int isb = lane / 10, k = lane % 10;
        const double2* S = sm + (size_t)(A.sacc + isb * 9) * kVevStride;
        const double2* T = sm + (size_t)(A.tacc + isb) * kVevStride;
        cplx<double> val{0.0, 0.0};
        const double g4 = id < 2 ? 1.0 : -1.0;
        if (k == 0 || k == 1) {
          const bool left = k == 1;
          const bool off = A.fixbc && (left ? x[3] == 0 : x[3] == A.n[3] - 1);
          if (!off) {
            Su3<double> u;
            cached_link(lk, __ldg(A.meta + kMFlk + 6 + (left ? 1 : 0)), u);
            const double2* Sv = S + (size_t)(left ? 7 : 8) * kVevStride + 3 * id;
            cplx<double> t{0.0, 0.0};
  #pragma unroll
            for (int b = 0; b < 3; ++b)
              t = cadd(t, left ? cmulconj(ucol(u, b, ic), ld(Sv + b)) : cmul(ld(Sv + b), urow(u, ic, b)));
            val = cscale(left ? r + g4 : -(r - g4), t);
          }
        } else if (k < 8) {
          const int mu = (k - 2) >> 1;
          const bool left = (k & 1) == 1;
          Su3<double> u;
          cached_link(lk, __ldg(A.meta + kMFlk + 2 * mu + (left ? 1 : 0)), u);
          const int od = mu < 2 ? 3 - id : (id ^ 2);
          const double2* Sv = S + (size_t)(left ? 2 * mu + 1 : 2 * mu + 2) * kVevStride;
          cplx<double> t{0.0, 0.0};
  #pragma unroll
          for (int b = 0; b < 3; ++b) {
            const cplx<double> sd = ld(Sv + 3 * id + b), so = ld(Sv + 3 * od + b);
            // ph_1 = 1, ph_2 = -i (id even) / i (id odd), ph_3 = 1 (id even) / -1 (id odd)
            cplx<double> po;
            if (mu == 0) po = so;
            else if (mu == 1) po = cmuli((id & 1) ? 1.0 : -1.0, so);
            else po = cscale((id & 1) ? -1.0 : 1.0, so);
            const cplx<double> w = cadd(cscale(left ? r : -r, sd), po);
            t = cadd(t, left ? cmulconj(ucol(u, b, ic), w) : cmul(w, urow(u, ic, b)));
          }
          val = t;
        } else if (k == 8) {
          val = ld(T + 3 * id + ic);
        } else {
          val = cmuli(id < 2 ? -1.0 : 1.0, ld(T + 3 * (id ^ 2) + ic));
        }
        st(sm + A.qbase + lane, val);
      }
      group_sync(grp);
      // this task's share of the lane's sums
      {
        const double2* Q = sm + A.qbase;
        const int spx = x[0] + A.n[0] * (x[1] + A.n[1] * x[2]);
        const int lx = (x[0] == 0 ? A.n[0] - 1 : x[0] - 1) + A.n[0] * (x[1] + A.n[1] * x[2]);
        const int ly = x[0] + A.n[0] * ((x[1] == 0 ? A.n[1] - 1 : x[1] - 1) + A.n[1] * x[2]);
        const int lz = x[0] + A.n[0] * (x[1] + A.n[1] * (x[2] == 0 ? A.n[2] - 1 : x[2] - 1));
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int e = lane + kVevGroupLanes * i;
          if (e >= kVevEntries) break;
          const int isb = e / 70, rem = e % 70, km = rem / 14, j = rem % 14;
          if (isb == 1 && A.nlev != 6) continue;
          const double2* q = Q + isb * 10;
          double v;
          if (km == 0) {
            switch (j) {
              case 0: v = q[0].x; break;
              case 1: v = q[0].y; break;
              case 2: v = q[8].x; break;
              case 3: v = q[8].y; break;
              case 4: v = q[2].x + q[3].x; break;
              case 5: v = q[2].y + q[3].y; break;
              case 6: v = q[4].x + q[5].x; break;
              case 7: v = q[4].y + q[5].y; break;
              case 8: v = q[6].x + q[7].x; break;
              case 9: v = q[6].y + q[7].y; break;
              case 10: v = q[9].x; break;
              case 11: v = q[9].y; break;
              case 12: v = q[1].x; break;
              default: v = q[1].y; break;
            }
          } else {
            const double* mh = A.mfac + ((size_t)spx * 4 + (km - 1)) * 4;
            const double ff = mh[0];
            auto fas = [&](int site, int a) { return A.mfac[((size_t)site * 4 + (km - 1)) * 4 + a]; };
            switch (j) {
              case 0: v = q[0].x * ff; break;
              case 1: v = q[0].y * ff; break;
              case 2: v = q[8].x * ff; break;
              case 3: v = q[8].y * ff; break;
              case 4: v = q[2].y * mh[3] + q[3].y * fas(lx, 3); break;
              case 5: v = q[4].y * mh[1] + q[5].y * fas(ly, 1); break;
              case 6: v = q[6].y * mh[2] + q[7].y * fas(lz, 2); break;
              case 7: v = q[2].y * mh[2] + q[3].y * fas(lx, 2); break;
              case 8: v = q[4].y * mh[3] + q[5].y * fas(ly, 3); break;
              case 9: v = q[6].y * mh[1] + q[7].y * fas(lz, 1); break;
              case 10: v = q[9].x * ff; break;
              case 11: v = q[9].y * ff; break;
              case 12: v = q[1].x * ff; break;
              default: v = q[1].y * ff; break;
            }
          }
          accE[i] += v;
        }
      }
      group_sync(grp);
    }
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int e = lane + kVevGroupLanes * i;
    if (e < kVevEntries) A.part[((size_t)blockIdx.x * A.ngroup + grp) * kVevEntries + e] = accE[i];
  }
}

// Jvev(2, nt, 6, nmom, nop) from the block partials, one thread per (t, isb, momentum,
// operator): the slice's own blocks in order, then (for the time current) the blocks
// of slice t + 1, whose x - t terms land on slice t.
__global__ void vev_reduce_kernel(const double* part, int chunks, int nt, int nlev, int nmom, double* J) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int per = 2 * nmom * 12;
  if (i >= nt * per) return;
  const int t = i / per, rem = i % per, isb = rem / (nmom * 12), km = (rem / 12) % nmom, op = rem % 12;
  if (isb == 1 && nlev != 6) return;
  const int e = isb * 70 + km * 14 + op;
  double v = 0.0;
  for (int c = 0; c < chunks; ++c) v += part[(size_t)(t * chunks + c) * kVevEntries + e];
  if (op < 2) {
    const int tn = t + 1 == nt ? 0 : t + 1;
    for (int c = 0; c < chunks; ++c) v += part[(size_t)(tn * chunks + c) * kVevEntries + e + 12];
  }
  const int lv = isb == 0 ? 3 : 5, iop = op / 2, ri = op % 2;
  J[(((size_t)iop * nmom + km) * 6 + lv) * nt * 2 + (size_t)t * 2 + ri] = v;
}

// ---- host: the gather program of one lattice shape ----

struct VevProgram {
  int dims[4] = {0, 0, 0, 0};
  std::vector<char4> off;
  std::vector<int> row;
  std::vector<uint32_t> edge;
  std::vector<int> lpk;  // link slots
  std::vector<uint32_t> item;  // work items of all levels
  std::vector<int> titem;      // per level: item offsets of its targets
  int ibase[7] = {0}, nitems[7] = {0}, tbase[7] = {0}, max_items = 0;
  int base[7], ns[7], rbase[7];
  int fr9[3][9], fr0[3], flk[8];
  int max_odd = 0, max_even = 0;
};

using Off = std::array<int, 4>;
}  // namespace

void momentum_table(const int* n, const int io[3], std::vector<double>& mf);

namespace {

template <class F>
void vev_shell(int md, F&& f) {  // the reference's shell order (:1172-1180)
  for (int bx = -md; bx <= md; ++bx)
    for (int by = -(md - std::abs(bx)); by <= md - std::abs(bx); ++by)
      for (int bz = -(md - std::abs(bx) - std::abs(by)); bz <= md - std::abs(bx) - std::abs(by); ++bz) {
        const int bt = md - std::abs(bx) - std::abs(by) - std::abs(bz);
        f(Off{bx, by, bz, bt});
        if (bt != 0) f(Off{bx, by, bz, -bt});
      }
}

int build_vev_program(const int* dims, VevProgram& P) {
  for (int d = 0; d < 4; ++d)
    if (dims[d] < 3 || dims[d] > 127) return set_error(QQ_BAD_ARG, "twvev needs every extent in 3..127");
  auto wrap = [&](Off b) {
    Off o;
    for (int d = 0; d < 4; ++d) o[d] = ((b[d] % dims[d]) + dims[d]) % dims[d];
    return o;
  };
  // sources of order n (multisets of unwrapped shell offsets, :1168-1450)
  std::vector<Off> src[7];
  auto add_shell = [&](int n, int md) { vev_shell(md, [&](Off b) { src[n].push_back(b); }); };
  src[1].push_back(Off{0, 0, 0, 0});
  add_shell(2, 1);
  src[3].push_back(Off{0, 0, 0, 0});
  add_shell(3, 2);
  add_shell(4, 1);
  add_shell(4, 3);
  src[5].push_back(Off{0, 0, 0, 0});
  add_shell(5, 2);
  add_shell(6, 1);
  const Off nine[9] = {{0, 0, 0, 0}, {-1, 0, 0, 0}, {1, 0, 0, 0}, {0, -1, 0, 0}, {0, 1, 0, 0},
                       {0, 0, -1, 0}, {0, 0, 1, 0}, {0, 0, 0, -1}, {0, 0, 0, 1}};
  // slots of each level: what the next order reads, plus the final read sites
  std::vector<Off> slot[7];
  std::map<Off, int> idx[7];
  auto add_slot = [&](int n, Off b) {
    const Off o = wrap(b);
    if (!idx[n].count(o)) {
      idx[n][o] = (int)slot[n].size();
      slot[n].push_back(o);
    }
  };
  add_slot(0, Off{0, 0, 0, 0});
  for (int n = 1; n <= 6; ++n) {
    if (n < 6)
      for (const Off& b : src[n + 1]) add_slot(n, b);
    if (n & 1)
      for (const Off& b : nine) add_slot(n, b);
    else
      add_slot(n, Off{0, 0, 0, 0});
  }
  int acc = 0;
  for (int n = 0; n <= 6; ++n) {
    P.base[n] = acc;
    P.ns[n] = (int)slot[n].size();
    if (P.ns[n] > kVevMaxSlot) return set_error(QQ_BAD_ARG, "twvev: too many slots");
    for (const Off& o : slot[n]) P.off.push_back(make_char4((char)o[0], (char)o[1], (char)o[2], (char)o[3]));
    acc += P.ns[n];
    if (n >= 1) (n & 1 ? P.max_odd : P.max_even) = std::max(n & 1 ? P.max_odd : P.max_even, P.ns[n]);
  }
  // link slots: the link each hop crosses (U_mu at the target for a hop to -mu, at the
  // source for a hop to +mu), and U_mu(x), U_mu(x - mu) for the operators
  std::map<std::pair<Off, int>, int> lidx;
  auto link_slot = [&](Off o, int mu) {
    const auto key = std::make_pair(wrap(o), mu);
    const auto it = lidx.find(key);
    if (it != lidx.end()) return it->second;
    const int l = (int)P.lpk.size();
    lidx[key] = l;
    const Off w = key.first;
    P.lpk.push_back(w[0] | w[1] << 7 | w[2] << 14 | w[3] << 21 | mu << 28);
    return l;
  };
  for (int mu = 0; mu < 4; ++mu) {
    Off m{0, 0, 0, 0};
    m[mu] = -1;
    P.flk[2 * mu] = link_slot(Off{0, 0, 0, 0}, mu);
    P.flk[2 * mu + 1] = link_slot(m, mu);
  }
  // edges, grouped by target slot
  for (int n = 1; n <= 6; ++n) {
    std::map<Off, int> mult;
    for (const Off& b : src[n]) ++mult[wrap(b)];
    std::vector<std::vector<uint32_t>> in(P.ns[n]);
    for (const auto& kv : mult) {
      const auto it = idx[n - 1].find(kv.first);
      if (it == idx[n - 1].end() || kv.second > 255) return set_error(QQ_BAD_ARG, "twvev program: bad source");
      for (int mu = 0; mu < 4; ++mu)
        for (int right = 0; right < 2; ++right) {
          Off b = kv.first;
          b[mu] += right ? 1 : -1;
          const Off o = wrap(b);
          const auto jt = idx[n].find(o);
          if (jt == idx[n].end()) continue;
          const int l = link_slot(right ? kv.first : o, mu);
          if (l > 1023) return set_error(QQ_BAD_ARG, "twvev program: too many links");
          in[jt->second].push_back((uint32_t)it->second | (uint32_t)right << 10 | (uint32_t)mu << 11 |
                                   (uint32_t)kv.second << 13 | (uint32_t)l << 21);
        }
    }
    P.rbase[n] = (int)P.row.size();
    int k = (int)P.edge.size();
    for (int j = 0; j < P.ns[n]; ++j) {
      P.row.push_back(k);
      std::sort(in[j].begin(), in[j].end());
      for (uint32_t e : in[j]) P.edge.push_back(e);
      k += (int)in[j].size();
    }
    P.row.push_back(k);
    // work items: the smallest K whose items (each <= K hops into one target) fit the
    // lanes of a group
    if (P.ns[n] > kVevGroupLanes) return set_error(QQ_BAD_ARG, "twvev program: a level has too many slots");
    int K = 1;
    for (;; ++K) {
      int cnt = 0;
      for (int j = 0; j < P.ns[n]; ++j) cnt += ((int)in[j].size() + K - 1) / K;
      if (cnt <= kVevGroupLanes) break;
      if (K > 63) return set_error(QQ_BAD_ARG, "twvev program: work items do not fit");
    }
    P.ibase[n] = (int)P.item.size();
    P.tbase[n] = (int)P.titem.size();
    int e0 = P.row[P.rbase[n]];
    for (int j = 0; j < P.ns[n]; ++j) {
      P.titem.push_back((int)P.item.size() - P.ibase[n]);
      const int ne = (int)in[j].size();
      for (int q = 0; q < ne; q += K) {
        const int c = std::min(K, ne - q);
        if (e0 + q > 0xFFFF) return set_error(QQ_BAD_ARG, "twvev program: too many edges");
        P.item.push_back((uint32_t)j | (uint32_t)(e0 + q) << 10 | (uint32_t)c << 26);
      }
      e0 += ne;
    }
    P.titem.push_back((int)P.item.size() - P.ibase[n]);
    P.nitems[n] = (int)P.item.size() - P.ibase[n];
    P.max_items = std::max(P.max_items, P.nitems[n]);
  }
  for (int w = 0; w < 3; ++w) {
    for (int s = 0; s < 9; ++s) P.fr9[w][s] = idx[2 * w + 1].at(wrap(nine[s]));
    P.fr0[w] = idx[2 * w + 2].at(Off{0, 0, 0, 0});
  }
  std::memcpy(P.dims, dims, sizeof(P.dims));
  return QQ_OK;
}

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_twvev(qq_ctx* c, double kappa, double delta, const int io[3], int dobndry, int ir, int nsub,
                        int nmom, int nop, double* Jvev) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!io || !Jvev) return set_error(QQ_BAD_ARG, "null argument");
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  if (dobndry != 0 && dobndry != 1) return set_error(QQ_BAD_ARG, "dobndry must be 0 or 1");
  if (ir != 1 && ir != -1) return set_error(QQ_BAD_ARG, "ir must be 1 or -1");
  if (nmom < 1 || nmom > 5) return set_error(QQ_BAD_ARG, "nmom must be 1..5");
  if (nop < 6) return set_error(QQ_BAD_ARG, "nop must be at least 6");
  QQ_CK(cudaSetDevice(c->device));
  const int nt = c->g.n[3];
  const size_t nJ = (size_t)2 * nt * 6 * nmom * nop;
  DevBuf dJ;
  QQ_CK(dJ.alloc(sizeof(double) * nJ));
  QQ_CK(cudaMemsetAsync(dJ.p, 0, sizeof(double) * nJ, c->st));
  if (nsub == 4 || nsub == 6) {
    VevProgram P;
    QQ_TRY(build_vev_program(c->g.n, P));
    const int nx = c->g.n[0], ny = c->g.n[1], nz = c->g.n[2], nxyz = nx * ny * nz;
    // momentum factors (:955-985), at spatial sites
    std::vector<double> mf;
    momentum_table(c->g.n, io, mf);
    // block shape: groups of 128 threads, one task each, sharing one site's link cache
    int dev_smem = 0;
    QQ_CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    const int gslots = 1 + P.max_odd + P.max_even + 20 + P.max_items;
    const size_t gbytes = ((size_t)gslots * kVevStride + kVevQ) * sizeof(double2);
    const size_t lbytes = P.lpk.size() * kLinkStride * sizeof(double2);
    int ngroup = 0;
    for (int w : {kVevMaxGroups, 2, 1})
      if (lbytes + w * gbytes <= (size_t)dev_smem) {
        ngroup = w;
        break;
      }
    if (ngroup == 0) return set_error(QQ_BAD_ARG, "twvev: shared memory plan too large");
    const size_t smem = lbytes + ngroup * gbytes;
    const int sps = nxyz;
    int chunks = std::max(1, (8 * 148 + nt - 1) / nt);
    chunks = std::min(chunks, sps);
    const int spc = (sps + chunks - 1) / chunks;
    chunks = (sps + spc - 1) / spc;
    const int nblk = nt * chunks;
    const size_t b_off = P.off.size() * sizeof(char4),
                 b_edge = P.edge.size() * sizeof(uint32_t), b_mf = mf.size() * sizeof(double),
                 b_part = (size_t)nblk * ngroup * kVevEntries * sizeof(double), b_lpk = P.lpk.size() * sizeof(int),
                 b_item = P.item.size() * sizeof(uint32_t), b_titem = P.titem.size() * sizeof(int);
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    DevBuf tab;
    QQ_CK(tab.alloc(al(b_off) + al(b_edge) + al(b_mf) + al(b_part) + al(kMSize * sizeof(int)) +
                    al(7 * sizeof(double)) + al(b_lpk) + al(b_item) + al(b_titem)));
    char* p = (char*)tab.p;
    VevArgs A{};
    for (int d = 0; d < 4; ++d) A.n[d] = c->g.n[d];
    A.vh = c->g.vh;
    A.gauge = c->gauge64.p;
    A.off = (const char4*)p;
    QQ_CK(cudaMemcpyAsync(p, P.off.data(), b_off, cudaMemcpyHostToDevice, c->st));
    p += al(b_off);
    A.edge = (const uint32_t*)p;
    QQ_CK(cudaMemcpyAsync(p, P.edge.data(), b_edge, cudaMemcpyHostToDevice, c->st));
    p += al(b_edge);
    A.mfac = (const double*)p;
    QQ_CK(cudaMemcpyAsync(p, mf.data(), b_mf, cudaMemcpyHostToDevice, c->st));
    p += al(b_mf);
    A.part = (double*)p;
    p += al(b_part);
    // shared memory: level 0 | odd orders | even orders | S[2][9] | T[2] | Q
    int meta[kMSize];
    for (int n = 0; n <= 6; ++n) {
      meta[kMBase + n] = P.base[n];
      meta[kMNs + n] = P.ns[n];
      meta[kMRbase + n] = n >= 1 ? P.rbase[n] : 0;
      meta[kMBuf + n] = n == 0 ? 0 : (n & 1 ? 1 : 1 + P.max_odd);
      meta[kMIbase + n] = P.ibase[n];
      meta[kMNitems + n] = P.nitems[n];
      meta[kMTbase + n] = P.tbase[n];
    }
    std::memcpy(meta + kMFr9, P.fr9, sizeof(P.fr9));
    std::memcpy(meta + kMFr0, P.fr0, sizeof(P.fr0));
    std::memcpy(meta + kMFlk, P.flk, sizeof(P.flk));
    A.meta = (const int*)p;
    QQ_CK(cudaMemcpyAsync(p, meta, sizeof(meta), cudaMemcpyHostToDevice, c->st));
    p += al(sizeof(meta));
    A.sacc = 1 + P.max_odd + P.max_even;
    A.tacc = A.sacc + 18;
    A.scr = A.tacc + 2;
    A.qbase = (A.scr + P.max_items) * kVevStride;
    A.nlev = nsub == 6 ? 6 : 4;
    A.twist = std::fabs(delta) > 1.e-12;
    A.fixbc = dobndry == 1;
    A.cosd = std::cos(delta);
    A.sind = std::sin(delta);
    A.r = ir;
    const double xkappa = kappa * A.cosd;
    double xk[7];
    xk[0] = 1.0;
    for (int n = 1; n <= 6; ++n) xk[n] = xk[n - 1] * xkappa;
    A.xk = (const double*)p;
    QQ_CK(cudaMemcpyAsync(p, xk, sizeof(xk), cudaMemcpyHostToDevice, c->st));
    p += al(sizeof(xk));
    A.lpk = (const int*)p;
    QQ_CK(cudaMemcpyAsync(p, P.lpk.data(), b_lpk, cudaMemcpyHostToDevice, c->st));
    p += al(b_lpk);
    A.item = (const uint32_t*)p;
    QQ_CK(cudaMemcpyAsync(p, P.item.data(), b_item, cudaMemcpyHostToDevice, c->st));
    p += al(b_item);
    A.titem = (const int*)p;
    QQ_CK(cudaMemcpyAsync(p, P.titem.data(), b_titem, cudaMemcpyHostToDevice, c->st));
    A.nlink = (int)P.lpk.size();
    A.gbytes = (int)gbytes;
    A.ngroup = ngroup;
    A.sps = sps;
    A.spc = spc;
    A.chunks = chunks;
    count_launch();
    if (c->recon64 == 18) {
      QQ_CK(cudaFuncSetAttribute(vev_sites_kernel<18>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      vev_sites_kernel<18><<<nblk, kVevGroupLanes * ngroup, smem, c->st>>>(A);
    } else {
      QQ_CK(cudaFuncSetAttribute(vev_sites_kernel<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      vev_sites_kernel<12><<<nblk, kVevGroupLanes * ngroup, smem, c->st>>>(A);
    }
    QQ_CK(cudaGetLastError());
    const int nout = nt * 2 * nmom * 12;
    count_launch();
    vev_reduce_kernel<<<(nout + 127) / 128, 128, 0, c->st>>>(A.part, chunks * ngroup, nt, A.nlev, nmom,
                                                             dJ.as<double>());
    QQ_CK(cudaGetLastError());
    QQ_CK(cudaMemcpyAsync(Jvev, dJ.p, sizeof(double) * nJ, cudaMemcpyDefault, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    return QQ_OK;
  }
  QQ_CK(cudaMemcpyAsync(Jvev, dJ.p, sizeof(double) * nJ, cudaMemcpyDefault, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}
