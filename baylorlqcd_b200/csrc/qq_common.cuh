// Common device definitions for the B200 qqcd solver library.
//
// HBM layout (one GPU, whole lattice resident):
//   * sites of one global checkerboard parity p (p = gblclr - 1 of the reference) are
//     numbered s = L/2 with L = x + nx*(y + ny*(z + nz*t)) the lexicographic index;
//   * a Dirac half-vector is 12 complex components (spin-major, colour-minor) per site,
//     stored component-major in 16-byte vectors ("planes"): plane q, site s at
//     [q*Vh + s].  FP64: 12 planes of double2.  FP32: 6 planes of float4 (two
//     complex per vector).  FP16: 3 planes of 8 halves + one float norm per site;
//   * a gauge field stores, for each parity p and direction mu, the link U_mu(x) of
//     every site x of parity p, component-major as well: recon-18 (9 complex) or
//     recon-12 (first two rows, 6 complex; row 3 = conj(row1 x row2)).
// A warp therefore reads 32 consecutive 16-byte vectors per plane: fully coalesced.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace qq {

struct Geom {
  int n[4];        // nx, ny, nz, nt
  int vh;          // sites per parity
  int nxh;         // nx / 2
  int bc[4];       // boundary factor per direction: 1, -1, 0
};

// Hopping coefficients of one Hsingle call, after folding idag and the projector
// decomposition (c1 -/+ c2 gamma) = a (1 - gamma) + b (1 + gamma).
struct HopCoef {
  double fm[4], fp[4];  // forward hop (x+mu): coefficient of (1-gamma), (1+gamma)
  double bm[4], bp[4];  // backward hop (x-mu): coefficient of (1-gamma), (1+gamma)
};

__host__ __device__ inline void site_coords(const Geom& g, int p, int s, int* x) {
  const int xh = s % g.nxh;
  int r = s / g.nxh;
  x[1] = r % g.n[1];
  r /= g.n[1];
  x[2] = r % g.n[2];
  x[3] = r / g.n[2];
  x[0] = 2 * xh + ((p + x[1] + x[2] + x[3]) & 1);
}

__host__ __device__ inline int site_index(const Geom& g, const int* x) {
  return (x[0] + g.n[0] * (x[1] + g.n[1] * (x[2] + g.n[2] * x[3]))) >> 1;
}

// Reference blocked layout (G/lattice.f90 siteindex/setblk/gblchker, Q/quark.f90:70-105):
// x = 2*xb + b per direction; isite, ieo, ibleo are 1-based.
__host__ __device__ inline void ref_site(const Geom& g, const int* x, int* isite, int* ieo,
                                         int* ibleo) {
  const int xb = x[0] >> 1, yb = x[1] >> 1, zb = x[2] >> 1, tb = x[3] >> 1;
  const int bx = x[0] & 1, by = x[1] & 1, bz = x[2] & 1, bt = x[3] & 1;
  *isite = 1 + (xb >> 1) + yb * (g.n[0] >> 2) + zb * ((g.n[0] * g.n[1]) >> 3) +
           tb * ((g.n[0] * g.n[1] * g.n[2]) >> 4);
  *ieo = 1 + ((xb + yb + zb + tb) & 1);
  const int ibl = 1 + bx + 2 * by + 4 * bz + 8 * bt;
  *ibleo = 1 + ((ibl - 1) >> 1);
}

// ---------------- complex helpers ----------------
template <class R>
struct cplx {
  R re, im;
};

template <class R>
__host__ __device__ inline cplx<R> cmul(cplx<R> a, cplx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class R>
__host__ __device__ inline cplx<R> cmulconj(cplx<R> a, cplx<R> b) {  // conj(a) * b
  return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}
template <class R>
__host__ __device__ inline cplx<R> cadd(cplx<R> a, cplx<R> b) {
  return {a.re + b.re, a.im + b.im};
}
template <class R>
__host__ __device__ inline cplx<R> csub(cplx<R> a, cplx<R> b) {
  return {a.re - b.re, a.im - b.im};
}
template <class R>
__host__ __device__ inline cplx<R> cscale(R s, cplx<R> a) {
  return {s * a.re, s * a.im};
}
template <class R>
__host__ __device__ inline cplx<R> ctimesi(cplx<R> a) {  // i*a
  return {-a.im, a.re};
}
template <class R>
__host__ __device__ inline cplx<R> cconj(cplx<R> a) {
  return {a.re, -a.im};
}

// ---------------- storage precisions ----------------
enum Prec : int { P64 = 0, P32 = 1, P16 = 2 };

// A Dirac half-vector in GPU layout.  For P16 `norm` holds one float per site.
struct Spinor {
  void* data;
  float* norm;
  int prec;
};

}  // namespace qq
