// Common device definitions for the B200 qqcd solver library.
//
// HBM layout (one GPU, whole lattice resident):
//   * sites of one global checkerboard parity p (p = gblclr - 1 of the reference) are
//     numbered s = L/2 with L = x + nx*(y + ny*(z + nz*t)) the lexicographic index;
//   * a Dirac half-vector is 12 complex components (spin-major, colour-minor) per site,
//     stored component-major in 16-byte vectors ("planes"): plane q, site s at
//     [q*Vh + s].  FP64: 12 planes of double2.  FP32: 6 planes of float4 (two
//     complex per vector).  FP16 and BF16: 3 planes of 8 16-bit values + one float norm
//     per site;
//   * a gauge field stores, for each parity p and direction mu, the link U_mu(x) of
//     every site x of parity p, component-major as well: recon-18 (9 complex) or
//     recon-12 (first two rows, 6 complex; row 3 = conj(row1 x row2)).
// A warp therefore reads 32 consecutive 16-byte vectors per plane: fully coalesced.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace qq {

// Division of a non-negative 31-bit n by a divisor d fixed at set-up, by one high
// multiply and a shift (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, section 4): with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1, n / d = (umulhi(n, m) + n) >> l, exact for
// 0 <= n < 2^31 (the sum stays below 2^32).  Device integer division by a runtime
// divisor otherwise costs a conversion-pipe sequence per quotient.
struct FastDiv {
  unsigned d = 1, m = 1;
  int l = 0;
  FastDiv() = default;
  explicit FastDiv(unsigned dv) : d(dv) {
    while ((1ull << l) < dv) ++l;
    m = (unsigned)((((1ull << l) - dv) << 32) / dv) + 1u;
  }
  __host__ __device__ inline int div(int n) const {
#ifdef __CUDA_ARCH__
    return (int)((__umulhi((unsigned)n, m) + (unsigned)n) >> l);
#else
    return (int)(((unsigned)(((unsigned long long)(unsigned)n * m) >> 32) + (unsigned)n) >> l);
#endif
  }
  __host__ __device__ inline int mod(int n, int q) const { return n - q * (int)d; }
};

struct Geom {
  int n[4];        // nx, ny, nz, nt
  int vh;          // sites per parity
  int nxh;         // nx / 2
  int bc[4];       // boundary factor per direction: 1, -1, 0
  float bcf[4];    // bc as float and double (no conversion inside the kernels)
  double bcd[4];
  FastDiv div_nxh, div_ny, div_nz;
};

// Fill the derived members of g from n and bc.
inline void geom_finish(Geom& g) {
  g.vh = g.n[0] * g.n[1] * g.n[2] * g.n[3] / 2;
  g.nxh = g.n[0] / 2;
  for (int mu = 0; mu < 4; ++mu) {
    g.bcf[mu] = (float)g.bc[mu];
    g.bcd[mu] = (double)g.bc[mu];
  }
  g.div_nxh = FastDiv((unsigned)g.nxh);
  g.div_ny = FastDiv((unsigned)g.n[1]);
  g.div_nz = FastDiv((unsigned)g.n[2]);
}

// Hopping coefficients of one Hsingle call, after folding idag and the projector
// decomposition (c1 -/+ c2 gamma) = a (1 - gamma) + b (1 + gamma); float copies for
// the single-precision kernels.
struct HopCoef {
  double fm[4], fp[4];  // forward hop (x+mu): coefficient of (1-gamma), (1+gamma)
  double bm[4], bp[4];  // backward hop (x-mu): coefficient of (1-gamma), (1+gamma)
  float fmf[4], fpf[4], bmf[4], bpf[4];
};

__host__ __device__ inline void site_coords(const Geom& g, int p, int s, int* x) {
  int r = g.div_nxh.div(s);
  const int xh = s - r * g.nxh;
  int r2 = g.div_ny.div(r);
  x[1] = r - r2 * g.n[1];
  x[3] = g.div_nz.div(r2);
  x[2] = r2 - x[3] * g.n[2];
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
enum Prec : int { P64 = 0, P32 = 1, P16 = 2, PB16 = 3 };

// The 16-bit storages (FP16, BF16) keep one FP32 scale per site beside the planes.
__host__ __device__ constexpr bool has_norm(int p) { return p == P16 || p == PB16; }

// Storage precision of a method's `precision` code: 64, 32, 16 (FP16) or -16 (BF16);
// -1 for anything else.
inline int prec_of_code(int code) {
  return code == 64 ? P64 : code == 32 ? P32 : code == 16 ? P16 : code == -16 ? PB16 : -1;
}

// A Dirac half-vector in GPU layout.  For P16 and PB16 `norm` holds one float per site.
struct Spinor {
  void* data;
  float* norm;
  int prec;
};

}  // namespace qq
