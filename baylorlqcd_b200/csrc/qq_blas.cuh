// Level-1 and Krylov-basis kernels on Dirac half-vectors (GPU layout of qq_common.cuh).
//
// All reductions accumulate in FP64 whatever the storage precision, and are
// deterministic: every block writes its partial sums to a fixed slot and a second
// single-block pass adds the slots in a fixed order.  Coefficients are complex and
// may live in device memory (so solver scalars never round-trip to the host).
#pragma once
#include "qq_fields.cuh"

namespace qq {

constexpr int kRedBlocks = 592;   // 4 x 148 SMs: fixed grid for every reduction
constexpr int kRedThreads = 256;

// A complex coefficient: immediate value, or read from device memory (optionally
// negated / conjugated).
struct Coef {
  double re, im;
  const double* ptr;  // if non-null: (re, im) = sign * ptr[0..1] (conj if cj)
  double sign;
  int cj;
  __device__ inline cplx<double> get() const {
    if (!ptr) return {re, im};
    double a = ptr[0], b = ptr[1];
    if (cj) b = -b;
    return {sign * a, sign * b};
  }
};
inline Coef cimm(double re, double im = 0.0) { return Coef{re, im, nullptr, 1.0, 0}; }
inline Coef cdev(const double* p, double sign = 1.0, int cj = 0) { return Coef{0, 0, p, sign, cj}; }

template <class R>
__device__ inline cplx<R> cmulc(cplx<double> a, cplx<R> b) {
  return {(R)a.re * b.re - (R)a.im * b.im, (R)a.re * b.im + (R)a.im * b.re};
}

// ---------------------------------------------------------------------------
// block reduction of NV doubles -> partial[blockIdx.x * NV + k]
// ---------------------------------------------------------------------------
template <int NV>
__device__ inline void block_reduce_store(double* v, double* partial) {
  __shared__ double red[NV][kRedThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[k][wid] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) s += red[threadIdx.x][w];
    partial[(size_t)blockIdx.x * NV + threadIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
// Site-wise fused linear combinations with optional reductions.
//   out = a*x + b*y + c*z          (terms with null pointers are skipped)
//   red: 0 none; 1 -> ||out||^2; 2 -> <w, out> and ||out||^2 (w given)
// ---------------------------------------------------------------------------
struct LinArgs {
  int vh;
  Spinor x, y, z, out, w;
  Coef a, b, c;
  int red;
  double* partial;
};

template <int PX, int PY, int PZ, int PO>
__global__ void __launch_bounds__(kRedThreads) lincomb_kernel(LinArgs L) {
  using RO = typename SpinorIO<PO>::R;
  double acc[3] = {0.0, 0.0, 0.0};
  const cplx<double> a = L.a.get(), b = L.b.get(), c = L.c.get();
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.vh; s += gridDim.x * blockDim.x) {
    cplx<RO> o[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) o[k] = {(RO)0, (RO)0};
    if (L.x.data) {
      cplx<typename SpinorIO<PX>::R> t[12];
      SpinorIO<PX>::load(L.x.data, L.x.norm, L.vh, s, t);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        cplx<RO> tt = {(RO)t[k].re, (RO)t[k].im};
        o[k] = cadd(o[k], cmulc(a, tt));
      }
    }
    if (L.y.data) {
      cplx<typename SpinorIO<PY>::R> t[12];
      SpinorIO<PY>::load(L.y.data, L.y.norm, L.vh, s, t);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        cplx<RO> tt = {(RO)t[k].re, (RO)t[k].im};
        o[k] = cadd(o[k], cmulc(b, tt));
      }
    }
    if (L.z.data) {
      cplx<typename SpinorIO<PZ>::R> t[12];
      SpinorIO<PZ>::load(L.z.data, L.z.norm, L.vh, s, t);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        cplx<RO> tt = {(RO)t[k].re, (RO)t[k].im};
        o[k] = cadd(o[k], cmulc(c, tt));
      }
    }
    SpinorIO<PO>::store(L.out.data, L.out.norm, L.vh, s, o);
    if (L.red >= 1) {
      // reduce on the stored (rounded) values for FP16 consistency
      cplx<RO> q[12];
      if (has_norm(PO))
        SpinorIO<PO>::load(L.out.data, L.out.norm, L.vh, s, q);
      else
        for (int k = 0; k < 12; ++k) q[k] = o[k];
#pragma unroll
      for (int k = 0; k < 12; ++k) acc[0] += (double)q[k].re * q[k].re + (double)q[k].im * q[k].im;
      if (L.red == 2) {
        cplx<typename SpinorIO<PO>::R> wv[12];
        SpinorIO<PO>::load(L.w.data, L.w.norm, L.vh, s, wv);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
          acc[1] += (double)wv[k].re * q[k].re + (double)wv[k].im * q[k].im;
          acc[2] += (double)wv[k].re * q[k].im - (double)wv[k].im * q[k].re;
        }
      }
    }
  }
  if (L.red >= 1) block_reduce_store<3>(acc, L.partial);
}

// <x, y> = sum conj(x) y and ||x||^2, ||y||^2 : partial[3] = {re, im, |y|^2}
template <int PX, int PY>
__global__ void __launch_bounds__(kRedThreads) dot_kernel(int vh, Spinor x, Spinor y,
                                                          double* partial) {
  double acc[3] = {0.0, 0.0, 0.0};
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < vh; s += gridDim.x * blockDim.x) {
    cplx<typename SpinorIO<PX>::R> a[12];
    cplx<typename SpinorIO<PY>::R> b[12];
    SpinorIO<PX>::load(x.data, x.norm, vh, s, a);
    SpinorIO<PY>::load(y.data, y.norm, vh, s, b);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      const double ar = a[k].re, ai = a[k].im, br = b[k].re, bi = b[k].im;
      acc[0] += ar * br + ai * bi;
      acc[1] += ar * bi - ai * br;
      acc[2] += br * br + bi * bi;
    }
  }
  block_reduce_store<3>(acc, partial);
}

// ---------------------------------------------------------------------------
// Krylov basis kernels.  A basis is `nvec` vectors of precision PB (P64 or P32) at
// base + i * stride_elems 16-byte elements; a vector has nel = 12*vh (P64) or
// 6*vh (P32) 16-byte elements.  Element-wise indexing is used (no per-site norm).
// ---------------------------------------------------------------------------
template <int PB>
struct BasisIO;
template <>
struct BasisIO<P64> {
  using V = double2;
  static constexpr int ncpx = 1;
  // spinor component held in slot t of plane q
  __device__ static constexpr int comp(int q, int t) { return q + t; }
  __device__ static inline void ld(const V* p, size_t e, cplx<double>* c) {
    V t = p[e];
    c[0] = {t.x, t.y};
  }
  __device__ static inline void st(V* p, size_t e, const cplx<double>* c) {
    p[e] = make_double2(c[0].re, c[0].im);
  }
};
template <>
struct BasisIO<P32> {  // the spin-paired planes of SpinorIO<P32>
  using V = float4;
  static constexpr int ncpx = 2;
  __device__ static constexpr int comp(int q, int t) { return p32_first(q) + 3 * t; }
  __device__ static inline void ld(const V* p, size_t e, cplx<double>* c) {
    V t = p[e];
    c[0] = {t.x, t.z};
    c[1] = {t.y, t.w};
  }
  __device__ static inline void st(V* p, size_t e, const cplx<double>* c) {
    p[e] = make_float4((float)c[0].re, (float)c[1].re, (float)c[0].im, (float)c[1].im);
  }
};

struct BasisArgs {
  const void* base;    // vector 0
  size_t stride;       // elements between vectors
  size_t nel;          // elements per vector
};

// h[i] = <v_i, w> for i in [0, nv): grid (kRedBlocks, ceil(nv/8)); partial layout
// [(group*8 + k) * 2 + {re,im}] per block -> partial[b * (ngroups*16) + ...]
template <int PB>
__global__ void __launch_bounds__(kRedThreads) multidot_kernel(BasisArgs V, int nv,
                                                               const void* w, double* partial) {
  using IO = BasisIO<PB>;
  using T = typename IO::V;
  const int g = blockIdx.y;
  const int i0 = g * 8;
  const int ni = min(8, nv - i0);
  double acc[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;
  const T* wp = static_cast<const T*>(w);
  const T* vb = static_cast<const T*>(V.base);
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < V.nel;
       e += (size_t)gridDim.x * blockDim.x) {
    cplx<double> wc[2];
    IO::ld(wp, e, wc);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k < ni) {
        cplx<double> vc[2];
        IO::ld(vb + (size_t)(i0 + k) * V.stride, e, vc);
#pragma unroll
        for (int q = 0; q < IO::ncpx; ++q) {
          acc[2 * k] += vc[q].re * wc[q].re + vc[q].im * wc[q].im;
          acc[2 * k + 1] += vc[q].re * wc[q].im - vc[q].im * wc[q].re;
        }
      }
    }
  }
  // reduce 16 values; store at partial[(blockIdx.x * gridDim.y + g) * 16 + k]
  __shared__ double red[16][kRedThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    double x = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[k][wid] = x;
  }
  __syncthreads();
  if (threadIdx.x < 16) {
    double s = 0.0;
    for (int ww = 0; ww < kRedThreads / 32; ++ww) s += red[threadIdx.x][ww];
    partial[((size_t)blockIdx.x * gridDim.y + g) * 16 + threadIdx.x] = s;
  }
}

// w <- w - sum_i h[i] v_i  (h complex in device memory, scaled by hsign), with the
// squared norm of the result reduced to partial (3 values per block: |w|^2, 0, 0).
// If `scale_ptr` is non-null the result is additionally multiplied by
// 1/sqrt(scale_ptr[0]) (normalisation fused in), and stored to `wout`.
template <int PB>
__global__ void __launch_bounds__(kRedThreads) multiaxpy_kernel(BasisArgs V, int nv,
                                                                const double* h, double hsign,
                                                                const void* w, void* wout,
                                                                double* partial) {
  using IO = BasisIO<PB>;
  using T = typename IO::V;
  __shared__ double hs[2 * 128];
  for (int k = threadIdx.x; k < 2 * nv && k < 256; k += blockDim.x) hs[k] = hsign * h[k];
  __syncthreads();
  double acc[3] = {0.0, 0.0, 0.0};
  const T* vb = static_cast<const T*>(V.base);
  const T* wp = static_cast<const T*>(w);
  T* wo = static_cast<T*>(wout);
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < V.nel;
       e += (size_t)gridDim.x * blockDim.x) {
    cplx<double> wc[2];
    IO::ld(wp, e, wc);
    for (int i = 0; i < nv; ++i) {
      cplx<double> vc[2];
      IO::ld(vb + (size_t)i * V.stride, e, vc);
      const double hr = hs[2 * i], hi = hs[2 * i + 1];
#pragma unroll
      for (int q = 0; q < IO::ncpx; ++q) {
        wc[q].re -= hr * vc[q].re - hi * vc[q].im;
        wc[q].im -= hr * vc[q].im + hi * vc[q].re;
      }
    }
    IO::st(wo, e, wc);
#pragma unroll
    for (int q = 0; q < IO::ncpx; ++q) acc[0] += wc[q].re * wc[q].re + wc[q].im * wc[q].im;
  }
  block_reduce_store<3>(acc, partial);
}

// v <- v * s where s = 1/sqrt(nrm[0]) (device scalar), optionally writing to out.
template <int PB>
__global__ void __launch_bounds__(kRedThreads) normalize_kernel(size_t nel, const void* in,
                                                                void* out, const double* nrm2) {
  using IO = BasisIO<PB>;
  using T = typename IO::V;
  const double s = 1.0 / sqrt(nrm2[0]);
  const T* ip = static_cast<const T*>(in);
  T* op = static_cast<T*>(out);
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
       e += (size_t)gridDim.x * blockDim.x) {
    cplx<double> c[2];
    IO::ld(ip, e, c);
#pragma unroll
    for (int q = 0; q < IO::ncpx; ++q) {
      c[q].re *= s;
      c[q].im *= s;
    }
    IO::st(op, e, c);
  }
}

// In-place basis rotation: v_j <- sum_{i<nin} v_i Z(i, j) for j < nout (nout <= nin),
// Z complex column-major (ldz) in device memory.  Each thread owns one element
// index across all vectors, so the in-place update is race free.
template <int PB, int MAXOUT>
__global__ void __launch_bounds__(128) rotate_kernel(BasisArgs V, int nin, int nout,
                                                     const double* Z, int ldz) {
  using IO = BasisIO<PB>;
  using T = typename IO::V;
  extern __shared__ double zs[];  // nin * nout complex
  for (int k = threadIdx.x; k < nin * nout; k += blockDim.x) {
    const int i = k % nin, j = k / nin;
    zs[2 * k] = Z[2 * ((size_t)i + (size_t)ldz * j)];
    zs[2 * k + 1] = Z[2 * ((size_t)i + (size_t)ldz * j) + 1];
  }
  __syncthreads();
  T* vb = static_cast<T*>(const_cast<void*>(V.base));
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < V.nel;
       e += (size_t)gridDim.x * blockDim.x) {
    cplx<double> out[MAXOUT][2];
#pragma unroll
    for (int j = 0; j < MAXOUT; ++j) out[j][0] = out[j][1] = {0.0, 0.0};
    for (int i = 0; i < nin; ++i) {
      cplx<double> vc[2];
      IO::ld(vb + (size_t)i * V.stride, e, vc);
#pragma unroll
      for (int j = 0; j < MAXOUT; ++j) {
        if (j < nout) {
          const double zr = zs[2 * (i + nin * j)], zi = zs[2 * (i + nin * j) + 1];
#pragma unroll
          for (int q = 0; q < IO::ncpx; ++q) {
            out[j][q].re += zr * vc[q].re - zi * vc[q].im;
            out[j][q].im += zr * vc[q].im + zi * vc[q].re;
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < MAXOUT; ++j)
      if (j < nout) IO::st(vb + (size_t)j * V.stride, e, out[j]);
  }
}

// x (precision PX, site layout) += sum_i y[i] v_i  (basis precision PB).
// Element-wise: for P64 basis an element is one complex; for P32 two complex.
template <int PB, int PX>
__global__ void __launch_bounds__(kRedThreads) basis_accum_kernel(BasisArgs V, int nv,
                                                                  const double* y, int vh,
                                                                  Spinor x) {
  using IO = BasisIO<PB>;
  using T = typename IO::V;
  __shared__ double ys[2 * 128];
  for (int k = threadIdx.x; k < 2 * nv && k < 256; k += blockDim.x) ys[k] = y[k];
  __syncthreads();
  const T* vb = static_cast<const T*>(V.base);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < vh; s += gridDim.x * blockDim.x) {
    cplx<typename SpinorIO<PX>::R> xs[12];
    SpinorIO<PX>::load(x.data, x.norm, vh, s, xs);
    cplx<double> acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = {(double)xs[c].re, (double)xs[c].im};
    for (int i = 0; i < nv; ++i) {
      const double yr = ys[2 * i], yi = ys[2 * i + 1];
      const T* v = vb + (size_t)i * V.stride;
#pragma unroll
      for (int q = 0; q < 12 / IO::ncpx; ++q) {
        cplx<double> vc[2];
        IO::ld(v, (size_t)q * vh + s, vc);
#pragma unroll
        for (int t = 0; t < IO::ncpx; ++t) {
          const int c = IO::comp(q, t);
          acc[c].re += yr * vc[t].re - yi * vc[t].im;
          acc[c].im += yr * vc[t].im + yi * vc[t].re;
        }
      }
    }
    cplx<typename SpinorIO<PX>::R> o[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) o[c] = {(typename SpinorIO<PX>::R)acc[c].re, (typename SpinorIO<PX>::R)acc[c].im};
    SpinorIO<PX>::store(x.data, x.norm, vh, s, o);
  }
}

}  // namespace qq
