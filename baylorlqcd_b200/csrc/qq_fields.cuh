// Load / store of Dirac half-vectors and SU(3) links in the GPU layout described in
// qq_common.cuh.  Every access is a 16-byte vector load/store along a plane.
#pragma once
#include "qq_common.cuh"

namespace qq {

// ---------------------------------------------------------------------------
// Spinors: 12 complex components c = 3*spin + colour.
// ---------------------------------------------------------------------------
template <int P>
struct SpinorIO;

template <>
struct SpinorIO<P64> {
  using R = double;
  static constexpr int planes = 12;
  static constexpr size_t bytes_per_site = 192;
  __device__ static inline void load(const void* base, const float*, int vh, int s,
                                     cplx<R>* v) {
    const double2* f = static_cast<const double2*>(base);
#pragma unroll
    for (int c = 0; c < 12; ++c) {
      double2 t = __ldg(f + (size_t)c * vh + s);
      v[c] = {t.x, t.y};
    }
  }
  __device__ static inline void store(void* base, float*, int vh, int s, const cplx<R>* v) {
    double2* f = static_cast<double2*>(base);
#pragma unroll
    for (int c = 0; c < 12; ++c) f[(size_t)c * vh + s] = make_double2(v[c].re, v[c].im);
  }
};

// FP32 planes hold spin pairs: plane q < 3 is colour q of spins (0, 1), plane q >= 3
// colour q - 3 of spins (2, 3), each float4 = (a.re, b.re, a.im, b.im) for the pair
// (a, b = a + 3) of component indices (spin * 3 + colour).  The real parts and the
// imaginary parts of a spin pair are then adjacent registers, so the Dirac operator
// applies the projections and SU(3) products to both halves of a half spinor with
// packed FP32x2 instructions.
__host__ __device__ constexpr int p32_first(int q) { return q < 3 ? q : q + 3; }

template <>
struct SpinorIO<P32> {
  using R = float;
  static constexpr int planes = 6;
  static constexpr size_t bytes_per_site = 96;
  __device__ static inline void load(const void* base, const float*, int vh, int s,
                                     cplx<R>* v) {
    const float4* f = static_cast<const float4*>(base);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      float4 t = __ldg(f + (size_t)q * vh + s);
      const int a = p32_first(q);
      v[a] = {t.x, t.z};
      v[a + 3] = {t.y, t.w};
    }
  }
  __device__ static inline void store(void* base, float*, int vh, int s, const cplx<R>* v) {
    float4* f = static_cast<float4*>(base);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const int a = p32_first(q);
      f[(size_t)q * vh + s] = make_float4(v[a].re, v[a + 3].re, v[a].im, v[a + 3].im);
    }
  }
};

// FP16 storage with one FP32 scale per site (max |component|), FP32 arithmetic.
template <>
struct SpinorIO<P16> {
  using R = float;
  static constexpr int planes = 3;
  static constexpr size_t bytes_per_site = 52;
  __device__ static inline void load(const void* base, const float* norm, int vh, int s,
                                     cplx<R>* v) {
    const int4* f = static_cast<const int4*>(base);
    const float nrm = __ldg(norm + s);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      int4 t = __ldg(f + (size_t)q * vh + s);
      const __half2* h = reinterpret_cast<const __half2*>(&t);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float2 ff = __half22float2(h[k]);
        v[4 * q + k] = {ff.x * nrm, ff.y * nrm};
      }
    }
  }
  __device__ static inline void store(void* base, float* norm, int vh, int s,
                                      const cplx<R>* v) {
    float m = 0.f;
#pragma unroll
    for (int c = 0; c < 12; ++c) m = fmaxf(m, fmaxf(fabsf(v[c].re), fabsf(v[c].im)));
    const float inv = m > 0.f ? 1.f / m : 0.f;
    int4* f = static_cast<int4*>(base);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      int4 t;
      __half2* h = reinterpret_cast<__half2*>(&t);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        h[k] = __floats2half2_rn(v[4 * q + k].re * inv, v[4 * q + k].im * inv);
      f[(size_t)q * vh + s] = t;
    }
    norm[s] = m;
  }
};

// BF16 storage with one FP32 scale per site, FP32 arithmetic: the layout of SpinorIO<P16>
// with bfloat16 values (8 exponent bits, 8 significant bits).
template <>
struct SpinorIO<PB16> {
  using R = float;
  static constexpr int planes = 3;
  static constexpr size_t bytes_per_site = 52;
  __device__ static inline void load(const void* base, const float* norm, int vh, int s,
                                     cplx<R>* v) {
    const int4* f = static_cast<const int4*>(base);
    const float nrm = __ldg(norm + s);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      int4 t = __ldg(f + (size_t)q * vh + s);
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&t);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        float2 ff = __bfloat1622float2(h[k]);
        v[4 * q + k] = {ff.x * nrm, ff.y * nrm};
      }
    }
  }
  __device__ static inline void store(void* base, float* norm, int vh, int s,
                                      const cplx<R>* v) {
    float m = 0.f;
#pragma unroll
    for (int c = 0; c < 12; ++c) m = fmaxf(m, fmaxf(fabsf(v[c].re), fabsf(v[c].im)));
    const float inv = m > 0.f ? 1.f / m : 0.f;
    int4* f = static_cast<int4*>(base);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      int4 t;
      __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&t);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        h[k] = __floats2bfloat162_rn(v[4 * q + k].re * inv, v[4 * q + k].im * inv);
      f[(size_t)q * vh + s] = t;
    }
    norm[s] = m;
  }
};

// ---------------------------------------------------------------------------
// Links.  Storage: per parity p and direction mu, `planes` 16-byte vectors per site,
// indexed [((p*4 + mu)*planes + q)*vh + s].
// ---------------------------------------------------------------------------
template <class R>
struct Su3 {
  cplx<R> e[3][3];
};

template <class R>
__device__ inline void reconstruct_row3(Su3<R>& u) {
  // row3 = conj(row1 x row2) for a special unitary matrix
  u.e[2][0] = cconj(csub(cmul(u.e[0][1], u.e[1][2]), cmul(u.e[0][2], u.e[1][1])));
  u.e[2][1] = cconj(csub(cmul(u.e[0][2], u.e[1][0]), cmul(u.e[0][0], u.e[1][2])));
  u.e[2][2] = cconj(csub(cmul(u.e[0][0], u.e[1][1]), cmul(u.e[0][1], u.e[1][0])));
}

template <int P, int RECON>
struct LinkIO;

template <>
struct LinkIO<P64, 18> {
  using R = double;
  static constexpr int planes = 9;
  static constexpr size_t bytes_per_link = 144;
  __device__ static inline void load(const void* base, int vh, int p, int mu, int s, Su3<R>& u) {
    const double2* f = static_cast<const double2*>(base) + (size_t)(p * 4 + mu) * planes * vh;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      double2 t = __ldg(f + (size_t)q * vh + s);
      u.e[q / 3][q % 3] = {t.x, t.y};
    }
  }
};

template <>
struct LinkIO<P64, 12> {
  using R = double;
  static constexpr int planes = 6;
  static constexpr size_t bytes_per_link = 96;
  __device__ static inline void load(const void* base, int vh, int p, int mu, int s, Su3<R>& u) {
    const double2* f = static_cast<const double2*>(base) + (size_t)(p * 4 + mu) * planes * vh;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      double2 t = __ldg(f + (size_t)q * vh + s);
      u.e[q / 3][q % 3] = {t.x, t.y};
    }
    reconstruct_row3(u);
  }
};

template <>
struct LinkIO<P32, 12> {
  using R = float;
  static constexpr int planes = 3;
  static constexpr size_t bytes_per_link = 48;
  __device__ static inline void load(const void* base, int vh, int p, int mu, int s, Su3<R>& u) {
    const float4* f = static_cast<const float4*>(base) + (size_t)(p * 4 + mu) * planes * vh;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float4 t = __ldg(f + (size_t)q * vh + s);
      const int c0 = 2 * q, c1 = 2 * q + 1;
      u.e[c0 / 3][c0 % 3] = {t.x, t.y};
      u.e[c1 / 3][c1 % 3] = {t.z, t.w};
    }
    reconstruct_row3(u);
  }
};

}  // namespace qq
