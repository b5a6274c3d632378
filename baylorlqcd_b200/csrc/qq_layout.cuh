// Conversions between the reference's Fortran layouts and the GPU layout.
//   Dirac half-vector  g(6, ntotal, 4, 2, 8)   Q/diracops.f90:41-59
//   Gauge field        u(18, ntotal, 4, 2, 16) Q/diracops.f90:312-313 (3x3 row-major)
// The site map is G/lattice.f90 siteindex/setblk/gblchker (see ref_site()).
#pragma once
#include "qq_fields.cuh"

namespace qq {

struct RefDims {
  int nvhalf, ntotal;
};

__host__ __device__ inline size_t ref_gi(const RefDims& d, int a, int isite, int id, int ieo,
                                         int ibleo) {
  return (size_t)(a - 1) +
         6 * ((size_t)(isite - 1) +
              (size_t)d.ntotal * ((size_t)(id - 1) + 4 * ((size_t)(ieo - 1) + 2 * (size_t)(ibleo - 1))));
}
__host__ __device__ inline size_t ref_ui(const RefDims& d, int a, int isite, int mu, int ieo,
                                         int ibl) {
  return (size_t)(a - 1) +
         18 * ((size_t)(isite - 1) +
               (size_t)d.ntotal * ((size_t)(mu - 1) + 4 * ((size_t)(ieo - 1) + 2 * (size_t)(ibl - 1))));
}

// GPU spinor (parity p) <- reference half-vector.
template <int PO>
__global__ void spinor_from_ref_kernel(Geom g, RefDims d, int p, const double* ref, Spinor out) {
  using R = typename SpinorIO<PO>::R;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.vh) return;
  int x[4], isite, ieo, ibleo;
  site_coords(g, p, s, x);
  ref_site(g, x, &isite, &ieo, &ibleo);
  cplx<R> v[12];
#pragma unroll
  for (int id = 1; id <= 4; ++id)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t k = ref_gi(d, 2 * c + 1, isite, id, ieo, ibleo);
      v[3 * (id - 1) + c] = {(R)ref[k], (R)ref[k + 1]};
    }
  SpinorIO<PO>::store(out.data, out.norm, g.vh, s, v);
}

// reference half-vector <- GPU spinor (interior sites only).
template <int PI>
__global__ void spinor_to_ref_kernel(Geom g, RefDims d, int p, Spinor in, double* ref) {
  using R = typename SpinorIO<PI>::R;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.vh) return;
  int x[4], isite, ieo, ibleo;
  site_coords(g, p, s, x);
  ref_site(g, x, &isite, &ieo, &ibleo);
  cplx<R> v[12];
  SpinorIO<PI>::load(in.data, in.norm, g.vh, s, v);
#pragma unroll
  for (int id = 1; id <= 4; ++id)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t k = ref_gi(d, 2 * c + 1, isite, id, ieo, ibleo);
      ref[k] = (double)v[3 * (id - 1) + c].re;
      ref[k + 1] = (double)v[3 * (id - 1) + c].im;
    }
}

// Zero the halo slots (isite > nvhalf) of a reference half-vector, as Hsingle's
// `gout = 0.0_KR` leaves them (Q/diracops.f90:590).
static __global__ void ref_zero_halo_kernel(RefDims d, double* ref) {
  const int nb = d.ntotal - d.nvhalf;
  const int total = nb * 6 * 4 * 2 * 8;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int r = t;
    const int a = r % 6; r /= 6;
    const int ib = r % nb; r /= nb;
    const int id = r % 4; r /= 4;
    const int ieo = r % 2; r /= 2;
    const int ibleo = r;
    ref[ref_gi(d, a + 1, d.nvhalf + ib + 1, id + 1, ieo + 1, ibleo + 1)] = 0.0;
  }
}

// GPU gauge field <- reference u(18, ntotal, 4, 2, 16).
// recon 18: planes 0..8 = all 9 complex; recon 12: planes hold rows 1, 2.
template <int PL, int RECON>
__global__ void gauge_from_ref_kernel(Geom g, RefDims d, const double* ref, void* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * g.vh) return;
  const int p = t / g.vh, s = t % g.vh;
  int x[4], isite, ieo, ibleo;
  site_coords(g, p, s, x);
  ref_site(g, x, &isite, &ieo, &ibleo);
  const int ibl = 1 + (x[0] & 1) + 2 * (x[1] & 1) + 4 * (x[2] & 1) + 8 * (x[3] & 1);
  for (int mu = 0; mu < 4; ++mu) {
    const double* u = ref + ref_ui(d, 1, isite, mu + 1, ieo, ibl);
    if (PL == P64) {
      constexpr int planes = RECON == 18 ? 9 : 6;
      double2* o = static_cast<double2*>(out) + (size_t)(p * 4 + mu) * planes * g.vh;
      for (int q = 0; q < planes; ++q) o[(size_t)q * g.vh + s] = make_double2(u[2 * q], u[2 * q + 1]);
    } else {
      constexpr int planes = 3;  // recon 12 only
      float4* o = static_cast<float4*>(out) + (size_t)(p * 4 + mu) * planes * g.vh;
      for (int q = 0; q < planes; ++q)
        o[(size_t)q * g.vh + s] = make_float4((float)u[4 * q], (float)u[4 * q + 1],
                                              (float)u[4 * q + 2], (float)u[4 * q + 3]);
    }
  }
}

// Largest |row3 - conj(row1 x row2)| over all links: decides if recon-12 is exact.
static __global__ void su3_defect_kernel(Geom g, RefDims d, const double* ref, double* partial) {
  double m = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * g.vh; t += gridDim.x * blockDim.x) {
    const int p = t / g.vh, s = t % g.vh;
    int x[4], isite, ieo, ibleo;
    site_coords(g, p, s, x);
    ref_site(g, x, &isite, &ieo, &ibleo);
    const int ibl = 1 + (x[0] & 1) + 2 * (x[1] & 1) + 4 * (x[2] & 1) + 8 * (x[3] & 1);
    for (int mu = 0; mu < 4; ++mu) {
      const double* u = ref + ref_ui(d, 1, isite, mu + 1, ieo, ibl);
      Su3<double> w;
      for (int q = 0; q < 9; ++q) w.e[q / 3][q % 3] = {u[2 * q], u[2 * q + 1]};
      Su3<double> r = w;
      reconstruct_row3(r);
      for (int c = 0; c < 3; ++c) {
        m = fmax(m, fabs(r.e[2][c].re - w.e[2][c].re));
        m = fmax(m, fabs(r.e[2][c].im - w.e[2][c].im));
      }
    }
  }
  // block max
  __shared__ double red[256];
  red[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

}  // namespace qq
