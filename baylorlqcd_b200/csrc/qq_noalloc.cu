// qq_vecdot_noalloc: the inner product vecdot (Q/inverters.f90:13485-13530) computed
// straight from two reference-layout half-vectors already in device memory, with no
// device allocation of any kind.
//
// Who needs it: a host code that commits the device memory to its own field arrays at
// start-up (the reference sizes every array once from the lattice dimensions) cannot
// let a library grow staging buffers or temporaries behind its back, and a caller
// inside a tight solver loop cannot afford cudaMalloc/cudaFree, whose implicit device
// synchronisation would serialise its streams.  qq_vecdot stages its inputs into
// pooled GPU-layout fields (which allocate on first use); this variant reads the
// reference layout in place and keeps its reduction partials in the file-scope
// array below, so the call allocates nothing: no cudaMalloc, no cudaFree, no
// allocating library routine.
//
// Scratch: g_vecdot_scratch, kScratchPartials complex partials (one per block of
// kRowsPerBlock rows) plus the final complex result, 16 KiB + 16 B per 1024 partials.
// A row is one (isite, id, ieo, ibl) entry of the half-vector: 3 complex colour
// components, 6 contiguous doubles.  A lattice of V sites has 2V interior rows, so
// the scratch bounds V at kScratchPartials * kRowsPerBlock / 2 = 4,194,304 sites;
// larger lattices are rejected with QQ_BAD_ARG.  Nothing in the scratch has to start
// at zero: stage 1 overwrites every partial stage 2 reads, and stage 2 overwrites the
// result before it is copied out.
//
// Setup: the first call on a device looks the array's address up once with
// cudaGetSymbolAddress (that device current, return code checked) and caches it per
// device; that first call should therefore come before any stream capture.
//
// The scratch is one array per device shared by every context on it: calls that
// overlap on one device (other threads, other streams) race on it and must be
// serialised by the caller.
#include <cstdint>
#include <mutex>

#include "qq_ctx.h"

namespace qq {

constexpr int kRowsPerBlock = 1024;     // 256 threads x 4 rows
constexpr int kNaThreads = 256;
constexpr int kScratchPartials = 8192;  // => at most 8192 * 1024 / 2 lattice sites
constexpr int kMaxDevices = 64;

// 8192 complex partials + the complex result: 131,088 bytes per device.
static __device__ __align__(256) double g_vecdot_scratch[2 * kScratchPartials + 2];

namespace {

double* g_scratch_dev[kMaxDevices];  // address of g_vecdot_scratch per device
std::mutex g_scratch_mu;

// Warp then block sum of (re, im) in a fixed order; result valid in thread 0.
__device__ inline void block_sum2(double& re, double& im) {
  __shared__ double sre[kNaThreads / 32], sim[kNaThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sre[w] = re;
    sim[w] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    re = 0.0;
    im = 0.0;
    for (int j = 0; j < kNaThreads / 32; ++j) {
      re += sre[j];
      im += sim[j];
    }
  }
}

// Stage 1: block b sums conj(a) b over rows [b * kRowsPerBlock, (b + 1) * kRowsPerBlock).
// Row r = plane * nvhalf + isite, plane = (ibl * 2 + ieo) * 4 + id, starts at double
// (plane * ntotal + isite) * 6 of the (8, 2, 4, ntotal, 6) array.
__global__ void __launch_bounds__(kNaThreads)
    vecdot_rows_kernel(const double2* __restrict__ a, const double2* __restrict__ b, long long nrows,
                       int nvhalf, int ntotal, double2* __restrict__ partial) {
  double re = 0.0, im = 0.0;
  const long long r0 = (long long)blockIdx.x * kRowsPerBlock;
#pragma unroll
  for (int j = 0; j < kRowsPerBlock / kNaThreads; ++j) {
    const long long r = r0 + threadIdx.x + (long long)j * kNaThreads;
    if (r < nrows) {
      const long long plane = r / nvhalf, isite = r - plane * nvhalf;
      const long long off = (plane * ntotal + isite) * 3;  // in complex numbers
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double2 x = a[off + c], y = b[off + c];
        re += x.x * y.x + x.y * y.y;
        im += x.x * y.y - x.y * y.x;
      }
    }
  }
  block_sum2(re, im);
  if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(re, im);
}

// Stage 2: one block sums the nblocks partials in a fixed order into *out.
__global__ void __launch_bounds__(kNaThreads)
    vecdot_partials_kernel(const double2* __restrict__ partial, int nblocks, double2* __restrict__ out) {
  double re = 0.0, im = 0.0;
  for (int j = threadIdx.x; j < nblocks; j += kNaThreads) {
    re += partial[j].x;
    im += partial[j].y;
  }
  block_sum2(re, im);
  if (threadIdx.x == 0) *out = make_double2(re, im);
}

// Address of the scratch on `dev` (the current device); looked up once per device.
int scratch_on_device(int dev, double** p) {
  if (dev < 0 || dev >= kMaxDevices) return set_error(QQ_BAD_ARG, "qq_vecdot_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_dev[dev]) {
    void* q = nullptr;
    QQ_CK(cudaGetSymbolAddress(&q, g_vecdot_scratch));
    g_scratch_dev[dev] = static_cast<double*>(q);
  }
  *p = g_scratch_dev[dev];
  return QQ_OK;
}

int check_input(const qq_ctx* c, const double* p, const char* name) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return set_error(QQ_BAD_ARG, std::string("qq_vecdot_noalloc: ") + name + " is not device memory");
  }
  if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
    return set_error(QQ_BAD_ARG, std::string("qq_vecdot_noalloc: ") + name +
                                     " must be device memory (host arrays would need a staging buffer)");
  if (at.type == cudaMemoryTypeDevice && at.device != c->device)
    return set_error(QQ_BAD_ARG, std::string("qq_vecdot_noalloc: ") + name + " lives on another device");
  if (reinterpret_cast<std::uintptr_t>(p) % 16 != 0)
    return set_error(QQ_BAD_ARG, std::string("qq_vecdot_noalloc: ") + name + " is not 16-byte aligned");
  return QQ_OK;
}

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_vecdot_noalloc(qq_ctx* c, const double* a, const double* b, double adb[2]) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!a || !b || !adb) return set_error(QQ_BAD_ARG, "qq_vecdot_noalloc: null argument");
  QQ_CK(cudaSetDevice(c->device));
  const long long nrows = 64LL * c->rd.nvhalf;
  const long long nblocks = (nrows + kRowsPerBlock - 1) / kRowsPerBlock;
  if (nblocks > kScratchPartials)
    return set_error(QQ_BAD_ARG, "qq_vecdot_noalloc: lattice of " + std::to_string(32LL * c->rd.nvhalf) +
                                     " sites exceeds the 4194304-site limit of its static scratch");
  QQ_TRY(check_input(c, a, "a"));
  QQ_TRY(check_input(c, b, "b"));
  double* scratch = nullptr;
  QQ_TRY(scratch_on_device(c->device, &scratch));
  double2* partial = reinterpret_cast<double2*>(scratch);
  double2* result = partial + kScratchPartials;
  vecdot_rows_kernel<<<(unsigned)nblocks, kNaThreads, 0, c->st>>>(
      reinterpret_cast<const double2*>(a), reinterpret_cast<const double2*>(b), nrows, c->rd.nvhalf,
      c->rd.ntotal, partial);
  QQ_CK(cudaGetLastError());
  vecdot_partials_kernel<<<1, kNaThreads, 0, c->st>>>(partial, (int)nblocks, result);
  QQ_CK(cudaGetLastError());
  count_launch(2);
  QQ_CK(cudaMemcpyAsync(adb, result, 2 * sizeof(double), cudaMemcpyDefault, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}
