// Instantiations and launchers of the library's CUDA kernels (sm_100a).
#include <atomic>
#include <map>
#include <mutex>
#include <utility>

#include "qq_blas.cuh"
#include "qq_dslash.cuh"
#include "qq_dslash_f2.cuh"
#include "qq_launch.h"
#include "qq_layout.cuh"

namespace qq {

static std::atomic<long long> g_launches{0};
static thread_local long long t_launches = 0;
void count_launch(long long n) {
  g_launches += n;
  t_launches += n;
}
long long launch_count() { return g_launches.load(); }
long long thread_launch_count() { return t_launches; }

// The dynamic shared-memory limit of a kernel is a per-device attribute: set it once per
// (kernel, device) -- the current device -- and remember the result.  Host threads that
// launch side by side (one per context) serialise here only on the first launch.
static cudaError_t smem_attr_once(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, cudaError_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(kernel, dev);
  auto it = done.find(key);
  if (it != done.end()) return it->second;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  done[key] = e;
  return e;
}

// ---------------------------------------------------------------------------
// Dslash
// ---------------------------------------------------------------------------
// Launch-time copy of the arguments with the block split and float factors filled in.
static HopArgs hop_prepare(const HopArgs& a, int per_block, int threads_per_site) {
  HopArgs b = a;
  b.per_block = per_block;
  b.div_nrhs = FastDiv((unsigned)threads_per_site);
  b.af = (float)a.a;
  b.f1f = (float)a.f1;
  b.f2f = (float)a.f2;
  b.f3f = (float)a.f3;
  return b;
}

template <int SP, int LP, int RECON, int TPS>
static cudaError_t hop_epi(const HopArgs& a, int epi, cudaStream_t st) {
  dim3 blk, grd;
  hop_block_shape(TPS, a.nrhs, a.g.vh, &blk, &grd);
  const HopArgs b = hop_prepare(a, hop_sites_per_block(TPS, a.nrhs), a.nrhs);
  switch (epi) {
    case EPI_STORE: hop_kernel<SP, LP, RECON, TPS, EPI_STORE><<<grd, blk, 0, st>>>(b); break;
    case EPI_TWIST: hop_kernel<SP, LP, RECON, TPS, EPI_TWIST><<<grd, blk, 0, st>>>(b); break;
    case EPI_DBLE: hop_kernel<SP, LP, RECON, TPS, EPI_DBLE><<<grd, blk, 0, st>>>(b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int SP, int LP, int RECON, int EPI>
static cudaError_t hop_staged_launch(const HopArgs& a, int T, cudaStream_t st) {
  const size_t smem = staged_smem_bytes<SP, LP, RECON>(T);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  const cudaError_t attr = smem_attr_once((const void*)hop_staged_kernel<SP, LP, RECON, EPI>, 227 * 1024);
  if (attr != cudaSuccess) return attr;
  const HopArgs b = hop_prepare(a, T / a.nrhs, a.nrhs);
  dim3 grd((a.g.vh + b.per_block - 1) / b.per_block);
  hop_staged_kernel<SP, LP, RECON, EPI><<<grd, T, smem, st>>>(b);
  return cudaGetLastError();
}

template <int SP, int LP, int RECON>
static cudaError_t hop_tps(const HopArgs& a, int epi, int tps, cudaStream_t st) {
  switch (tps) {
    case 1: return hop_epi<SP, LP, RECON, 1>(a, epi, st);
    case 2: return hop_epi<SP, LP, RECON, 2>(a, epi, st);
    case 4: return hop_epi<SP, LP, RECON, 4>(a, epi, st);
    case 32:
    case 64:
    case 96:
    case 128:
      switch (epi) {
        case EPI_STORE: return hop_staged_launch<SP, LP, RECON, EPI_STORE>(a, tps, st);
        case EPI_TWIST: return hop_staged_launch<SP, LP, RECON, EPI_TWIST>(a, tps, st);
        case EPI_DBLE: return hop_staged_launch<SP, LP, RECON, EPI_DBLE>(a, tps, st);
        default: return cudaErrorInvalidValue;
      }
    default: return cudaErrorInvalidValue;
  }
}

// Block fields, RPT right-hand sides per thread.
template <int SP, int LP, int RECON, int RPT>
static cudaError_t hop_mrhs_rpt(const HopArgs& a, int epi, cudaStream_t st) {
  const int G = a.nrhs / RPT;  // threads per site
  const int per_block = hop_sites_per_block(1, G);
  const HopArgs b = hop_prepare(a, per_block, G);
  const dim3 blk(per_block * G), grd((a.g.vh + per_block - 1) / per_block);
  switch (epi) {
    case EPI_STORE: hop_mrhs_kernel<SP, LP, RECON, RPT, EPI_STORE><<<grd, blk, 0, st>>>(b); break;
    case EPI_TWIST: hop_mrhs_kernel<SP, LP, RECON, RPT, EPI_TWIST><<<grd, blk, 0, st>>>(b); break;
    case EPI_DBLE: hop_mrhs_kernel<SP, LP, RECON, RPT, EPI_DBLE><<<grd, blk, 0, st>>>(b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int SP, int LP, int RECON>
static cudaError_t hop_mrhs(const HopArgs& a, int epi, int rpt, cudaStream_t st) {
  switch (rpt) {
    case 2: return hop_mrhs_rpt<SP, LP, RECON, 2>(a, epi, st);
    case 3: return hop_mrhs_rpt<SP, LP, RECON, 3>(a, epi, st);
    case 4: return hop_mrhs_rpt<SP, LP, RECON, 4>(a, epi, st);
    default: return cudaErrorInvalidValue;
  }
}

// FP32 spinors, packed FP32x2 arithmetic, RPT right-hand sides per thread.
template <int RPT>
static cudaError_t hop_f2_rpt(const HopArgs& a, int epi, cudaStream_t st) {
  const int G = a.nrhs / RPT;  // threads per site
  const int per_block = hop_sites_per_block(1, G);
  const HopArgs b = hop_prepare(a, per_block, G);
  const dim3 blk(per_block * G), grd((a.g.vh + per_block - 1) / per_block);
  switch (epi) {
    case EPI_STORE: hop_f2_kernel<RPT, EPI_STORE><<<grd, blk, 0, st>>>(b); break;
    case EPI_TWIST: hop_f2_kernel<RPT, EPI_TWIST><<<grd, blk, 0, st>>>(b); break;
    case EPI_DBLE: hop_f2_kernel<RPT, EPI_DBLE><<<grd, blk, 0, st>>>(b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

static cudaError_t hop_f2p(const HopArgs& a, int epi, cudaStream_t st) {
  const int per_block = hop_sites_per_block(1, a.nrhs);
  const HopArgs b = hop_prepare(a, per_block, a.nrhs);
  const dim3 blk(per_block * a.nrhs), grd((a.g.vh + per_block - 1) / per_block);
  switch (epi) {
    case EPI_STORE: hop_f2p_kernel<EPI_STORE><<<grd, blk, 0, st>>>(b); break;
    case EPI_TWIST: hop_f2p_kernel<EPI_TWIST><<<grd, blk, 0, st>>>(b); break;
    case EPI_DBLE: hop_f2p_kernel<EPI_DBLE><<<grd, blk, 0, st>>>(b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

static cudaError_t hop_f2s(const HopArgs& a, int epi, cudaStream_t st) {
  const int per_block = hop_sites_per_block(1, a.nrhs);
  if (per_block > kLinkStageSites) return cudaErrorInvalidValue;  // nrhs >= 8 only
  const HopArgs b = hop_prepare(a, per_block, a.nrhs);
  const dim3 blk(per_block * a.nrhs), grd((a.g.vh + per_block - 1) / per_block);
  switch (epi) {
    case EPI_STORE: hop_f2s_kernel<EPI_STORE><<<grd, blk, 0, st>>>(b); break;
    case EPI_TWIST: hop_f2s_kernel<EPI_TWIST><<<grd, blk, 0, st>>>(b); break;
    case EPI_DBLE: hop_f2s_kernel<EPI_DBLE><<<grd, blk, 0, st>>>(b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Copy-ring kernel: D stages in flight per thread, RPT right-hand sides per thread,
// registers capped for MINB resident blocks.
template <int EPI, int D, int RPT, int MINB, int MB>
static cudaError_t hop_f2a_epi(const HopArgs& b, size_t smem, cudaStream_t st) {
  // The limit is 227 KiB less the kernel's static shared memory (the same on every
  // device; a function-local static is initialised once even under concurrent launches).
  struct Attr {
    cudaError_t err;
    size_t max_dyn;
  };
  static const Attr attr = [] {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, hop_f2a_kernel<EPI, D, RPT, MINB, MB>);
    if (e != cudaSuccess) return Attr{e, 0};
    return Attr{cudaSuccess, (size_t)227 * 1024 - fa.sharedSizeBytes};
  }();
  if (attr.err != cudaSuccess) return attr.err;
  if (smem > attr.max_dyn) return cudaErrorInvalidValue;
  const cudaError_t e = smem_attr_once((const void*)hop_f2a_kernel<EPI, D, RPT, MINB, MB>, (int)attr.max_dyn);
  if (e != cudaSuccess) return e;
  const int G = b.nrhs / RPT;
  const dim3 blk(b.per_block * G), grd((b.g.vh + b.per_block - 1) / b.per_block);
  hop_f2a_kernel<EPI, D, RPT, MINB, MB><<<grd, blk, smem, st>>>(b);
  return cudaGetLastError();
}

template <int D, int RPT, int MINB = 4, int MB = 0>
static cudaError_t hop_f2a(const HopArgs& a, int epi, cudaStream_t st) {
  if (a.nrhs % RPT != 0 || (RPT > 1 && !a.blk)) return cudaErrorInvalidValue;
  const int G = a.nrhs / RPT;  // threads per site
  int per_block = hop_sites_per_block(1, G);
  // Pre-broadcast hop matrices (MB) take 1.2 KB of shared memory per site: with one
  // thread per site, fewer sites per block (whole warps kept).
  while (MB && f2a_smem_bytes(per_block, per_block * G, D, RPT, MB) > 200 * 1024 && per_block % 2 == 0 &&
         (per_block / 2 * G) % 32 == 0)
    per_block /= 2;
  const HopArgs b = hop_prepare(a, per_block, G);
  const size_t smem = f2a_smem_bytes(per_block, per_block * G, D, RPT, MB);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  switch (epi) {
    case EPI_STORE: return hop_f2a_epi<EPI_STORE, D, RPT, MINB, MB>(b, smem, st);
    case EPI_TWIST: return hop_f2a_epi<EPI_TWIST, D, RPT, MINB, MB>(b, smem, st);
    case EPI_DBLE: return hop_f2a_epi<EPI_DBLE, D, RPT, MINB, MB>(b, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

// tps: 1, 2, 4 = register kernel with that many direction groups per site;
// 32, 64, 96, 128 = staged kernel with that many threads per block;
// kShapeMrhs + RPT (RPT = 2, 3, 4) = block fields with RPT right-hand sides per thread
// (FP32 / FP16 spinors, nrhs divisible by RPT);
// kShapeF2 + RPT (RPT = 1, 2, 3) = FP32 spinors with packed FP32x2 arithmetic (RPT > 1
// on block fields only); kShapeF2 + 4 = the same, loads a hop ahead; + 5 = links staged
// in shared memory (block fields); + 6, 7, 8 = copy ring with 2, 3, 4 stages in flight;
// + 9, 10 = copy ring with 2 stages, registers capped for 5 / 6 resident blocks;
// + 11 = copy ring with 3 stages and pre-broadcast hop matrices read row by row.
cudaError_t launch_hop(const HopArgs& a, int sp, int recon, int epi, int tps, cudaStream_t st) {
  count_launch();
  const int maxr = a.blk ? kMaxBatch : kMaxRhs;
  if (a.nrhs < 1 || a.nrhs > maxr) return cudaErrorInvalidValue;
  if (tps > kShapeF2) {
    const int rpt = tps - kShapeF2;
    if (sp != P32 || ((rpt == 2 || rpt == 3) && (a.nrhs % rpt != 0 || !a.blk)))
      return cudaErrorInvalidValue;
    switch (rpt) {
      case 1: return hop_f2_rpt<1>(a, epi, st);
      case 2: return hop_f2_rpt<2>(a, epi, st);
      case 3: return hop_f2_rpt<3>(a, epi, st);
      case 4: return hop_f2p(a, epi, st);  // pipelined, one RHS per thread
      case 5: return a.blk ? hop_f2s(a, epi, st) : cudaErrorInvalidValue;  // + staged links
      case 6: return hop_f2a<2, 1>(a, epi, st);  // copy ring, 2 / 3 / 4 stages in flight
      case 7: return hop_f2a<3, 1>(a, epi, st);
      case 8: return hop_f2a<4, 1>(a, epi, st);
      case 9: return hop_f2a<2, 1, 5>(a, epi, st);
      case 10: return hop_f2a<2, 1, 6>(a, epi, st);
      case 11: return hop_f2a<3, 1, 4, 1>(a, epi, st);

      default: return cudaErrorInvalidValue;
    }
  }
  if (tps > kShapeMrhs) {
    const int rpt = tps - kShapeMrhs;
    if (!a.blk || rpt < 2 || a.nrhs % rpt != 0) return cudaErrorInvalidValue;
    if (sp == P32) return hop_mrhs<P32, P32, 12>(a, epi, rpt, st);
    if (sp == P16) return hop_mrhs<P16, P32, 12>(a, epi, rpt, st);
    if (sp == PB16) return hop_mrhs<PB16, P32, 12>(a, epi, rpt, st);
    return cudaErrorInvalidValue;
  }
  const int per = tps <= 4 ? 128 / tps : tps;
  if (a.nrhs > per) return cudaErrorInvalidValue;
  if (sp == P64) {
    if (recon == 18) return hop_tps<P64, P64, 18>(a, epi, tps, st);
    if (recon == 12) return hop_tps<P64, P64, 12>(a, epi, tps, st);
    return cudaErrorInvalidValue;
  }
  if (sp == P32) return hop_tps<P32, P32, 12>(a, epi, tps, st);
  if (sp == P16) return hop_tps<P16, P32, 12>(a, epi, tps, st);
  if (sp == PB16) return hop_tps<PB16, P32, 12>(a, epi, tps, st);
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Level 1
// ---------------------------------------------------------------------------
template <int PX, int PY, int PZ, int PO>
static cudaError_t lin4(const LinArgs& L, cudaStream_t st) {
  lincomb_kernel<PX, PY, PZ, PO><<<kRedBlocks, kRedThreads, 0, st>>>(L);
  return cudaGetLastError();
}

// Supported combinations: all operands of one precision, or FP64 output with any
// single lower-precision operand in x (promotion), or lower output from FP64 x
// (demotion).
cudaError_t launch_lincomb(const LinArgs& L, int px, int py, int pz, int po, cudaStream_t st) {
  count_launch();
  if (!L.y.data) py = po;
  if (!L.z.data) pz = po;
  if (!L.x.data) px = po;
  if (px == po && py == po && pz == po) {
    if (po == P64) return lin4<P64, P64, P64, P64>(L, st);
    if (po == P32) return lin4<P32, P32, P32, P32>(L, st);
    if (po == P16) return lin4<P16, P16, P16, P16>(L, st);
    if (po == PB16) return lin4<PB16, PB16, PB16, PB16>(L, st);
  }
  if (po == P64 && py == P64 && pz == P64) {
    if (px == P32) return lin4<P32, P64, P64, P64>(L, st);
    if (px == P16) return lin4<P16, P64, P64, P64>(L, st);
    if (px == PB16) return lin4<PB16, P64, P64, P64>(L, st);
  }
  if (px == P64 && py == po && pz == po) {
    if (po == P32) return lin4<P64, P32, P32, P32>(L, st);
    if (po == P16) return lin4<P64, P16, P16, P16>(L, st);
    if (po == PB16) return lin4<P64, PB16, PB16, PB16>(L, st);
  }
  if (po == P16 && px == P32 && py == P16 && pz == P16) return lin4<P32, P16, P16, P16>(L, st);
  if (po == P32 && px == P16 && py == P32 && pz == P32) return lin4<P16, P32, P32, P32>(L, st);
  if (po == PB16 && px == P32 && py == PB16 && pz == PB16) return lin4<P32, PB16, PB16, PB16>(L, st);
  if (po == P32 && px == PB16 && py == P32 && pz == P32) return lin4<PB16, P32, P32, P32>(L, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_dot(int vh, Spinor x, Spinor y, double* partial, cudaStream_t st) {
  count_launch();
  if (x.prec == P64 && y.prec == P64)
    dot_kernel<P64, P64><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, partial);
  else if (x.prec == P32 && y.prec == P32)
    dot_kernel<P32, P32><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, partial);
  else if (x.prec == P16 && y.prec == P16)
    dot_kernel<P16, P16><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, partial);
  else if (x.prec == PB16 && y.prec == PB16)
    dot_kernel<PB16, PB16><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, partial);
  else if (x.prec == P64 && y.prec == P32)
    dot_kernel<P64, P32><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, partial);
  else if (x.prec == P32 && y.prec == P64)
    dot_kernel<P32, P64><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, partial);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

__global__ void finalize_sum_kernel(const double* partial, int nblocks, int nvstride, int nout,
                                    double* out, int add) {
  const int v = blockIdx.x;
  if (v >= nout) return;
  __shared__ double red[256];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partial[(size_t)b * nvstride + v];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[v] = add ? out[v] + red[0] : red[0];
}

cudaError_t launch_finalize(const double* partial, int nblocks, int nvstride, int nout,
                            double* out, int add, cudaStream_t st) {
  count_launch();
  finalize_sum_kernel<<<nout, 256, 0, st>>>(partial, nblocks, nvstride, nout, out, add);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Krylov basis
// ---------------------------------------------------------------------------
cudaError_t launch_multidot(int pb, const BasisArgs& V, int nv, const void* w, double* partial,
                            int* ngroups_out, cudaStream_t st) {
  count_launch();
  const int ng = (nv + 7) / 8;
  *ngroups_out = ng;
  dim3 grd(kRedBlocks, ng);
  if (pb == P64)
    multidot_kernel<P64><<<grd, kRedThreads, 0, st>>>(V, nv, w, partial);
  else if (pb == P32)
    multidot_kernel<P32><<<grd, kRedThreads, 0, st>>>(V, nv, w, partial);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_multiaxpy(int pb, const BasisArgs& V, int nv, const double* h, double hsign,
                             const void* w, void* wout, double* partial, cudaStream_t st) {
  count_launch();
  if (nv > 128) return cudaErrorInvalidValue;
  if (pb == P64)
    multiaxpy_kernel<P64><<<kRedBlocks, kRedThreads, 0, st>>>(V, nv, h, hsign, w, wout, partial);
  else if (pb == P32)
    multiaxpy_kernel<P32><<<kRedBlocks, kRedThreads, 0, st>>>(V, nv, h, hsign, w, wout, partial);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_normalize(int pb, size_t nel, const void* in, void* out, const double* nrm2,
                             cudaStream_t st) {
  count_launch();
  if (pb == P64)
    normalize_kernel<P64><<<kRedBlocks, kRedThreads, 0, st>>>(nel, in, out, nrm2);
  else if (pb == P32)
    normalize_kernel<P32><<<kRedBlocks, kRedThreads, 0, st>>>(nel, in, out, nrm2);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_rotate(int pb, const BasisArgs& V, int nin, int nout, const double* Z, int ldz,
                          cudaStream_t st) {
  count_launch();
  const size_t smem = sizeof(double) * 2 * (size_t)nin * nout;
  if (smem > 200 * 1024 || nout > 64) return cudaErrorInvalidValue;
  const int grid = 148 * 4;
  // The attribute is the bound checked above, the same for every call, so host threads
  // that launch side by side (one per context) never lower it under another's launch.
#define QQ_ROT(PB, MO)                                                                       \
  do {                                                                                       \
    auto k = rotate_kernel<PB, MO>;                                                          \
    const cudaError_t ea = smem_attr_once((const void*)k, 200 * 1024);                       \
    if (ea != cudaSuccess) return ea;                                                        \
    k<<<grid, 128, smem, st>>>(V, nin, nout, Z, ldz);                                        \
  } while (0)
  if (pb == P64) {
    if (nout <= 16) QQ_ROT(P64, 16);
    else if (nout <= 32) QQ_ROT(P64, 32);
    else QQ_ROT(P64, 64);
  } else if (pb == P32) {
    if (nout <= 16) QQ_ROT(P32, 16);
    else if (nout <= 32) QQ_ROT(P32, 32);
    else QQ_ROT(P32, 64);
  } else {
    return cudaErrorInvalidValue;
  }
#undef QQ_ROT
  return cudaGetLastError();
}

cudaError_t launch_basis_accum(int pb, const BasisArgs& V, int nv, const double* y, int vh,
                               Spinor x, cudaStream_t st) {
  count_launch();
  if (nv > 128) return cudaErrorInvalidValue;
  if (pb == P64 && x.prec == P64)
    basis_accum_kernel<P64, P64><<<kRedBlocks, kRedThreads, 0, st>>>(V, nv, y, vh, x);
  else if (pb == P32 && x.prec == P64)
    basis_accum_kernel<P32, P64><<<kRedBlocks, kRedThreads, 0, st>>>(V, nv, y, vh, x);
  else if (pb == P32 && x.prec == P32)
    basis_accum_kernel<P32, P32><<<kRedBlocks, kRedThreads, 0, st>>>(V, nv, y, vh, x);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

__global__ void hcol_update_kernel(double* H, int ldh, int j, const double* h2, int nh,
                                   const double* nrm2) {
  const int t = threadIdx.x;
  double* col = H + 2 * (size_t)ldh * j;
  for (int i = t; i < nh; i += blockDim.x) {
    col[2 * i] += h2[2 * i];
    col[2 * i + 1] += h2[2 * i + 1];
  }
  if (t == 0) {
    col[2 * (j + 1)] = sqrt(nrm2[0]);
    col[2 * (j + 1) + 1] = 0.0;
  }
}

cudaError_t launch_hcol_update(double* H, int ldh, int j, const double* h2, int nh,
                               const double* nrm2, cudaStream_t st) {
  count_launch();
  hcol_update_kernel<<<1, 128, 0, st>>>(H, ldh, j, h2, nh, nrm2);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Layout
// ---------------------------------------------------------------------------
cudaError_t launch_spinor_from_ref(const Geom& g, const RefDims& d, int p, const double* ref,
                                   Spinor out, cudaStream_t st) {
  count_launch();
  dim3 blk(128), grd((g.vh + 127) / 128);
  if (out.prec == P64)
    spinor_from_ref_kernel<P64><<<grd, blk, 0, st>>>(g, d, p, ref, out);
  else if (out.prec == P32)
    spinor_from_ref_kernel<P32><<<grd, blk, 0, st>>>(g, d, p, ref, out);
  else if (out.prec == P16)
    spinor_from_ref_kernel<P16><<<grd, blk, 0, st>>>(g, d, p, ref, out);
  else
    spinor_from_ref_kernel<PB16><<<grd, blk, 0, st>>>(g, d, p, ref, out);
  return cudaGetLastError();
}

cudaError_t launch_spinor_to_ref(const Geom& g, const RefDims& d, int p, Spinor in, double* ref,
                                 cudaStream_t st) {
  count_launch();
  dim3 blk(128), grd((g.vh + 127) / 128);
  if (in.prec == P64)
    spinor_to_ref_kernel<P64><<<grd, blk, 0, st>>>(g, d, p, in, ref);
  else if (in.prec == P32)
    spinor_to_ref_kernel<P32><<<grd, blk, 0, st>>>(g, d, p, in, ref);
  else if (in.prec == P16)
    spinor_to_ref_kernel<P16><<<grd, blk, 0, st>>>(g, d, p, in, ref);
  else
    spinor_to_ref_kernel<PB16><<<grd, blk, 0, st>>>(g, d, p, in, ref);
  return cudaGetLastError();
}

cudaError_t launch_ref_zero_halo(const RefDims& d, double* ref, cudaStream_t st) {
  count_launch();
  if (d.ntotal == d.nvhalf) return cudaSuccess;
  ref_zero_halo_kernel<<<148, 256, 0, st>>>(d, ref);
  return cudaGetLastError();
}

cudaError_t launch_gauge_from_ref(const Geom& g, const RefDims& d, const double* ref, void* out,
                                  int prec, int recon, cudaStream_t st) {
  count_launch();
  dim3 blk(128), grd((2 * g.vh + 127) / 128);
  if (prec == P64 && recon == 18)
    gauge_from_ref_kernel<P64, 18><<<grd, blk, 0, st>>>(g, d, ref, out);
  else if (prec == P64 && recon == 12)
    gauge_from_ref_kernel<P64, 12><<<grd, blk, 0, st>>>(g, d, ref, out);
  else if (prec == P32 && recon == 12)
    gauge_from_ref_kernel<P32, 12><<<grd, blk, 0, st>>>(g, d, ref, out);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

cudaError_t launch_su3_defect(const Geom& g, const RefDims& d, const double* ref, double* partial,
                              cudaStream_t st) {
  count_launch();
  su3_defect_kernel<<<kRedBlocks, 256, 0, st>>>(g, d, ref, partial);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Spin mixing: out = a x + ta J(x) + b y + tb J(y)
// ---------------------------------------------------------------------------
template <int P>
__global__ void spinmix_kernel(int vh, Spinor x, Spinor y, Spinor out, double a, double ta,
                               double b, double tb) {
  using R = typename SpinorIO<P>::R;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < vh; s += gridDim.x * blockDim.x) {
    cplx<R> xv[12], yv[12], o[12];
    SpinorIO<P>::load(x.data, x.norm, vh, s, xv);
    if (y.data)
      SpinorIO<P>::load(y.data, y.norm, vh, s, yv);
    else
      for (int c = 0; c < 12; ++c) yv[c] = {(R)0, (R)0};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      // J(v) = (v2, v3, -v0, -v1)
      o[0 + c] = cadd(cadd(cscale((R)a, xv[0 + c]), cscale((R)ta, xv[6 + c])),
                      cadd(cscale((R)b, yv[0 + c]), cscale((R)tb, yv[6 + c])));
      o[3 + c] = cadd(cadd(cscale((R)a, xv[3 + c]), cscale((R)ta, xv[9 + c])),
                      cadd(cscale((R)b, yv[3 + c]), cscale((R)tb, yv[9 + c])));
      o[6 + c] = cadd(csub(cscale((R)a, xv[6 + c]), cscale((R)ta, xv[0 + c])),
                      csub(cscale((R)b, yv[6 + c]), cscale((R)tb, yv[0 + c])));
      o[9 + c] = cadd(csub(cscale((R)a, xv[9 + c]), cscale((R)ta, xv[3 + c])),
                      csub(cscale((R)b, yv[9 + c]), cscale((R)tb, yv[3 + c])));
    }
    SpinorIO<P>::store(out.data, out.norm, vh, s, o);
  }
}

cudaError_t launch_spinmix(int vh, Spinor x, Spinor y, Spinor out, double a, double ta, double b,
                           double tb, int prec, cudaStream_t st) {
  count_launch();
  if (prec == P64)
    spinmix_kernel<P64><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, out, a, ta, b, tb);
  else if (prec == P32)
    spinmix_kernel<P32><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, out, a, ta, b, tb);
  else if (prec == P16)
    spinmix_kernel<P16><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, out, a, ta, b, tb);
  else
    spinmix_kernel<PB16><<<kRedBlocks, kRedThreads, 0, st>>>(vh, x, y, out, a, ta, b, tb);
  return cudaGetLastError();
}

}  // namespace qq
