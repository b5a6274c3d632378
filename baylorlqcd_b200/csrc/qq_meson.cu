// Local meson correlators of a propagator column (qq_pionrho): pionrho,
// Q/quark.f90:1033-1212.  For the solution (xe, xo) of one source spin idsrc, per time
// slice t and summed over the slice's sites, colours and the real and imaginary parts:
//   pion(t)  += sum |x|^2 over the four spins (the reference's gamma_5 rotation at two
//               time slices permutes spins with signs and leaves the sum unchanged)
//   rho(t)   += rsgn(idsrc) sum (|x_1|^2 - |x_2|^2 - |x_3|^2 + |x_4|^2),
//               rsgn = (1, -1, -1, 1)  (third component of the vector current)
//   decay(t) += sum (|x_1|^2 + |x_2|^2 - |x_3|^2 - |x_4|^2)  (fourth axial component)
// in FP64.  The sites of one time slice and parity are a contiguous range of the
// checkerboard index, so one thread block reduces each (slice, parity) in a fixed
// order and the host adds the two parities.
#include <cstring>
#include <vector>

#include "qq_ctx.h"

namespace qq {
namespace {

constexpr int kMesonThreads = 256;

__global__ void __launch_bounds__(kMesonThreads) pionrho_kernel(int vt, Spinor f, int vh, double* partial) {
  __shared__ double red[3][kMesonThreads];
  const int t = blockIdx.x;
  double a[3] = {0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < vt; i += blockDim.x) {
    const int s = t * vt + i;
    cplx<double> v[12];
    SpinorIO<P64>::load(f.data, f.norm, vh, s, v);
    double sp[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      sp[d] = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) sp[d] += v[3 * d + c].re * v[3 * d + c].re + v[3 * d + c].im * v[3 * d + c].im;
    }
    a[0] += sp[0] + sp[1] + sp[2] + sp[3];
    a[1] += sp[0] - sp[1] - sp[2] + sp[3];
    a[2] += sp[0] + sp[1] - sp[2] - sp[3];
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) red[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 3; ++q) partial[(size_t)t * 3 + q] = red[q][0];
}

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_pionrho(qq_ctx* c, const double* xe, const double* xo, int idsrc, double* pion, double* rho,
                          double* decay) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  if (!xe || !xo || !pion || !rho || !decay) return set_error(QQ_BAD_ARG, "null argument");
  if (idsrc < 1 || idsrc > 4) return set_error(QQ_BAD_ARG, "idsrc must be 1..4");
  QQ_CK(cudaSetDevice(c->device));
  const int nt = c->g.n[3];
  const int vt = c->g.vh / nt;  // sites of one parity on one time slice
  const size_t nv = c->ref_doubles();
  Tmp f(c, P64);
  DevBuf part;
  QQ_CK(part.alloc(sizeof(double) * 3 * nt * 2));
  for (int p = 0; p < 2; ++p) {
    const double* d = nullptr;
    QQ_TRY(stage_in(c, 1, p == 0 ? xe : xo, nv, &d));
    QQ_TRY(ref_to_field(c, d, p, f.sp()));
    count_launch();
    pionrho_kernel<<<nt, kMesonThreads, 0, c->st>>>(vt, f.sp(), c->g.vh, part.as<double>() + (size_t)p * 3 * nt);
    QQ_CK(cudaGetLastError());
  }
  std::vector<double> h(6 * (size_t)nt);
  QQ_CK(cudaMemcpyAsync(h.data(), part.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  const double rsgn[4] = {1.0, -1.0, -1.0, 1.0};
  std::vector<double> out(3 * (size_t)nt);
  double* dst[3] = {pion, rho, decay};
  for (int q = 0; q < 3; ++q) {
    QQ_CK(cudaMemcpy(out.data() + (size_t)q * nt, dst[q], sizeof(double) * nt, cudaMemcpyDefault));
    for (int t = 0; t < nt; ++t) {
      const double v = h[(size_t)t * 3 + q] + h[(size_t)(3 * nt) + (size_t)t * 3 + q];
      out[(size_t)q * nt + t] += q == 1 ? rsgn[idsrc - 1] * v : v;
    }
    QQ_CK(cudaMemcpy(dst[q], out.data() + (size_t)q * nt, sizeof(double) * nt, cudaMemcpyDefault));
  }
  return QQ_OK;
}
