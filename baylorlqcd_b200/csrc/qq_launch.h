// Host-side launchers for the library's CUDA kernels (implemented in qq_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "qq_common.cuh"

namespace qq {

// Kernel-launch counter (every launcher below adds its launches): the process total,
// and the launches made by the calling host thread.
void count_launch(long long n = 1);
long long launch_count();
long long thread_launch_count();

struct HopArgs;
struct LinArgs;
struct BasisArgs;
struct Coef;

// Dirac hopping term.  sp: spinor precision (P64/P32/P16/PB16); recon: 18 or 12 (P64
// links) -- P32 and 16-bit spinors always use the FP32 recon-12 links; epi: Epilogue;
// tps: threads per site (direction groups: 1, 2 or 4).
cudaError_t launch_hop(const HopArgs& a, int sp, int recon, int epi, int tps, cudaStream_t st);

// out = a x + b y + c z (+ reductions into partial).  Precisions per operand.
cudaError_t launch_lincomb(const LinArgs& L, int px, int py, int pz, int po, cudaStream_t st);
cudaError_t launch_dot(int vh, Spinor x, Spinor y, double* partial, cudaStream_t st);
// out[v] = sum_b partial[b*nvstride + v] for v < nout (add: out += sum).
cudaError_t launch_finalize(const double* partial, int nblocks, int nvstride, int nout,
                            double* out, int add, cudaStream_t st);

// Krylov basis (pb = P64 or P32)
cudaError_t launch_multidot(int pb, const BasisArgs& V, int nv, const void* w, double* partial,
                            int* ngroups_out, cudaStream_t st);
cudaError_t launch_multiaxpy(int pb, const BasisArgs& V, int nv, const double* h, double hsign,
                             const void* w, void* wout, double* partial, cudaStream_t st);
cudaError_t launch_normalize(int pb, size_t nel, const void* in, void* out, const double* nrm2,
                             cudaStream_t st);
cudaError_t launch_rotate(int pb, const BasisArgs& V, int nin, int nout, const double* Z,
                          int ldz, cudaStream_t st);
cudaError_t launch_basis_accum(int pb, const BasisArgs& V, int nv, const double* y, int vh,
                               Spinor x, cudaStream_t st);
// H(j+1, j) = sqrt(nrm2[0]) and column add: H[:, j] += h2[0..nh)
cudaError_t launch_hcol_update(double* H, int ldh, int j, const double* h2, int nh,
                               const double* nrm2, cudaStream_t st);

// Layout conversion
struct RefDims;
cudaError_t launch_spinor_from_ref(const Geom& g, const RefDims& d, int p, const double* ref,
                                   Spinor out, cudaStream_t st);
cudaError_t launch_spinor_to_ref(const Geom& g, const RefDims& d, int p, Spinor in, double* ref,
                                 cudaStream_t st);
cudaError_t launch_ref_zero_halo(const RefDims& d, double* ref, cudaStream_t st);
cudaError_t launch_gauge_from_ref(const Geom& g, const RefDims& d, const double* ref, void* out,
                                  int prec, int recon, cudaStream_t st);
cudaError_t launch_su3_defect(const Geom& g, const RefDims& d, const double* ref,
                              double* partial, cudaStream_t st);

// Spin-diagonal site maps used by fermprop / twMshift / gamma5vector:
//   out = a x + ta J(x) + b y + tb J(y),  J: (s0,s1,s2,s3) -> (s2, s3, -s0, -s1)
// (J = i gamma5 in the reference basis, so 1 + t J = 1 + i t gamma5.)
cudaError_t launch_spinmix(int vh, Spinor x, Spinor y, Spinor out, double a, double ta,
                           double b, double tb, int prec, cudaStream_t st);

}  // namespace qq
