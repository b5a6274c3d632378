// Internal context of the B200 qqcd library (host side).
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/qqcd_gpu.h"
#include "qq_blas.cuh"
#include "qq_dense.h"
#include "qq_dslash.cuh"
#include "qq_launch.h"
#include "qq_layout.cuh"

namespace qq {

int set_error(int code, const std::string& msg);

#define QQ_CK(x)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (x);                                                           \
    if (e_ != cudaSuccess)                                                          \
      return ::qq::set_error(QQ_CUDA_ERR, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define QQ_TRY(x)             \
  do {                        \
    int s_ = (x);             \
    if (s_ != QQ_OK) return s_; \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// A Dirac half-vector in GPU layout.
struct Field {
  DevBuf data, norm;
  int prec = P64;
  Spinor sp() const { return Spinor{data.p, norm.as<float>(), prec}; }
};

inline size_t field_bytes(int prec, int vh) {
  return prec == P64 ? (size_t)192 * vh : prec == P32 ? (size_t)96 * vh : (size_t)48 * vh;
}

// Deflation space: k+1 basis vectors (GPU layout, precision pb) and the projected
// (k+1) x k matrix of A V_k = V_{k+1} Hk.
struct DeflSpace {
  int k = 0;
  int pb = P64;
  size_t nel = 0;
  DevBuf V;
  dense::Mat Hk;
};

}  // namespace qq

struct qq_defl {
  qq_ctx* ctx;
  int nmax, kmax;
  qq::DeflSpace space;
};

struct qq_ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  qq::Geom g{};
  qq::RefDims rd{};
  double c1[4], c2[4];
  qq::DevBuf gauge64, gauge32;
  int recon64 = 0;
  bool have_gauge = false;
  qq::DevBuf stage[4];      // reference-layout staging buffers
  qq::DevBuf partial;       // reduction partials
  qq::DevBuf scal;          // device scalar slots
  qq::DevBuf trace_buf;     // per-site loop-trace values and the time-slice sums
  double* hpin = nullptr;   // pinned host memory: [0, 1024) read_scalars staging,
                            // [1024, 3072) the batched solver's two scalar snapshots
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t tev0 = nullptr, tev1 = nullptr;       // autotuner timing
  std::map<int, int> hop_tune;                       // shape -> threads per site
  int forced_tps = 0;                                // 0: autotune
  bool prof_hop = false;                             // per-launch hop timing
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
  std::vector<double> prof_bytes;
  std::vector<int> prof_shape;                       // per profiled launch: Prec * 1000 + nrhs
  size_t prof_used = 0;
  std::vector<std::unique_ptr<qq::Field>> pool[4];  // temporaries per precision (Prec)
  std::vector<bool> pool_busy[4];
  // Persistent workspaces of the batched solver, by id (qq::ws_get): allocated on first
  // use, grown when a later call needs more, freed with the context.
  std::map<int, std::unique_ptr<qq::DevBuf>> ws;
  cudaStream_t aux_st = nullptr;  // second stream: graph capture of reliable updates

  size_t ref_doubles() const { return (size_t)6 * rd.ntotal * 64; }
};

namespace qq {

// Workspace `id` of the context with at least `bytes` bytes.  Repeated solves of the
// same size reuse it, so they call neither cudaMalloc nor the device-synchronising
// cudaFree.  Ids are owned by one routine at a time (see qq_batch.cu).
inline cudaError_t ws_get(qq_ctx* c, int id, size_t bytes, void** p) {
  auto& slot = c->ws[id];
  if (!slot) slot.reset(new DevBuf());
  const cudaError_t e = slot->alloc(bytes);
  *p = slot->p;
  return e;
}

// Temporary field from the context pool (returned on scope exit).
struct Tmp {
  qq_ctx* c;
  int prec;
  int idx;
  Field* f;
  Tmp(qq_ctx* c_, int prec_);
  ~Tmp();
  Spinor sp() const { return f->sp(); }
  Tmp(const Tmp&) = delete;
  Tmp& operator=(const Tmp&) = delete;
};

// ---- operator and level-1 helpers (qq_ops.cu) ----
int launch_hop_tuned(qq_ctx* c, const HopArgs& a, int prec, int epi);
// Key of the autotuner's table (c->hop_tune) for this launch shape.
int hop_tune_key(qq_ctx* c, const HopArgs& a, int prec, int epi);
int op_hsingle(qq_ctx* c, Spinor out, Spinor in, int idag, int pout);
int op_hsingle_multi(qq_ctx* c, const Spinor* out, const Spinor* in, int n, int idag, int pout);
// he = Hdbletm(ge), tmp is an odd-parity temporary of the same precision.
int op_dbletm(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int idag, const double kappa[2]);
// out = gamma5mult(in) - sigma in (Q/diracops.f90:1750-1860), tmp odd-parity.
int op_g5mult(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int idag, const double kappa[2],
              double sigma);
int op_dbletm_multi(qq_ctx* c, const Spinor* out, const Spinor* in, const Spinor* tmp, int n,
                    int idag, const double kappa[2]);
// RHS-interleaved block fields of nb right-hand sides (element (q, s, r) at
// q * (vh * nb) + s * nb + r); one launch pair for the whole block.
int op_dbletm_block_impl(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int nb, int idag, const double kappa[2],
                         Spinor dot_op, double* dot_part, int dot_mode, int* fused_blocks);
int op_dbletm_block_dot(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int nb, const double kappa[2],
                        Spinor dot_op, double* dot_part, int dot_mode, int* fused_blocks);
int hop_block_count(qq_ctx* c, int nb);
int op_dbletm_block(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int nb, int idag,
                    const double kappa[2]);
int lin(qq_ctx* c, Spinor out, Coef a, Spinor x, Coef b = cimm(0), Spinor y = Spinor{nullptr, nullptr, P64},
        Coef cc = cimm(0), Spinor z = Spinor{nullptr, nullptr, P64}, double* nrm2_dev = nullptr);
int dot_dev(qq_ctx* c, Spinor x, Spinor y, double* out3);  // out3 = {re, im, |y|^2}
int dot_host(qq_ctx* c, Spinor x, Spinor y, std::complex<double>* d, double* ynrm2);
int norm2_host(qq_ctx* c, Spinor x, double* n2);
int copy_field(qq_ctx* c, Spinor out, Spinor in);
int zero_field(qq_ctx* c, Spinor f);
int read_scalars(qq_ctx* c, const double* dev, int n, double* host);

// reference layout <-> GPU layout
int ref_to_field(qq_ctx* c, const double* ref_dev, int parity, Spinor out);
int field_to_ref(qq_ctx* c, Spinor in, int parity, double* ref_dev);
// Stage a caller pointer (host or device) into device memory; returns device ptr.
int stage_in(qq_ctx* c, int slot, const double* p, size_t ndoubles, const double** dev);
int stage_out_begin(qq_ctx* c, int slot, double* p, size_t ndoubles, double** dev);
int stage_out_end(qq_ctx* c, int slot, double* p, size_t ndoubles, double* dev);
bool is_device_ptr(const void* p);

// ---- Krylov solvers (qq_solvers.cu) ----
struct SolveStats {
  int itercount = 0, mvp = 0, ncycles = 0;
  int fallback = 0;     // 1: the reference method finished this solve (qq_solve_info.fallback)
  int finished_by = 0;  // qq_solve_info.finished_by
  int restarts = 0;     // qq_solve_info.restarts
  double true_rel = 0.0;
  std::vector<double> hist;
  std::vector<int> hist_mvp;
  std::vector<std::complex<double>> ritz;
};

// Reference-faithful FP64 GMRES-DR (Q/inverters.f90:2871-3572 semantics).
int gmresdr_fp64(qq_ctx* c, Spinor phi, Spinor x, int m, int k, double resmax, int itermin,
                 const double kappa[2], DeflSpace* defl, SolveStats* st);
// Multi-shift GMRES-DR on gamma5mult (Q/inverters.f90:6041-7179): xs/rs hold one solution
// and one residual field per shift; resid receives ||r_s||.
int gmresdrshift_fp64(qq_ctx* c, Spinor b, const std::vector<Spinor>& xs, const std::vector<Spinor>& rs,
                      const double* sigma, int m, int k, double resmax, int itermin, const double kappa[2],
                      double* resid, SolveStats* st);
int gmresproj_fp64(qq_ctx* c, Spinor b, Spinor x, int m, int k, double resmax, int itermin,
                   const double kappa[2], const DeflSpace& defl, SolveStats* st);
int bicgstab_fp64(qq_ctx* c, Spinor phi, Spinor x, double resmax, int itermin, int maxiter,
                  const double kappa[2], SolveStats* st);
// Mixed precision (FP32 Arnoldi, FP64 residual/solution); returns an FP32 deflation space.
int gmresdr_mixed(qq_ctx* c, Spinor b, Spinor x, int m, int k, double tol, int max_cycles,
                  const double kappa[2], DeflSpace* defl, SolveStats* st);
int defl_project(qq_ctx* c, const DeflSpace& d, Spinor b, Spinor x, Spinor r, const double kappa[2],
                 double* rn);

void fill_info(qq_solve_info* info, int status, const SolveStats& s, double seconds);
// Tune every hopping shape a qq_fermprop_batch(nrhs, meth) launches (qq_batch.cu).
int tune_batch_shapes(qq_ctx* c, int nrhs, const double kappa[2], const qq_method* meth);
// Flexible GMRES(m) with right preconditioner M(z, v): z = M v (qq_solvers.cu).
int fgmres_fp64(qq_ctx* c, Spinor phi, Spinor x, int m, double resmax, int max_cycles, const double kappa[2],
                const std::function<int(Spinor, Spinor)>& M, SolveStats* st, bool* stalled);
// Flexible GMRES-DR(m, k) with right preconditioner M (qq_solvers.cu).
int fgmresdr_fp64(qq_ctx* c, Spinor phi, Spinor x, int m, int k, double resmax, int max_cycles,
                  const double kappa[2], const std::function<int(Spinor, Spinor)>& M, SolveStats* st,
                  bool* stalled);

}  // namespace qq
