// Batched mixed-precision propagators (qq_fermprop_batch).
//
// Method for nrhs sources on one configuration (solver = 1):
//   1. source preparation and odd-half reconstruction exactly as fermprop
//      (Q/quark.f90:595-618, :787-824), in FP64;
//   2. optionally (deflate = 1) mixed-precision GMRES-DR(m, k) on the first source
//      to tolerance defl_tol builds an FP32 deflation space (k harmonic-Ritz vectors);
//   3. the right-hand sides are solved together, in blocks of rhs_block, by BiCGStab
//      on RHS-interleaved block fields in FP64, FP32, FP16 or BF16 with FP64 reliable
//      updates: whenever the iterated residual has dropped by `delta` since the last
//      update, the FP64 solution is updated and the FP64 true residual replaces the
//      low-precision one (projected onto the deflation space when there is one);
//   4. every answer is judged by its FP64 true full-lattice residual.
// solver = 0 runs the plain FP64 GMRES-DR(m, k) of the reference on every RHS.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "qq_ctx.h"
#include "qq_mrhs.cuh"

namespace qq {

namespace {

// Workspace ids of the batched solver in the context (qq_ctx::ws).  Solves of the
// same size reuse the buffers, so a repeated qq_fermprop_batch allocates nothing.
enum WsId : int {
  WS_BLOCK = 0,  // + 2 f: data of block field f (7 fields), + 2 f + 1: its 16-bit norms
  WS_SCAL = 20,  // scalars and control words
  WS_PART,       // reduction partials
  WS_DSLOTS,     // scalar slot of each right-hand side
  WS_HIST,       // true-residual history
  WS_HITS,       // iterations at each history entry
  WS_RHS = 64,   // + 3 i + j: right-hand side i's b, x, r64
};

// A field carved from a context workspace (non-owning).
struct WsField {
  Spinor s{nullptr, nullptr, P64};
  size_t bytes = 0, norm_bytes = 0;
  Spinor sp() const { return s; }
};

int ws_field(qq_ctx* c, WsField& f, int id, int prec, int nsites_mult = 1) {
  void* d = nullptr;
  void* n = nullptr;
  f.bytes = field_bytes(prec, c->g.vh) * nsites_mult;
  QQ_CK(ws_get(c, id, f.bytes, &d));
  f.norm_bytes = 0;
  if (has_norm(prec)) {
    f.norm_bytes = sizeof(float) * c->g.vh * nsites_mult;
    QQ_CK(ws_get(c, id + 1, f.norm_bytes, &n));
  }
  f.s = Spinor{d, static_cast<float*>(n), prec};
  return QQ_OK;
}

// The seven block fields of a batched BiCGStab, zeroed.
int block_fields(qq_ctx* c, int prec, int nb, WsField* const* fs) {
  for (int i = 0; i < 7; ++i) {
    QQ_TRY(ws_field(c, *fs[i], WS_BLOCK + 2 * i, prec, nb));
    QQ_CK(cudaMemsetAsync(fs[i]->s.data, 0, fs[i]->bytes, c->st));
    if (has_norm(prec)) QQ_CK(cudaMemsetAsync(fs[i]->s.norm, 0, fs[i]->norm_bytes, c->st));
  }
  return QQ_OK;
}

struct PerRhs {
  WsField b, x;                // FP64 even-system source and solution
  WsField r64;                 // FP64 residual
  double bn = 0.0, rmax = 0.0, rn = 0.0;
  bool done = false;
};

template <int P>
int launch_block_op(qq_ctx* c, const BlockBiArgs& A, int op) {
  const int tb = A.nb * (kRedThreads / A.nb);
  switch (op) {
    case OP_DOT_RHAT_R: bicg_block_kernel<P, OP_DOT_RHAT_R><<<kRedBlocks, tb, 0, c->st>>>(A); break;
    case OP_P_UPDATE: bicg_block_kernel<P, OP_P_UPDATE><<<kRedBlocks, tb, 0, c->st>>>(A); break;
    case OP_DOT_RHAT_V: bicg_block_kernel<P, OP_DOT_RHAT_V><<<kRedBlocks, tb, 0, c->st>>>(A); break;
    case OP_S_UPDATE: bicg_block_kernel<P, OP_S_UPDATE><<<kRedBlocks, tb, 0, c->st>>>(A); break;
    case OP_DOTS_T: bicg_block_kernel<P, OP_DOTS_T><<<kRedBlocks, tb, 0, c->st>>>(A); break;
    case OP_XR_UPDATE: bicg_block_kernel<P, OP_XR_UPDATE><<<kRedBlocks, tb, 0, c->st>>>(A); break;
    default: return set_error(QQ_BAD_ARG, "bad batched op");
  }
  QQ_CK(cudaGetLastError());
  return QQ_OK;
}

struct ScalarCtl {
  unsigned* ctl;     // control words (active, pending)
  double delta;      // reliable-update threshold
  double half_tol;   // 0.5 * tolerance
  int window;        // stall window in iterations (0: none)
};

int block_op(qq_ctx* c, int prec, const BlockBiArgs& A, int op, const int* dslots, int step,
             const ScalarCtl& sc) {
  count_launch(step >= 0 ? 2 : 1);
  if (prec == P32)
    QQ_TRY(launch_block_op<P32>(c, A, op));
  else if (prec == P16)
    QQ_TRY(launch_block_op<P16>(c, A, op));
  else if (prec == PB16)
    QQ_TRY(launch_block_op<PB16>(c, A, op));
  else
    QQ_TRY(launch_block_op<P64>(c, A, op));
  if (step >= 0) {
    bicg_scalar_kernel<<<A.nb, 256, 0, c->st>>>(A.S, dslots, A.partial, kRedBlocks, step, sc.ctl,
                                                sc.delta, sc.half_tol, sc.window);
    QQ_CK(cudaGetLastError());
  }
  return QQ_OK;
}

// The scalar step alone, on partials already written (by a hop with a fused dot product,
// one per hop block: a long list, folded by a grid first).
int scalar_step(qq_ctx* c, const BlockBiArgs& A, const int* dslots, int step, int nblocks, const ScalarCtl& sc) {
  const double* part = A.partial;
  if (nblocks > 2 * kFoldChunks) {
    count_launch();
    partial_fold_kernel<<<dim3(kFoldChunks, A.nb), 256, 0, c->st>>>(A.partial, nblocks, A.partial2, kFoldChunks);
    QQ_CK(cudaGetLastError());
    part = A.partial2;
    nblocks = kFoldChunks;
  }
  count_launch();
  bicg_scalar_kernel<<<A.nb, 256, 0, c->st>>>(A.S, dslots, part, nblocks, step, sc.ctl, sc.delta,
                                              sc.half_tol, sc.window);
  QQ_CK(cudaGetLastError());
  return QQ_OK;
}

// v = A p with <rhat, v> (step ST_ALPHA), or t = A s with <t, s>, ||t||^2 (ST_OMEGA):
// fused into the second hop when its kernel supports it, else a separate reduction.
int op_and_dot(qq_ctx* c, int prec, const BlockBiArgs& A, Spinor out, Spinor in, Spinor tmp, Spinor dot_op,
               int mode, const double kappa[2], const int* dslots, const ScalarCtl& sc) {
  int fb = 0;
  QQ_TRY(op_dbletm_block_dot(c, out, in, tmp, A.nb, kappa, dot_op, A.partial, mode, &fb));
  const int step = mode == 1 ? ST_ALPHA : ST_OMEGA;
  if (fb) return scalar_step(c, A, dslots, step, fb, sc);
  return block_op(c, prec, A, mode == 1 ? OP_DOT_RHAT_V : OP_DOTS_T, dslots, step, sc);
}

// mode 0: block[k] = x ; 1: x += block[k] ; 2: block[k] = 0.  With `pred`, only when
// bit k of the device word *pred is set.
int block_slot(qq_ctx* c, int prec, int nb, int k, Spinor blockf, Spinor x, int mode,
               const unsigned* pred = nullptr) {
  count_launch();
  if (prec == P32)
    block_slot_kernel<P32><<<kRedBlocks, kRedThreads, 0, c->st>>>(c->g.vh, nb, k, blockf, x, mode, pred);
  else if (prec == P16)
    block_slot_kernel<P16><<<kRedBlocks, kRedThreads, 0, c->st>>>(c->g.vh, nb, k, blockf, x, mode, pred);
  else if (prec == PB16)
    block_slot_kernel<PB16><<<kRedBlocks, kRedThreads, 0, c->st>>>(c->g.vh, nb, k, blockf, x, mode, pred);
  else
    block_slot_kernel<P64><<<kRedBlocks, kRedThreads, 0, c->st>>>(c->g.vh, nb, k, blockf, x, mode, pred);
  QQ_CK(cudaGetLastError());
  return QQ_OK;
}

// Stall window of the batched BiCGStab (iterations without a 10x fall of the FP64 true
// residual) when the method leaves it at 0.
constexpr int kStallWindow = 2000;
// The same for a 16-bit iteration, which the batched FP32 iteration continues when it
// stops: near critical kappa it stalls at a true residual of ~1e-2 (11 or 8 significant
// bits), so a shorter window hands it over sooner; where 16-bit converges it gains 10x in
// far fewer iterations (about 15 at kappa = 0.15).
constexpr int kStallWindow16 = 400;

// Iteration limit of the batched BiCGStab when the method sets none: 40 iterations per
// lattice extent per decade of tolerance, clamped to [2000, 100000] -- 20,000 for
// 24^3x48 at 1e-10, 3,600 for 8^4.  Near critical kappa the iteration count grows with
// the lattice extent (the lowest Dirac mode falls like 1/L), and linearly with the
// decades to cover.
int default_maxiter(const Geom& g, double tol) {
  const int lmax = std::max(std::max(g.n[0], g.n[1]), std::max(g.n[2], g.n[3]));
  const double decades = std::max(1.0, std::ceil(-std::log10(std::max(tol, 1e-300))));
  return (int)std::min(100000.0, std::max(2000.0, 40.0 * lmax * decades));
}

// After right-hand side k's FP64 residual went back into slot k of r: the next
// iteration's rho' = <rhat, r> and beta for k alone (the fused dot of the iteration saw
// the old residual).  pred: the insert mask (graph and host-driven loops), or nullptr
// (the host did the insertion).
int reinsert_rho(qq_ctx* c, int prec, const BlockBiArgs& A, int k, const int* dslots, unsigned* ctl,
                 const unsigned* pred) {
  count_launch(2);
  if (prec == P32)
    slot_dot_kernel<P32><<<kRedBlocks, kRedThreads, 0, c->st>>>(A.vh, A.nb, k, A.rhat, A.r, pred, A.partial);
  else if (prec == P16)
    slot_dot_kernel<P16><<<kRedBlocks, kRedThreads, 0, c->st>>>(A.vh, A.nb, k, A.rhat, A.r, pred, A.partial);
  else if (prec == PB16)
    slot_dot_kernel<PB16><<<kRedBlocks, kRedThreads, 0, c->st>>>(A.vh, A.nb, k, A.rhat, A.r, pred, A.partial);
  else
    slot_dot_kernel<P64><<<kRedBlocks, kRedThreads, 0, c->st>>>(A.vh, A.nb, k, A.rhat, A.r, pred, A.partial);
  QQ_CK(cudaGetLastError());
  reliable_rho_kernel<<<1, 256, 0, c->st>>>(A.S, dslots, ctl, k, A.partial, kRedBlocks, pred ? 0 : 1);
  QQ_CK(cudaGetLastError());
  return QQ_OK;
}

bool host_loop_forced() {
  const char* e = std::getenv("QQ_HOST_LOOP");  // testing: the host-driven loop
  return e && std::atoi(e) != 0;
}

// The graph of the graph-driven batched BiCGStab: WHILE(iteration; IF(pending k) update k
// for every k; loop condition).  Built by stream capture into the conditional nodes'
// body graphs; per_iter and per_update count the library kernels of one iteration and
// of one reliable update, for the launch counter.
struct GraphLoop {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t aux = nullptr;  // the context's second stream (kept with the context)
  long long per_iter = 0, per_update = 0;
  // The launches of a finished run: iters iterations and nupd reliable updates.
  void count(long long iters, long long nupd) const { count_launch(per_iter * iters + per_update * nupd); }
  ~GraphLoop() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  template <class Chunk, class Update>
  int build(qq_ctx* c, int nb, unsigned* ctl, unsigned all, int maxiter, Chunk& chunk, Update& update) {
    if (!c->aux_st) QQ_CK(cudaStreamCreateWithFlags(&c->aux_st, cudaStreamNonBlocking));
    aux = c->aux_st;
    QQ_CK(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle hw;
    QQ_CK(cudaGraphConditionalHandleCreate(&hw, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hw;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wn;
    QQ_CK(cudaGraphAddNode(&wn, graph, nullptr, 0, &wp));
    CondHandles hs = {};
    for (int k = 0; k < nb; ++k) QQ_CK(cudaGraphConditionalHandleCreate(&hs.h[k], wp.conditional.phGraph_out[0], 0, 0));
    // launches are counted per host thread, so contexts capturing side by side (the
    // uneven batch) do not pick up each other's launches
    const long long n0 = thread_launch_count();
    QQ_CK(cudaStreamBeginCaptureToGraph(c->st, wp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
    int rc = chunk();
    per_iter = thread_launch_count() - n0 + 2;  // + the two condition kernels
    if (rc == QQ_OK) {
      count_launch();
      reliable_conds_kernel<<<1, 32, 0, c->st>>>(ctl, hs, nb);
      if (cudaGetLastError() != cudaSuccess) rc = set_error(QQ_CUDA_ERR, "condition kernel launch failed");
    }
    for (int k = 0; k < nb && rc == QQ_OK; ++k) {
      cudaStreamCaptureStatus cs;
      cudaGraph_t cg = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t nd = 0;
      cudaGraphNodeParams ip = {};
      ip.type = cudaGraphNodeTypeConditional;
      ip.conditional.handle = hs.h[k];
      ip.conditional.type = cudaGraphCondTypeIf;
      ip.conditional.size = 1;
      cudaGraphNode_t in;
      if (cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &cg, &deps, &nd) != cudaSuccess ||
          cudaGraphAddNode(&in, cg, deps, nd, &ip) != cudaSuccess ||
          cudaStreamUpdateCaptureDependencies(c->st, &in, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) {
        rc = set_error(QQ_CUDA_ERR, "conditional node construction failed");
        break;
      }
      // the IF body: right-hand side k's update, captured from the second stream
      std::swap(c->st, aux);
      const long long m0 = thread_launch_count();
      if (cudaStreamBeginCaptureToGraph(c->st, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        std::swap(c->st, aux);
        rc = set_error(QQ_CUDA_ERR, "capture of a reliable update failed");
        break;
      }
      rc = update(k);
      per_update = thread_launch_count() - m0;
      cudaGraph_t ig = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(c->st, &ig);
      std::swap(c->st, aux);
      if (rc == QQ_OK && ee != cudaSuccess) rc = set_error(QQ_CUDA_ERR, "capture of a reliable update failed");
    }
    if (rc == QQ_OK) {
      count_launch();
      loop_cond_kernel<<<1, 1, 0, c->st>>>(ctl, all, (unsigned)maxiter, hw);
      if (cudaGetLastError() != cudaSuccess) rc = set_error(QQ_CUDA_ERR, "condition kernel launch failed");
    }
    cudaGraph_t bg = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->st, &bg);
    count_launch(-(thread_launch_count() - n0));  // captured, not launched: counted when the graph runs
    if (rc != QQ_OK) return rc;
    QQ_CK(e);
    QQ_CK(cudaGraphInstantiate(&exec, graph, 0));
    return QQ_OK;
  }
};

int full_residual(qq_ctx* c, Spinor be, Spinor bo, Spinor xe, Spinor xo, const double kappa[2],
                  double* rel) {
  Tmp h(c, P64), m(c, P64);
  const double tk = 2.0 * kappa[0] * kappa[1];
  double num = 0.0, den = 0.0;
  for (int par = 0; par < 2; ++par) {
    Spinor xs = par == 0 ? xe : xo, xother = par == 0 ? xo : xe, bs = par == 0 ? be : bo;
    QQ_TRY(op_hsingle(c, h.sp(), xother, 0, par));
    // m = x + tk J x - kappa H x_other ; then r = b - m
    QQ_CK(launch_spinmix(c->g.vh, xs, h.sp(), m.sp(), 1.0, tk, -kappa[0], 0.0, P64, c->st));
    double* s = c->scal.as<double>();
    QQ_TRY(lin(c, m.sp(), cimm(1.0), bs, cimm(-1.0), m.sp(), cimm(0), Spinor{nullptr, nullptr, P64}, s));
    double n2 = 0.0, b2 = 0.0;
    QQ_TRY(read_scalars(c, s, 1, &n2));
    QQ_TRY(norm2_host(c, bs, &b2));
    num += n2;
    den += b2;
  }
  *rel = std::sqrt(num / den);
  return QQ_OK;
}

// Scalars of a right-hand side before its first iteration: rhat = r = the FP64
// residual of the initial guess, whose norm also anchors the stall test.
void init_scalars(double* sc, const PerRhs& R) {
  // rhat = r = the residual, so rho = <rhat, r> = ||r||^2; with p = v = 0 the first
  // P_UPDATE gives p = r whatever beta is
  sc[SC_ALPHA] = sc[SC_OMEGA] = 1.0;
  sc[SC_RHO] = R.rn * R.rn;
  sc[SC_RHO + 1] = 0.0;
  sc[SC_BETA] = sc[SC_BETA + 1] = 0.0;
  sc[SC_RMAX] = R.rmax;
  sc[SC_BN] = R.bn > 0.0 ? R.bn : 1.0;
  sc[SC_R2] = R.rn * R.rn;
  sc[SC_RHATN] = R.rn;
  sc[SC_CHK_R] = R.rn;
  sc[SC_CHK_ITS] = 0.0;
  sc[SC_FAIL] = 0.0;
  sc[SC_NRST] = 0.0;
}

}  // namespace

// BiCGStab on a block of right-hand sides in precision `prec` (block fields), FP64
// reliable updates (Sleijpen & van der Vorst): when ||r|| has dropped by `delta` since
// the last update, x64 += x_low, the FP64 true residual replaces the iterated one
// (projected onto the deflation space first, if any) and the iteration continues with
// the same search direction.
int bicgstab_block_sync(qq_ctx* c, std::vector<PerRhs*>& rhs, int prec, double tol, double delta,
                        int maxiter, int window, const double kappa[2], const DeflSpace* defl,
                        std::vector<SolveStats>& stats) {
  const int nb = (int)rhs.size();
  if (nb == 0) return QQ_OK;
  if (nb > kMaxBatch) return set_error(QQ_BAD_ARG, "too many right-hand sides in one block");
  WsField r, rhat, p, v, t, xl, tmp;
  {
    WsField* const fs[7] = {&r, &rhat, &p, &v, &t, &xl, &tmp};
    QQ_TRY(block_fields(c, prec, nb, fs));
  }
  // scalars of every right-hand side, then the control words
  constexpr size_t kScalDoubles = (size_t)kScal * kMaxBatch;
  constexpr size_t kSyncDoubles = kScalDoubles + (kCtlWords + 1) / 2;
  double *Sd = nullptr, *partd = nullptr;
  int* ds = nullptr;
  QQ_CK(ws_get(c, WS_SCAL, sizeof(double) * (kSyncDoubles), reinterpret_cast<void**>(&Sd)));
  const size_t npart = (size_t)3 * std::max(kRedBlocks, hop_block_count(c, nb)) * kMaxBatch;
  QQ_CK(ws_get(c, WS_PART, sizeof(double) * (npart + (size_t)3 * kFoldChunks * kMaxBatch),
               reinterpret_cast<void**>(&partd)));
  QQ_CK(ws_get(c, WS_DSLOTS, sizeof(int) * kMaxBatch, reinterpret_cast<void**>(&ds)));
  unsigned* ctl = reinterpret_cast<unsigned*>(Sd + kScalDoubles);
  Tmp tmp64(c, P64), h(c, P64);
  double* s1 = c->scal.as<double>();
  // FP64 residual of x (and of the deflated x) -> slot k of r and rhat
  auto true_res = [&](PerRhs& R, SolveStats& st) -> int {
    QQ_TRY(op_dbletm(c, h.sp(), R.x.sp(), tmp64.sp(), 0, kappa));
    QQ_TRY(lin(c, R.r64.sp(), cimm(1.0), R.b.sp(), cimm(-1.0), h.sp(), cimm(0), Spinor{nullptr, nullptr, P64}, s1));
    double n2;
    QQ_TRY(read_scalars(c, s1, 1, &n2));
    R.rn = std::sqrt(n2);
    st.mvp += 1;
    if (defl && defl->k > 0 && R.rn / R.bn > tol) {
      QQ_TRY(defl_project(c, *defl, R.b.sp(), R.x.sp(), R.r64.sp(), kappa, &R.rn));
      st.mvp += 1;
    }
    return QQ_OK;
  };
  // host mirror in the solver's half of the context's pinned buffer
  static_assert(kSyncDoubles <= 1024, "scalar mirror exceeds the pinned buffer");
  double* hS = c->hpin + 1024;
  std::fill(hS, hS + kSyncDoubles, 0.0);
  unsigned* hctl = reinterpret_cast<unsigned*>(hS + kScalDoubles);
  std::vector<int> slots(nb);
  unsigned active = 0;
  for (int k = 0; k < nb; ++k) {
    PerRhs& R = *rhs[k];
    slots[k] = k;
    QQ_TRY(norm2_host(c, R.b.sp(), &R.bn));
    R.bn = std::sqrt(R.bn);
    QQ_TRY(true_res(R, stats[k]));
    R.rmax = R.rn;
    R.done = !(R.bn > 0.0) || R.rn / R.bn <= tol;
    stats[k].true_rel = R.bn > 0.0 ? R.rn / R.bn : 0.0;
    if (!R.done) active |= 1u << k;
    QQ_TRY(block_slot(c, prec, nb, k, r.sp(), R.r64.sp(), 0));
    QQ_TRY(block_slot(c, prec, nb, k, rhat.sp(), R.r64.sp(), 0));
    init_scalars(&hS[(size_t)k * kScal], R);
  }
  hctl[CTL_ACTIVE] = active;
  hctl[CTL_PENDING] = 0u;
  QQ_CK(cudaMemcpyAsync(Sd, hS, sizeof(double) * (kSyncDoubles), cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaMemcpyAsync(ds, slots.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  BlockBiArgs A;
  std::memset(&A, 0, sizeof(A));
  A.vh = c->g.vh;
  A.nb = nb;
  A.active = ctl + CTL_ACTIVE;
  A.r = r.sp();
  A.rhat = rhat.sp();
  A.p = p.sp();
  A.v = v.sp();
  A.t = t.sp();
  A.x = xl.sp();
  for (int k = 0; k < nb; ++k) A.slot[k] = k;
  A.S = Sd;
  A.partial = partd;
  A.partial2 = partd + npart;
  const ScalarCtl sc{ctl, delta, 0.5 * tol, window};
  // Iterations run in chunks without host synchronisation: a right-hand side whose
  // residual calls for a reliable update (or may have converged) takes itself out of
  // the active mask on the device and waits, pending, for the end of the chunk, where
  // the host does the FP64 update and puts it back.
  constexpr int kChunk = 4;
  int done_its = 0;
  while (active && done_its < maxiter) {
    const int nchunk = std::min(kChunk, maxiter - done_its);
    for (int i = 0; i < nchunk; ++i) {
      QQ_TRY(block_op(c, prec, A, OP_P_UPDATE, ds, -1, sc));
      QQ_TRY(op_and_dot(c, prec, A, v.sp(), p.sp(), tmp.sp(), rhat.sp(), 1, kappa, ds, sc));
      QQ_TRY(block_op(c, prec, A, OP_S_UPDATE, ds, -1, sc));
      QQ_TRY(op_and_dot(c, prec, A, t.sp(), r.sp(), tmp.sp(), r.sp(), 2, kappa, ds, sc));
      QQ_TRY(block_op(c, prec, A, OP_XR_UPDATE, ds, ST_R2, sc));
    }
    done_its += nchunk;
    QQ_CK(cudaMemcpyAsync(hS, Sd, sizeof(double) * (kSyncDoubles), cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    // right-hand sides the device stopped (NaN, breakdown, stagnation) leave the loop
    const unsigned failed = hctl[CTL_FAIL] & active;
    for (int k = 0; k < nb; ++k)
      if ((failed >> k) & 1u) stats[k].fallback = (int)hS[(size_t)k * kScal + SC_FAIL];
    active &= ~failed;
    const unsigned pending = hctl[CTL_PENDING] & active;
    unsigned back = 0;  // right-hand sides that iterate again after their update
    for (int k = 0; k < nb; ++k) {
      PerRhs& R = *rhs[k];
      SolveStats& st = stats[k];
      const int its = (int)hS[(size_t)k * kScal + SC_ITS];
      st.mvp += 2 * (its - st.itercount);
      st.itercount = its;
      st.restarts = (int)hS[(size_t)k * kScal + SC_NRST];
      if (!((pending >> k) & 1u)) continue;
      double* sk = &hS[(size_t)k * kScal];
      // reliable update
      QQ_TRY(block_slot(c, prec, nb, k, xl.sp(), R.x.sp(), 1));
      QQ_TRY(block_slot(c, prec, nb, k, xl.sp(), R.x.sp(), 2));
      QQ_TRY(true_res(R, st));
      st.true_rel = R.rn / R.bn;
      st.hist.push_back(st.true_rel);
      st.hist_mvp.push_back(st.mvp);
      if (R.rn < 0.1 * sk[SC_CHK_R]) {  // progress anchor of the stall test
        sk[SC_CHK_R] = R.rn;
        sk[SC_CHK_ITS] = its;
      }
      const bool restart = (hctl[CTL_RESTART] >> k) & 1u;
      hctl[CTL_RESTART] &= ~(1u << k);
      if (!std::isfinite(R.rn)) {
        st.fallback = FAIL_NAN;
        active &= ~(1u << k);
        continue;
      }
      if (R.rn / R.bn <= tol) {
        R.done = true;
        active &= ~(1u << k);
        continue;
      }
      QQ_TRY(block_slot(c, prec, nb, k, r.sp(), R.r64.sp(), 0));
      if (restart) {  // the residual becomes the shadow residual (reinsert_rho sees the mark)
        QQ_TRY(block_slot(c, prec, nb, k, rhat.sp(), R.r64.sp(), 0));
        hctl[CTL_RESTART] |= 1u << k;
      }
      R.rmax = R.rn;
      sk[SC_RMAX] = R.rmax;
      sk[SC_R2] = R.rn * R.rn;
      back |= 1u << k;
    }
    if (pending || failed) {
      active = (hctl[CTL_ACTIVE] | back) & active;
      hctl[CTL_ACTIVE] = active;
      hctl[CTL_PENDING] = 0u;
      QQ_CK(cudaMemcpyAsync(Sd, hS, sizeof(double) * (kSyncDoubles), cudaMemcpyHostToDevice, c->st));
      for (int k = 0; k < nb; ++k)  // rho and beta of the re-inserted residuals, on the device
        if ((back >> k) & 1u) QQ_TRY(reinsert_rho(c, prec, A, k, ds, ctl, nullptr));
    }
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  for (int k = 0; k < nb; ++k)
    if (!rhs[k]->done && stats[k].fallback == FAIL_NONE) stats[k].fallback = FAIL_MAXITER;
  bool all_done = true;
  for (auto* R : rhs) all_done = all_done && R->done;
  return all_done ? QQ_OK : QQ_NOT_CONVERGED;
}

// Device-driven variant (no deflation): the reliable update itself runs on the device
// -- the FP64 true residual, its norm, the convergence decision, the re-insertion of
// the residual and the re-activation are stream-ordered kernels, the decision a
// one-thread kernel.  Two drivers share those kernels:
//  - graph loop (default): one CUDA graph holds the whole solve.  A WHILE conditional
//    node repeats the iteration; after it one IF node per right-hand side runs that
//    right-hand side's reliable update when it went pending, and a one-thread kernel
//    sets the WHILE condition (some right-hand side still moving, fewer than maxiter
//    iterations).  The host launches the graph once and waits, so a descheduled host
//    thread cannot leave the GPU idle, and a pending right-hand side resumes in the
//    next iteration.  The true-residual history is recorded on the device.
//  - host loop (when hop profiling is on, or QQ_HOST_LOOP=1): the host queues an
//    iteration and a snapshot of the scalars, reads the previous snapshot while it
//    runs and queues the updates of right-hand sides that went pending.  Updates queued
//    at step c are visible from snapshot c + 1 on, so earlier snapshots' pending marks
//    for them are skipped.
int bicgstab_block(qq_ctx* c, std::vector<PerRhs*>& rhs, int prec, double tol, double delta,
                   int maxiter, int window, const double kappa[2], const DeflSpace* defl,
                   std::vector<SolveStats>& stats) {
  if (defl && defl->k > 0)
    return bicgstab_block_sync(c, rhs, prec, tol, delta, maxiter, window, kappa, defl, stats);
  const int nb = (int)rhs.size();
  if (nb == 0) return QQ_OK;
  if (nb > kMaxBatch) return set_error(QQ_BAD_ARG, "too many right-hand sides in one block");
  WsField r, rhat, p, v, t, xl, tmp;
  {
    WsField* const fs[7] = {&r, &rhat, &p, &v, &t, &xl, &tmp};
    QQ_TRY(block_fields(c, prec, nb, fs));
  }
  constexpr size_t kScalDoubles = (size_t)kScal * kMaxBatch;
  constexpr size_t kSnap = kScalDoubles + (kCtlWords + 1) / 2;  // scalars + control words
  constexpr int kHist = 1024;  // true-residual history per right-hand side (qq_solve_info)
  const size_t sbytes = sizeof(double) * kSnap;
  static_assert(1024 + 2 * kSnap <= 3072, "snapshots exceed the pinned buffer");
  double *Sd = nullptr, *partd = nullptr, *dhist = nullptr;
  int *ds = nullptr, *dhits = nullptr;
  QQ_CK(ws_get(c, WS_SCAL, sbytes, reinterpret_cast<void**>(&Sd)));
  QQ_CK(ws_get(c, WS_HIST, sizeof(double) * kHist * nb, reinterpret_cast<void**>(&dhist)));
  QQ_CK(ws_get(c, WS_HITS, sizeof(int) * kHist * nb, reinterpret_cast<void**>(&dhits)));
  const size_t npart = (size_t)3 * std::max(kRedBlocks, hop_block_count(c, nb)) * kMaxBatch;
  QQ_CK(ws_get(c, WS_PART, sizeof(double) * (npart + (size_t)3 * kFoldChunks * kMaxBatch),
               reinterpret_cast<void**>(&partd)));
  QQ_CK(ws_get(c, WS_DSLOTS, sizeof(int) * kMaxBatch, reinterpret_cast<void**>(&ds)));
  unsigned* ctl = reinterpret_cast<unsigned*>(Sd + kScalDoubles);
  double* snap[2] = {c->hpin + 1024, c->hpin + 1024 + kSnap};
  Tmp tmp64(c, P64), h(c, P64);
  double* s1 = c->scal.as<double>();
  // initial FP64 residuals (synchronous, once)
  double* hS = snap[0];
  std::fill(hS, hS + kSnap, 0.0);
  unsigned* hctl = reinterpret_cast<unsigned*>(hS + kScalDoubles);
  std::vector<int> slots(nb);
  unsigned active = 0, done = 0;
  for (int k = 0; k < nb; ++k) {
    PerRhs& R = *rhs[k];
    slots[k] = k;
    QQ_TRY(norm2_host(c, R.b.sp(), &R.bn));
    R.bn = std::sqrt(R.bn);
    QQ_TRY(op_dbletm(c, h.sp(), R.x.sp(), tmp64.sp(), 0, kappa));
    QQ_TRY(lin(c, R.r64.sp(), cimm(1.0), R.b.sp(), cimm(-1.0), h.sp(), cimm(0), Spinor{nullptr, nullptr, P64}, s1));
    double n2;
    QQ_TRY(read_scalars(c, s1, 1, &n2));
    R.rn = std::sqrt(n2);
    stats[k].mvp += 1;
    R.rmax = R.rn;
    R.done = !(R.bn > 0.0) || R.rn / R.bn <= tol;
    stats[k].true_rel = R.bn > 0.0 ? R.rn / R.bn : 0.0;
    if (R.done)
      done |= 1u << k;
    else
      active |= 1u << k;
    QQ_TRY(block_slot(c, prec, nb, k, r.sp(), R.r64.sp(), 0));
    QQ_TRY(block_slot(c, prec, nb, k, rhat.sp(), R.r64.sp(), 0));
    init_scalars(&hS[(size_t)k * kScal], R);
  }
  hctl[CTL_ACTIVE] = active;
  hctl[CTL_DONE] = done;
  QQ_CK(cudaMemcpyAsync(Sd, hS, sbytes, cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaMemcpyAsync(ds, slots.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  const unsigned all = nb == 32 ? 0xffffffffu : (1u << nb) - 1u;
  if ((done & all) == all) return QQ_OK;
  BlockBiArgs A;
  std::memset(&A, 0, sizeof(A));
  A.vh = c->g.vh;
  A.nb = nb;
  A.active = ctl + CTL_ACTIVE;
  A.r = r.sp();
  A.rhat = rhat.sp();
  A.p = p.sp();
  A.v = v.sp();
  A.t = t.sp();
  A.x = xl.sp();
  for (int k = 0; k < nb; ++k) A.slot[k] = k;
  A.S = Sd;
  A.partial = partd;
  A.partial2 = partd + npart;
  const ScalarCtl sctl{ctl, delta, 0.5 * tol, window};
  constexpr int kChunk = 1;  // a pending RHS idles 1-2 iterations before its update runs
  auto run_chunk = [&]() -> int {
    for (int i = 0; i < kChunk; ++i) {
      QQ_TRY(block_op(c, prec, A, OP_P_UPDATE, ds, -1, sctl));
      QQ_TRY(op_and_dot(c, prec, A, v.sp(), p.sp(), tmp.sp(), rhat.sp(), 1, kappa, ds, sctl));
      QQ_TRY(block_op(c, prec, A, OP_S_UPDATE, ds, -1, sctl));
      QQ_TRY(op_and_dot(c, prec, A, t.sp(), r.sp(), tmp.sp(), r.sp(), 2, kappa, ds, sctl));
      QQ_TRY(block_op(c, prec, A, OP_XR_UPDATE, ds, ST_R2, sctl));
    }
    return QQ_OK;
  };
  // right-hand side k's reliable update, all on the device
  auto reliable = [&](int k) -> int {
    PerRhs& R = *rhs[k];
    QQ_TRY(block_slot(c, prec, nb, k, xl.sp(), R.x.sp(), 1));
    QQ_TRY(block_slot(c, prec, nb, k, xl.sp(), R.x.sp(), 2));
    QQ_TRY(op_dbletm(c, h.sp(), R.x.sp(), tmp64.sp(), 0, kappa));
    QQ_TRY(lin(c, R.r64.sp(), cimm(1.0), R.b.sp(), cimm(-1.0), h.sp(), cimm(0), Spinor{nullptr, nullptr, P64},
               Sd + (size_t)k * kScal + SC_T2));
    count_launch(2);
    reliable_decide_kernel<<<1, 1, 0, c->st>>>(Sd, ds, ctl, k, tol, dhist, dhits, kHist);
    QQ_CK(cudaGetLastError());
    QQ_TRY(block_slot(c, prec, nb, k, r.sp(), R.r64.sp(), 0, ctl + CTL_INSERT));
    QQ_TRY(block_slot(c, prec, nb, k, rhat.sp(), R.r64.sp(), 0, ctl + CTL_RESTART));  // a restart
    QQ_TRY(reinsert_rho(c, prec, A, k, ds, ctl, ctl + CTL_INSERT));
    reliable_resume_kernel<<<1, 1, 0, c->st>>>(ctl, k);
    QQ_CK(cudaGetLastError());
    return QQ_OK;
  };
  if (!c->prof_hop && !host_loop_forced()) {
    // every hop shape of the loop is tuned here, outside the capture (the autotuner
    // times its candidates with synchronising events); v is overwritten before use
    QQ_TRY(op_dbletm_block(c, v.sp(), p.sp(), tmp.sp(), nb, 0, kappa));
    QQ_CK(cudaStreamSynchronize(c->st));
    GraphLoop gl;
    QQ_TRY(gl.build(c, nb, ctl, all, maxiter, run_chunk, reliable));
    QQ_CK(cudaGraphLaunch(gl.exec, c->st));
    QQ_CK(cudaMemcpyAsync(hS, Sd, sbytes, cudaMemcpyDeviceToHost, c->st));
    std::vector<double> hist((size_t)kHist * nb);
    std::vector<int> hits((size_t)kHist * nb);
    QQ_CK(cudaMemcpyAsync(hist.data(), dhist, sizeof(double) * hist.size(), cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaMemcpyAsync(hits.data(), dhits, sizeof(int) * hits.size(), cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    const unsigned* hc = reinterpret_cast<const unsigned*>(hS + kScalDoubles);
    long long nupd_all = 0;
    const unsigned failed = hc[CTL_FAIL] & all;
    for (int k = 0; k < nb; ++k) {
      SolveStats& st = stats[k];
      const double* sk = hS + (size_t)k * kScal;
      const int its = (int)sk[SC_ITS], nupd = (int)sk[SC_NUPD];
      st.itercount = its;
      st.mvp += 2 * its + nupd;
      for (int j = 0; j < std::min(nupd, kHist); ++j) {
        st.hist.push_back(hist[(size_t)k * kHist + j]);
        st.hist_mvp.push_back(1 + 2 * hits[(size_t)k * kHist + j] + j + 1);
      }
      if (nupd > 0) st.true_rel = sk[SC_TRUE];
      nupd_all += nupd;
      if ((failed >> k) & 1u) st.fallback = (int)sk[SC_FAIL];
      st.restarts = (int)sk[SC_NRST];
    }
    gl.count(hc[CTL_ITER], nupd_all);
    done = hc[CTL_DONE] & ~failed;  // converged
    for (int k = 0; k < nb; ++k) {
      rhs[k]->done = (done >> k) & 1u;
      if (!rhs[k]->done && stats[k].fallback == FAIL_NONE) stats[k].fallback = FAIL_MAXITER;
    }
    return (done & all) == all ? QQ_OK : QQ_NOT_CONVERGED;
  }
  cudaEvent_t ev[2];
  QQ_CK(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  QQ_CK(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } evg{ev};
  std::vector<int> enq(nb, -1), nupd_seen(nb, 0);
  unsigned failed = 0;
  int chunks = 0;
  QQ_TRY(run_chunk());
  ++chunks;
  QQ_CK(cudaMemcpyAsync(snap[0], Sd, sbytes, cudaMemcpyDeviceToHost, c->st));
  QQ_CK(cudaEventRecord(ev[0], c->st));
  bool expect_active = true;
  int rc = QQ_OK;
  for (int step = 1;; ++step) {
    const bool more = expect_active && (long long)chunks * kChunk < maxiter;
    if (more) {
      QQ_TRY(run_chunk());
      ++chunks;
    }
    QQ_CK(cudaMemcpyAsync(snap[step % 2], Sd, sbytes, cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaEventRecord(ev[step % 2], c->st));
    // snapshot step - 1, taken before everything queued at this step
    QQ_CK(cudaEventSynchronize(ev[(step - 1) % 2]));
    const double* sv = snap[(step - 1) % 2];
    const unsigned* sc = reinterpret_cast<const unsigned*>(sv + kScalDoubles);
    const int sidx = step - 1;
    for (int k = 0; k < nb; ++k) {
      SolveStats& st = stats[k];
      const double* sk = sv + (size_t)k * kScal;
      const int its = (int)sk[SC_ITS];
      st.mvp += 2 * (its - st.itercount);
      st.itercount = its;
      const int nupd = (int)sk[SC_NUPD];
      if (nupd > nupd_seen[k]) {
        const double rel = sk[SC_TRUE];
        st.mvp += nupd - nupd_seen[k];
        st.true_rel = rel;
        st.hist.push_back(rel);
        st.hist_mvp.push_back(st.mvp);
        nupd_seen[k] = nupd;
      }
    }
    failed = sc[CTL_FAIL] & all;
    done = sc[CTL_DONE];  // converged or stopped
    if ((done & all) == all) break;
    const unsigned pend = sc[CTL_PENDING] & ~done;
    bool queued = false, inflight = false;
    for (int k = 0; k < nb; ++k) {
      if (enq[k] >= sidx) inflight = true;
      if (!((pend >> k) & 1u) || enq[k] >= sidx) continue;
      QQ_TRY(reliable(k));
      enq[k] = step;
      queued = true;
    }
    const unsigned act = sc[CTL_ACTIVE] & ~done;
    expect_active = act != 0 || queued || inflight;
    if (!queued && !inflight && (!more || act == 0)) {
      rc = QQ_NOT_CONVERGED;  // iteration limit reached (or nothing left that can move)
      break;
    }
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  {  // the final scalars: failure reasons of stopped right-hand sides
    QQ_CK(cudaMemcpy(hS, Sd, sbytes, cudaMemcpyDeviceToHost));
    const unsigned* hc = reinterpret_cast<const unsigned*>(hS + kScalDoubles);
    failed = hc[CTL_FAIL] & all;
    done = hc[CTL_DONE] & ~failed;
  }
  for (int k = 0; k < nb; ++k) {
    rhs[k]->done = (done >> k) & 1u;
    if ((failed >> k) & 1u) stats[k].fallback = (int)hS[(size_t)k * kScal + SC_FAIL];
    else if (!rhs[k]->done) stats[k].fallback = FAIL_MAXITER;
    stats[k].restarts = (int)hS[(size_t)k * kScal + SC_NRST];
  }
  return rc == QQ_OK && (done & all) == all ? QQ_OK : QQ_NOT_CONVERGED;
}

int batch_solve(qq_ctx* c, int nrhs, const double* be, const double* bo, const double kappa[2],
                const qq_method* meth, double* xe, double* xo, qq_solve_info* infos) {
  const int prec = prec_of_code(meth->precision);
  if (prec < 0) return set_error(QQ_BAD_ARG, "precision must be 64, 32, 16 or -16 (BF16)");
  if (meth->solver != 0 && meth->solver != 1) return set_error(QQ_BAD_ARG, "solver must be 0 or 1");
  if (meth->m < 2 || meth->k < 1 || meth->k >= meth->m || meth->m > 127)
    return set_error(QQ_BAD_ARG, "GMRES(m,k) out of range");
  if (!(meth->tol > 0.0)) return set_error(QQ_BAD_ARG, "tol must be > 0");
  const int block = std::max(1, std::min(meth->rhs_block, kMaxBatch));
  const size_t nv = c->ref_doubles();
  const double tk = 2.0 * kappa[0] * kappa[1];
  const double fac1 = 1.0 / (kappa[0] * kappa[0]);
  const double fac2 = 1.0 / (kappa[0] * (1.0 + tk * tk));
  // even-system tolerance: the full-lattice residual is checked at the end
  const double tol_even = meth->tol * 0.25;
  std::vector<std::unique_ptr<PerRhs>> R(nrhs);
  std::vector<SolveStats> stats(nrhs);
  std::vector<double> seconds(nrhs, 0.0);
  std::vector<int> status(nrhs, QQ_OK);
  Tmp fbe(c, P64), fbo(c, P64), h(c, P64);
  for (int i = 0; i < nrhs; ++i) {
    R[i].reset(new PerRhs());
    PerRhs& r = *R[i];
    QQ_TRY(ws_field(c, r.b, WS_RHS + 3 * i, P64));
    QQ_TRY(ws_field(c, r.x, WS_RHS + 3 * i + 1, P64));
    QQ_TRY(ws_field(c, r.r64, WS_RHS + 3 * i + 2, P64));
    QQ_TRY(zero_field(c, r.x.sp()));
    // fermprop source: b_e/kappa^2 + H_eo (1 - 2 i kappa mu gamma5) b_o / (kappa (1 + tk^2))
    const double* de = nullptr;
    const double* dO = nullptr;
    QQ_TRY(stage_in(c, 1, be + (size_t)i * nv, nv, &de));
    QQ_TRY(ref_to_field(c, de, 0, fbe.sp()));
    QQ_TRY(stage_in(c, 2, bo + (size_t)i * nv, nv, &dO));
    QQ_TRY(ref_to_field(c, dO, 1, fbo.sp()));
    QQ_CK(launch_spinmix(c->g.vh, fbo.sp(), Spinor{nullptr, nullptr, P64}, r.r64.sp(), 1.0, -tk, 0.0, 0.0, P64, c->st));
    QQ_TRY(op_hsingle(c, h.sp(), r.r64.sp(), 0, 0));
    QQ_TRY(lin(c, r.b.sp(), cimm(fac1), fbe.sp(), cimm(fac2), h.sp()));
  }
  cudaEvent_t e0, e1;
  QQ_CK(cudaEventCreate(&e0));
  QQ_CK(cudaEventCreate(&e1));
  auto tic = [&]() { cudaEventRecord(e0, c->st); };
  auto toc = [&]() {
    cudaEventRecord(e1, c->st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms * 1e-3;
  };
  int rc = QQ_OK;
  const int maxiter = meth->max_outer > 0 ? 1000 * meth->max_outer : default_maxiter(c->g, meth->tol);
  const int window = meth->stall_window > 0 ? meth->stall_window : kStallWindow;
  const int window16 = meth->stall_window > 0 ? meth->stall_window : kStallWindow16;
  if (meth->solver == 0) {
    for (int i = 0; i < nrhs && rc == QQ_OK; ++i) {
      tic();
      status[i] = gmresdr_fp64(c, R[i]->b.sp(), R[i]->x.sp(), meth->m, meth->k, tol_even, 0, kappa,
                               nullptr, &stats[i]);
      seconds[i] = toc();
      if (status[i] != QQ_OK && status[i] != QQ_NOT_CONVERGED) rc = status[i];
    }
  } else {
    DeflSpace defl;
    double defl_sec = 0.0;
    if (meth->deflate) {
      // deflation space from the first right-hand side; its partial solution is kept
      // as that right-hand side's initial guess
      tic();
      const double dt = meth->defl_tol > 0.0 ? meth->defl_tol : 1e-5;
      const int st0 = gmresdr_mixed(c, R[0]->b.sp(), R[0]->x.sp(), meth->m, meth->k, std::max(dt, tol_even),
                                    200, kappa, &defl, &stats[0]);
      defl_sec = toc();
      if (st0 != QQ_OK && st0 != QQ_NOT_CONVERGED) rc = st0;
    }
    for (int i0 = 0; i0 < nrhs && rc == QQ_OK; i0 += block) {
      const int nb = std::min(block, nrhs - i0);
      std::vector<PerRhs*> blk;
      std::vector<SolveStats> bst(nb);
      for (int k = 0; k < nb; ++k) blk.push_back(R[i0 + k].get());
      tic();
      int st = bicgstab_block(c, blk, prec, tol_even, 0.1, maxiter, prec == P16 || prec == PB16 ? window16 : window,
                              kappa, defl.k > 0 ? &defl : nullptr,
                              bst);
      // A 16-bit iteration that stopped short (near critical kappa it stalls at a true
      // residual of ~1e-2: 11 or 8 significant bits cannot resolve the low modes) is
      // continued by the batched FP32 BiCGStab from its FP64 solution, before any
      // right-hand side goes to FP64 GMRES-DR; fallback keeps the 16-bit reason.
      if ((prec == P16 || prec == PB16) && (st == QQ_OK || st == QQ_NOT_CONVERGED)) {
        std::vector<PerRhs*> again;
        std::vector<int> which;
        for (int k = 0; k < nb; ++k)
          if (!blk[k]->done) {
            again.push_back(blk[k]);
            which.push_back(k);
          }
        if (!again.empty()) {
          std::vector<SolveStats> bst32(again.size());
          st = bicgstab_block(c, again, P32, tol_even, 0.1, maxiter, window, kappa, defl.k > 0 ? &defl : nullptr,
                              bst32);
          for (size_t i = 0; i < again.size(); ++i) {
            SolveStats& b0 = bst[which[i]];
            const SolveStats& b1 = bst32[i];
            const int mvp0 = b0.mvp;
            b0.itercount += b1.itercount;
            b0.mvp += b1.mvp;
            b0.restarts += b1.restarts;
            b0.true_rel = b1.true_rel;
            for (size_t h = 0; h < b1.hist.size(); ++h) {
              b0.hist.push_back(b1.hist[h]);
              b0.hist_mvp.push_back(mvp0 + b1.hist_mvp[h]);
            }
            if (again[i]->done) b0.finished_by = 32;
          }
        }
      }
      const double sec = toc();
      // Every right-hand side the batched BiCGStab did not finish -- a breakdown (NaN,
      // vanishing rho or omega), a stall, or the iteration limit; bst[k].fallback holds
      // the reason -- goes to the reference method, plain FP64 GMRES-DR(m, k).  It
      // starts from the BiCGStab's FP64 solution when that is finite and better than
      // zero, with its relative tolerance rescaled so that it stops at the same
      // ||b - A x|| <= tol ||b||.  Finished right-hand sides keep their solutions; the
      // full-lattice residual below judges every one.
      std::vector<int> fb_status(nb, -1);
      std::vector<double> fb_sec(nb, 0.0);
      if (st == QQ_OK || st == QQ_NOT_CONVERGED) {
        for (int k = 0; k < nb && rc == QQ_OK; ++k) {
          if (blk[k]->done) continue;
          PerRhs& B = *blk[k];
          tic();
          double r0 = 0.0;
          QQ_TRY(op_dbletm(c, h.sp(), B.x.sp(), fbo.sp(), 0, kappa));
          QQ_TRY(lin(c, B.r64.sp(), cimm(1.0), B.b.sp(), cimm(-1.0), h.sp(), cimm(0),
                     Spinor{nullptr, nullptr, P64}, c->scal.as<double>()));
          QQ_TRY(read_scalars(c, c->scal.as<double>(), 1, &r0));
          r0 = std::sqrt(r0);
          double resmax = tol_even;
          if (std::isfinite(r0) && r0 > 0.0 && r0 < B.bn) {
            resmax = std::min(1.0, tol_even * B.bn / r0);
          } else {
            QQ_TRY(zero_field(c, B.x.sp()));
          }
          SolveStats fs;
          const int sf = gmresdr_fp64(c, B.b.sp(), B.x.sp(), meth->m, meth->k, resmax, 0, kappa, nullptr, &fs);
          fb_sec[k] = toc();
          if (sf != QQ_OK && sf != QQ_NOT_CONVERGED) rc = sf;
          fs.itercount += bst[k].itercount;
          fs.mvp += bst[k].mvp + 1;
          fs.fallback = bst[k].fallback != FAIL_NONE ? bst[k].fallback : FAIL_MAXITER;
          fs.finished_by = 64;
          fs.restarts = bst[k].restarts;
          bst[k] = fs;
          fb_status[k] = sf == QQ_OK ? QQ_OK : QQ_NOT_CONVERGED;
        }
        st = QQ_OK;
      }
      for (int k = 0; k < nb; ++k) {
        // the deflation-building solve is charged to the first right-hand side
        if (i0 + k == 0 && meth->deflate) {
          bst[k].itercount += stats[0].itercount;
          bst[k].mvp += stats[0].mvp;
          bst[k].ritz = stats[0].ritz;
        }
        stats[i0 + k] = bst[k];
        seconds[i0 + k] = sec / nb + fb_sec[k] + (i0 + k == 0 ? defl_sec : 0.0);
        status[i0 + k] = fb_status[k] >= 0 ? fb_status[k] : blk[k]->done ? QQ_OK : QQ_NOT_CONVERGED;
      }
      if (st != QQ_OK && st != QQ_NOT_CONVERGED) rc = st;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != QQ_OK) return rc;
  // odd reconstruction, full-lattice residual, output
  Tmp fxo(c, P64);
  for (int i = 0; i < nrhs; ++i) {
    PerRhs& r = *R[i];
    const double* de = nullptr;
    const double* dO = nullptr;
    QQ_TRY(stage_in(c, 1, be + (size_t)i * nv, nv, &de));
    QQ_TRY(ref_to_field(c, de, 0, fbe.sp()));
    QQ_TRY(stage_in(c, 2, bo + (size_t)i * nv, nv, &dO));
    QQ_TRY(ref_to_field(c, dO, 1, fbo.sp()));
    QQ_TRY(op_hsingle(c, h.sp(), r.x.sp(), 0, 1));
    const double f = 1.0 / (1.0 + tk * tk);
    QQ_CK(launch_spinmix(c->g.vh, fbo.sp(), h.sp(), fxo.sp(), f, -tk * f, f * kappa[0], -tk * f * kappa[0], P64, c->st));
    double rel = 0.0;
    QQ_TRY(full_residual(c, fbe.sp(), fbo.sp(), r.x.sp(), fxo.sp(), kappa, &rel));
    stats[i].true_rel = rel;
    if (rel > meth->tol && status[i] == QQ_OK) status[i] = QQ_NOT_CONVERGED;
    double* dxe = nullptr;
    double* dxo = nullptr;
    QQ_TRY(stage_out_begin(c, 1, xe + (size_t)i * nv, nv, &dxe));
    QQ_TRY(field_to_ref(c, r.x.sp(), 0, dxe));
    QQ_TRY(stage_out_end(c, 1, xe + (size_t)i * nv, nv, dxe));
    QQ_TRY(stage_out_begin(c, 2, xo + (size_t)i * nv, nv, &dxo));
    QQ_TRY(field_to_ref(c, fxo.sp(), 1, dxo));
    QQ_TRY(stage_out_end(c, 2, xo + (size_t)i * nv, nv, dxo));
    QQ_CK(cudaStreamSynchronize(c->st));
    if (infos) fill_info(&infos[i], status[i], stats[i], seconds[i]);
  }
  for (int i = 0; i < nrhs; ++i)
    if (status[i] != QQ_OK) return QQ_NOT_CONVERGED;
  return QQ_OK;
}

// Launch once every hopping shape a qq_fermprop_batch of nrhs sources with this method
// uses, so the autotuner makes its choices now and caches them in the context: the
// block operator (and its fused-dot form) at every block size the solve will form, and
// the FP64 single-field operators of the setup, the reliable updates and the fallback.
// The uneven batch runs this for each context on the calling thread before its worker
// threads start, so no candidate is timed while other contexts' solves share the GPU.
int tune_batch_shapes(qq_ctx* c, int nrhs, const double kappa[2], const qq_method* meth) {
  const int prec = prec_of_code(meth->precision);
  if (prec < 0 || nrhs < 1) return set_error(QQ_BAD_ARG, "bad method or nrhs");
  Tmp a64(c, P64), b64(c, P64), t64(c, P64);
  QQ_TRY(zero_field(c, a64.sp()));
  QQ_TRY(op_dbletm(c, b64.sp(), a64.sp(), t64.sp(), 0, kappa));
  QQ_TRY(op_hsingle(c, b64.sp(), a64.sp(), 0, 0));
  QQ_TRY(op_hsingle(c, b64.sp(), a64.sp(), 0, 1));
  if (meth->solver == 1) {
    const int block = std::max(1, std::min(meth->rhs_block, kMaxBatch));
    for (int nb : {std::min(block, nrhs), nrhs % block}) {
      if (nb < 1) continue;
      WsField in, out, tmp;
      WsField* const fs[3] = {&in, &out, &tmp};
      for (int i = 0; i < 3; ++i) {
        QQ_TRY(ws_field(c, *fs[i], WS_BLOCK + 2 * i, prec, nb));
        QQ_CK(cudaMemsetAsync(fs[i]->s.data, 0, fs[i]->bytes, c->st));
        if (has_norm(prec)) QQ_CK(cudaMemsetAsync(fs[i]->s.norm, 0, fs[i]->norm_bytes, c->st));
      }
      QQ_TRY(op_dbletm_block(c, out.sp(), in.sp(), tmp.sp(), nb, 0, kappa));
    }
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

// H (output parity pout) on nrhs reference-layout fields, computed at precision prec
// on one RHS-interleaved block field (a plain field for nrhs = 1) by kernel shape
// `shape` (0: the autotuned choice), returned in FP64 reference layout.
int hsingle_block(qq_ctx* c, int prec, int nrhs, int shape, double* gout, const double* gin, int idag,
                  int pout) {
  const int vh = c->g.vh;
  const size_t nv = c->ref_doubles();
  Field in, out;
  in.prec = out.prec = prec;
  QQ_CK(in.data.alloc(field_bytes(prec, vh) * nrhs));
  QQ_CK(out.data.alloc(field_bytes(prec, vh) * nrhs));
  if (has_norm(prec)) {
    QQ_CK(in.norm.alloc(sizeof(float) * vh * nrhs));
    QQ_CK(out.norm.alloc(sizeof(float) * vh * nrhs));
  }
  Tmp one(c, P64);
  for (int k = 0; k < nrhs; ++k) {
    const double* d = nullptr;
    QQ_TRY(stage_in(c, 1, gin + (size_t)k * nv, nv, &d));
    QQ_TRY(ref_to_field(c, d, 1 - pout, one.sp()));
    QQ_TRY(block_slot(c, prec, nrhs, k, in.sp(), one.sp(), 0));
  }
  HopArgs a;
  std::memset(&a, 0, sizeof(a));
  a.g = c->g;
  a.c = make_hopcoef(c->c1, c->c2, idag);
  a.pout = pout;
  a.gauge = c->gauge32.p;
  a.nrhs = nrhs;
  a.blk = nrhs > 1 ? 1 : 0;
  a.in[0] = in.data.p;
  a.in_norm[0] = in.norm.as<float>();
  a.out[0] = out.data.p;
  a.out_norm[0] = out.norm.as<float>();
  if (shape == 0) {
    QQ_TRY(launch_hop_tuned(c, a, prec, EPI_STORE));
  } else if (launch_hop(a, prec, 12, EPI_STORE, shape, c->st) != cudaSuccess) {
    cudaGetLastError();
    return set_error(QQ_BAD_ARG, "kernel shape not available for this precision and RHS count");
  }
  for (int k = 0; k < nrhs; ++k) {
    QQ_TRY(zero_field(c, one.sp()));
    QQ_TRY(block_slot(c, prec, nrhs, k, out.sp(), one.sp(), 1));
    double* d = nullptr;
    QQ_TRY(stage_out_begin(c, 2, gout + (size_t)k * nv, nv, &d));
    QQ_TRY(field_to_ref(c, one.sp(), pout, d));
    QQ_TRY(stage_out_end(c, 2, gout + (size_t)k * nv, nv, d));
    QQ_CK(cudaStreamSynchronize(c->st));
  }
  return QQ_OK;
}

}  // namespace qq
