// Operator application, level-1 helpers and reference-layout staging for the C ABI.
#include <algorithm>
#include <map>
#include <mutex>
#include <cmath>
#include <cstring>
#include <string>

#include "qq_ctx.h"

namespace qq {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

const char* last_error() { return g_last_error.c_str(); }

Tmp::Tmp(qq_ctx* c_, int prec_) : c(c_), prec(prec_), idx(-1), f(nullptr) {
  auto& pool = c->pool[prec];
  auto& busy = c->pool_busy[prec];
  for (size_t i = 0; i < pool.size(); ++i)
    if (!busy[i]) {
      idx = (int)i;
      break;
    }
  if (idx < 0) {
    pool.emplace_back(new Field());
    busy.push_back(false);
    idx = (int)pool.size() - 1;
    Field* nf = pool.back().get();
    nf->prec = prec;
    if (nf->data.alloc(field_bytes(prec, c->g.vh)) != cudaSuccess) {
      f = nullptr;
      return;
    }
    if (has_norm(prec)) nf->norm.alloc(sizeof(float) * c->g.vh);
  }
  busy[idx] = true;
  f = pool[idx].get();
}

Tmp::~Tmp() {
  if (idx >= 0) c->pool_busy[prec][idx] = false;
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int stage_in(qq_ctx* c, int slot, const double* p, size_t n, const double** dev) {
  if (!p) return set_error(QQ_BAD_ARG, "null array");
  if (is_device_ptr(p)) {
    *dev = p;
    return QQ_OK;
  }
  QQ_CK(c->stage[slot].alloc(n * sizeof(double)));
  QQ_CK(cudaMemcpyAsync(c->stage[slot].p, p, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
  *dev = c->stage[slot].as<double>();
  return QQ_OK;
}

int stage_out_begin(qq_ctx* c, int slot, double* p, size_t n, double** dev) {
  if (!p) return set_error(QQ_BAD_ARG, "null array");
  if (is_device_ptr(p)) {
    *dev = p;
    return QQ_OK;
  }
  QQ_CK(c->stage[slot].alloc(n * sizeof(double)));
  *dev = c->stage[slot].as<double>();
  return QQ_OK;
}

int stage_out_end(qq_ctx* c, int slot, double* p, size_t n, double* dev) {
  if (dev != p) QQ_CK(cudaMemcpyAsync(p, dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  (void)slot;
  return QQ_OK;
}

int ref_to_field(qq_ctx* c, const double* ref_dev, int parity, Spinor out) {
  QQ_CK(launch_spinor_from_ref(c->g, c->rd, parity, ref_dev, out, c->st));
  return QQ_OK;
}

int field_to_ref(qq_ctx* c, Spinor in, int parity, double* ref_dev) {
  QQ_CK(launch_ref_zero_halo(c->rd, ref_dev, c->st));
  QQ_CK(launch_spinor_to_ref(c->g, c->rd, parity, in, ref_dev, c->st));
  return QQ_OK;
}

static HopArgs hop_base(qq_ctx* c, int idag, int pout, int prec) {
  HopArgs a;
  std::memset(&a, 0, sizeof(a));
  a.g = c->g;
  a.c = make_hopcoef(c->c1, c->c2, idag);
  a.pout = pout;
  a.gauge = prec == P64 ? c->gauge64.p : c->gauge32.p;
  return a;
}

static int recon_of(qq_ctx* c, int prec) { return prec == P64 ? c->recon64 : 12; }

// Launch the hopping kernel with the number of direction groups (threads per site)
// that ran fastest for this (precision, links, RHS count, epilogue) on this lattice.
// The first launch of a shape times each candidate on the real operands (the kernel
// is idempotent: inputs are never outputs) and caches the winner in the context.
// Algorithmic bytes of one hop launch: every link once, every input and output spinor
// once, and the epilogue's extra input for EPI_DBLE.
static double hop_bytes(qq_ctx* c, int prec, int nrhs, int epi) {
  const int recon = recon_of(c, prec);
  const double link = prec == P64 ? (recon == 18 ? 144.0 : 96.0) : 48.0;
  const double spin = prec == P64 ? 192.0 : prec == P32 ? 96.0 : 52.0;
  return (double)c->g.vh * (8.0 * link + nrhs * (epi == EPI_DBLE ? 3.0 : 2.0) * spin);
}

static int launch_hop_profiled(qq_ctx* c, const HopArgs& a, int prec, int recon, int epi, int tps) {
  if (!c->prof_hop) {
    QQ_CK(launch_hop(a, prec, recon, epi, tps, c->st));
    return QQ_OK;
  }
  if (c->prof_used == c->prof_events.size()) {
    cudaEvent_t e0, e1;
    QQ_CK(cudaEventCreate(&e0));
    QQ_CK(cudaEventCreate(&e1));
    c->prof_events.emplace_back(e0, e1);
    c->prof_bytes.push_back(0.0);
    c->prof_shape.push_back(0);
  }
  auto& ev = c->prof_events[c->prof_used];
  c->prof_bytes[c->prof_used] = hop_bytes(c, prec, a.nrhs, epi);
  c->prof_shape[c->prof_used] = prec * 1000 + a.nrhs;
  ++c->prof_used;
  QQ_CK(cudaEventRecord(ev.first, c->st));
  QQ_CK(launch_hop(a, prec, recon, epi, tps, c->st));
  QQ_CK(cudaEventRecord(ev.second, c->st));
  return QQ_OK;
}

// The autotuner's L2 flush buffer: one per device, shared by every context on it and
// kept until the process exits, so a context's first tuning allocates nothing (and does
// not synchronise the device under other contexts' solves) once any context has tuned.
static cudaError_t tune_flush_buffer(void** p, size_t* bytes) {
  static std::mutex mu;
  static std::map<int, void*> bufs;
  constexpr size_t kBytes = (size_t)256 << 20;  // twice the L2
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  void*& b = bufs[dev];
  if (!b) {
    e = cudaMalloc(&b, kBytes);
    if (e != cudaSuccess) {
      b = nullptr;
      return e;
    }
  }
  *p = b;
  *bytes = kBytes;
  return cudaSuccess;
}

int hop_tune_key(qq_ctx* c, const HopArgs& a, int prec, int epi) {
  return (((prec * 64 + recon_of(c, prec)) * 64 + a.nrhs) * 4 + epi) * 2 + a.blk;
}

int launch_hop_tuned(qq_ctx* c, const HopArgs& a, int prec, int epi) {
  const int recon = recon_of(c, prec);
  const int key = hop_tune_key(c, a, prec, epi);
  auto it = c->hop_tune.find(key);
  if (it != c->hop_tune.end()) return launch_hop_profiled(c, a, prec, recon, epi, it->second);
  if (c->forced_tps > 0) {  // a forced shape (tests) where this launch supports it
    if (launch_hop(a, prec, recon, epi, c->forced_tps, c->st) == cudaSuccess) {
      c->hop_tune[key] = c->forced_tps;
      return QQ_OK;
    }
    cudaGetLastError();
  }
  // Candidates are timed as the solvers run them, with operands streamed from HBM: a
  // 256 MiB buffer (twice the L2) is overwritten before every timed launch.  Each
  // candidate is timed three times and its median kept, so the choice is stable.
  void* flush = nullptr;
  size_t flush_bytes = 0;
  QQ_CK(tune_flush_buffer(&flush, &flush_bytes));
  int best = 1;
  float best_ms = 1e30f;
  for (int tps : {1, 2, 32, 64, 96, 128, kShapeMrhs + 2, kShapeMrhs + 3, kShapeMrhs + 4, kShapeF2 + 1,
                  kShapeF2 + 2, kShapeF2 + 3, kShapeF2 + 4, kShapeF2 + 5, kShapeF2 + 6, kShapeF2 + 7,
                  kShapeF2 + 8, kShapeF2 + 9, kShapeF2 + 10, kShapeF2 + 11}) {
    const int per = tps <= 4 ? 128 / tps : tps;
    if (a.nrhs > per) continue;
    if (tps >= kShapeF2 + 6) {  // copy ring, every variant (its shared memory pays off from 4 RHS up)
      if (prec != P32 || a.nrhs < 4) continue;
    } else if (tps == kShapeF2 + 5) {  // + links staged in shared memory (block fields, nrhs >= 8)
      if (prec != P32 || !a.blk || a.nrhs < 8) continue;
    } else if (tps == kShapeF2 + 4) {  // pipelined packed kernel, one RHS per thread
      if (prec != P32) continue;
    } else if (tps > kShapeF2) {
      const int rpt = tps - kShapeF2;
      if (prec != P32 || a.nrhs % rpt != 0 || (rpt > 1 && !a.blk)) continue;
    } else if (tps > kShapeMrhs && (!a.blk || prec == P64 || a.nrhs % (tps - kShapeMrhs) != 0)) {
      continue;
    }
    if (launch_hop(a, prec, recon, epi, tps, c->st) != cudaSuccess) {  // warm-up
      cudaGetLastError();  // shape not launchable (shared memory): skip it
      continue;
    }
    float t[3];
    for (int rep = 0; rep < 3; ++rep) {
      QQ_CK(cudaMemsetAsync(flush, rep + 1, flush_bytes, c->st));
      QQ_CK(cudaEventRecord(c->tev0, c->st));
      QQ_CK(launch_hop(a, prec, recon, epi, tps, c->st));
      QQ_CK(cudaEventRecord(c->tev1, c->st));
      QQ_CK(cudaEventSynchronize(c->tev1));
      QQ_CK(cudaEventElapsedTime(&t[rep], c->tev0, c->tev1));
    }
    std::sort(t, t + 3);
    const float ms = t[1];
    if (ms < best_ms) {
      best_ms = ms;
      best = tps;
    }
  }
  c->hop_tune[key] = best;
  return launch_hop_profiled(c, a, prec, recon, epi, best);
}

int op_hsingle_multi(qq_ctx* c, const Spinor* out, const Spinor* in, int n, int idag, int pout) {
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  const int prec = in[0].prec;
  for (int r0 = 0; r0 < n; r0 += kMaxRhs) {
    const int nb = std::min(kMaxRhs, n - r0);
    HopArgs a = hop_base(c, idag, pout, prec);
    a.nrhs = nb;
    for (int r = 0; r < nb; ++r) {
      a.in[r] = in[r0 + r].data;
      a.in_norm[r] = in[r0 + r].norm;
      a.out[r] = out[r0 + r].data;
      a.out_norm[r] = out[r0 + r].norm;
    }
    QQ_TRY(launch_hop_tuned(c, a, prec, EPI_STORE));
  }
  return QQ_OK;
}

int op_hsingle(qq_ctx* c, Spinor out, Spinor in, int idag, int pout) {
  return op_hsingle_multi(c, &out, &in, 1, idag, pout);
}

int op_dbletm_multi(qq_ctx* c, const Spinor* out, const Spinor* in, const Spinor* tmp, int n,
                    int idag, const double kappa[2]) {
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  const int prec = in[0].prec;
  const bool wilson = kappa[1] < 0.00000001;  // Q/diracops.f90:467
  for (int r0 = 0; r0 < n; r0 += kMaxRhs) {
    const int nb = std::min(kMaxRhs, n - r0);
    HopArgs a = hop_base(c, idag, 1, prec);
    a.nrhs = nb;
    for (int r = 0; r < nb; ++r) {
      a.in[r] = in[r0 + r].data;
      a.in_norm[r] = in[r0 + r].norm;
      a.out[r] = tmp[r0 + r].data;
      a.out_norm[r] = tmp[r0 + r].norm;
    }
    a.a = 2.0 * kappa[0] * kappa[1];
    QQ_TRY(launch_hop_tuned(c, a, prec, wilson ? EPI_STORE : EPI_TWIST));
    HopArgs b = hop_base(c, idag, 0, prec);
    b.nrhs = nb;
    for (int r = 0; r < nb; ++r) {
      b.in[r] = tmp[r0 + r].data;
      b.in_norm[r] = tmp[r0 + r].norm;
      b.out[r] = out[r0 + r].data;
      b.out_norm[r] = out[r0 + r].norm;
      b.aux[r] = in[r0 + r].data;
      b.aux_norm[r] = in[r0 + r].norm;
    }
    b.f1 = 1.0 / (kappa[0] * kappa[0]);
    if (wilson) {
      b.f2 = 0.0;
      b.f3 = 1.0;
    } else {
      const double t = 2.0 * kappa[0] * kappa[1];
      b.f2 = 2.0 * kappa[1] / kappa[0];
      b.f3 = 1.0 / (1.0 + t * t);
    }
    QQ_TRY(launch_hop_tuned(c, b, prec, EPI_DBLE));
  }
  return QQ_OK;
}

// Thread blocks of the copy-ring hop kernel for block fields of nb right-hand sides
// (the partials a fused dot product writes per right-hand side).
int hop_block_count(qq_ctx* c, int nb) {
  const int per = hop_sites_per_block(1, nb);
  return (c->g.vh + per - 1) / per;
}

// Hdbletm on block fields with, when the autotuned second launch is the FP32 copy-ring
// kernel, a dot product of the output fused into its epilogue (HopArgs::dot_mode):
// *fused_blocks = the number of per-block partials written to dot_part, 0 when the
// caller must compute the dot product itself.
int op_dbletm_block_dot(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int nb, const double kappa[2],
                        Spinor dot_op, double* dot_part, int dot_mode, int* fused_blocks) {
  *fused_blocks = 0;
  return op_dbletm_block_impl(c, out, in, tmp, nb, 0, kappa, dot_op, dot_part, dot_mode, fused_blocks);
}

// Hdbletm on RHS-interleaved block fields of nb right-hand sides (one launch pair).
int op_dbletm_block(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int nb, int idag,
                    const double kappa[2]) {
  return op_dbletm_block_impl(c, out, in, tmp, nb, idag, kappa, Spinor{nullptr, nullptr, in.prec}, nullptr, 0,
                              nullptr);
}

int op_dbletm_block_impl(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int nb, int idag, const double kappa[2],
                         Spinor dot_op, double* dot_part, int dot_mode, int* fused_blocks) {
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  if (nb < 1 || nb > 32) return set_error(QQ_BAD_ARG, "block of 1..32 right-hand sides");
  const int prec = in.prec;
  const bool wilson = kappa[1] < 0.00000001;  // Q/diracops.f90:467
  HopArgs a = hop_base(c, idag, 1, prec);
  a.nrhs = nb;
  a.blk = 1;
  a.in[0] = in.data;
  a.in_norm[0] = in.norm;
  a.out[0] = tmp.data;
  a.out_norm[0] = tmp.norm;
  a.a = 2.0 * kappa[0] * kappa[1];
  QQ_TRY(launch_hop_tuned(c, a, prec, wilson ? EPI_STORE : EPI_TWIST));
  HopArgs b = hop_base(c, idag, 0, prec);
  b.nrhs = nb;
  b.blk = 1;
  b.in[0] = tmp.data;
  b.in_norm[0] = tmp.norm;
  b.out[0] = out.data;
  b.out_norm[0] = out.norm;
  b.aux[0] = in.data;
  b.aux_norm[0] = in.norm;
  b.f1 = 1.0 / (kappa[0] * kappa[0]);
  if (wilson) {
    b.f2 = 0.0;
    b.f3 = 1.0;
  } else {
    const double t = 2.0 * kappa[0] * kappa[1];
    b.f2 = 2.0 * kappa[1] / kappa[0];
    b.f3 = 1.0 / (1.0 + t * t);
  }
  if (dot_mode && prec == P32 && fused_blocks) {
    // the fusion depends on the tuned shape: tune first (that launch's output is
    // recomputed below), so the first call of a solve is fused like every later one
    const int key = hop_tune_key(c, b, prec, EPI_DBLE);
    if (c->hop_tune.find(key) == c->hop_tune.end()) QQ_TRY(launch_hop_tuned(c, b, prec, EPI_DBLE));
    auto it = c->hop_tune.find(key);
    if (it != c->hop_tune.end() && it->second >= kShapeF2 + 6 && it->second <= kShapeF2 + 11) {
      b.dot_op = dot_op.data;
      b.dot_part = dot_part;
      b.dot_mode = dot_mode;
      *fused_blocks = hop_block_count(c, nb);
    }
  }
  return launch_hop_tuned(c, b, prec, EPI_DBLE);
}

// gamma5mult (Q/diracops.f90:1750-1860) minus a real shift:
//   out = -i gamma5 [ (1 + 2 i kappa mu gamma5)/kappa^2
//                     - H_eo (1 - 2 i kappa mu gamma5) H_oe / (1 + 4 kappa^2 mu^2) ] in / (2 kappa mu)
//         - sigma in.
// The bracket is Hdbletm's twisted form for every mu /= 0 (Hdbletm itself switches to
// Hdouble below mu = 1e-8, gamma5mult does not).  -i gamma5 takes the spins
// (v0, v1, v2, v3) to (-v2, -v3, v0, v1), which is -J of the spin-mixing kernel.
int op_g5mult(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int idag, const double kappa[2],
              double sigma) {
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  const double t = 2.0 * kappa[0] * kappa[1];
  if (!(t != 0.0) || !std::isfinite(1.0 / t)) return set_error(QQ_BAD_ARG, "gamma5mult needs kappa*mu /= 0");
  const int prec = in.prec;
  HopArgs a = hop_base(c, idag, 1, prec);
  a.nrhs = 1;
  a.in[0] = in.data;
  a.in_norm[0] = in.norm;
  a.out[0] = tmp.data;
  a.out_norm[0] = tmp.norm;
  a.a = t;
  QQ_TRY(launch_hop_tuned(c, a, prec, EPI_TWIST));
  HopArgs b = hop_base(c, idag, 0, prec);
  b.nrhs = 1;
  b.in[0] = tmp.data;
  b.in_norm[0] = tmp.norm;
  b.out[0] = out.data;
  b.out_norm[0] = out.norm;
  b.aux[0] = in.data;
  b.aux_norm[0] = in.norm;
  b.f1 = 1.0 / (kappa[0] * kappa[0]);
  b.f2 = 2.0 * kappa[1] / kappa[0];
  b.f3 = 1.0 / (1.0 + t * t);
  QQ_TRY(launch_hop_tuned(c, b, prec, EPI_DBLE));
  QQ_CK(launch_spinmix(c->g.vh, in, out, out, -sigma, 0.0, 0.0, -1.0 / t, prec, c->st));
  return QQ_OK;
}

int op_dbletm(qq_ctx* c, Spinor out, Spinor in, Spinor tmp, int idag, const double kappa[2]) {
  return op_dbletm_multi(c, &out, &in, &tmp, 1, idag, kappa);
}

int lin(qq_ctx* c, Spinor out, Coef a, Spinor x, Coef b, Spinor y, Coef cc, Spinor z,
        double* nrm2_dev) {
  LinArgs L;
  std::memset(&L, 0, sizeof(L));
  L.vh = c->g.vh;
  L.x = x;
  L.y = y;
  L.z = z;
  L.out = out;
  L.a = a;
  L.b = b;
  L.c = cc;
  L.red = nrm2_dev ? 1 : 0;
  L.partial = c->partial.as<double>();
  QQ_CK(launch_lincomb(L, x.prec, y.prec, z.prec, out.prec, c->st));
  if (nrm2_dev) QQ_CK(launch_finalize(L.partial, kRedBlocks, 3, 1, nrm2_dev, 0, c->st));
  return QQ_OK;
}

int dot_dev(qq_ctx* c, Spinor x, Spinor y, double* out3) {
  QQ_CK(launch_dot(c->g.vh, x, y, c->partial.as<double>(), c->st));
  QQ_CK(launch_finalize(c->partial.as<double>(), kRedBlocks, 3, 3, out3, 0, c->st));
  return QQ_OK;
}

int read_scalars(qq_ctx* c, const double* dev, int n, double* host) {
  QQ_CK(cudaMemcpyAsync(c->hpin, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  std::memcpy(host, c->hpin, sizeof(double) * n);
  return QQ_OK;
}

int dot_host(qq_ctx* c, Spinor x, Spinor y, std::complex<double>* d, double* ynrm2) {
  double* s = c->scal.as<double>();
  QQ_TRY(dot_dev(c, x, y, s));
  double h[3];
  QQ_TRY(read_scalars(c, s, 3, h));
  if (d) *d = {h[0], h[1]};
  if (ynrm2) *ynrm2 = h[2];
  return QQ_OK;
}

int norm2_host(qq_ctx* c, Spinor x, double* n2) { return dot_host(c, x, x, nullptr, n2); }

int copy_field(qq_ctx* c, Spinor out, Spinor in) { return lin(c, out, cimm(1.0), in); }

int zero_field(qq_ctx* c, Spinor f) {
  QQ_CK(cudaMemsetAsync(f.data, 0, field_bytes(f.prec, c->g.vh), c->st));
  if (has_norm(f.prec) && f.norm) QQ_CK(cudaMemsetAsync(f.norm, 0, sizeof(float) * c->g.vh, c->st));
  return QQ_OK;
}

void fill_info(qq_solve_info* info, int status, const SolveStats& s, double seconds) {
  if (!info) return;
  std::memset(info, 0, sizeof(*info));
  info->status = status;
  info->itercount = s.itercount;
  info->mvp = s.mvp;
  info->ncycles = s.ncycles;
  info->true_rel = s.true_rel;
  info->seconds = seconds;
  info->fallback = s.fallback;
  info->finished_by = s.finished_by;
  info->restarts = s.restarts;
  info->nhist = (int)std::min<size_t>(s.hist.size(), 1024);
  for (int i = 0; i < info->nhist; ++i) {
    info->hist[i] = s.hist[i];
    info->hist_mvp[i] = s.hist_mvp[i];
  }
  info->nritz = (int)std::min<size_t>(s.ritz.size(), 512);
  for (int i = 0; i < info->nritz; ++i) {
    info->ritz[2 * i] = s.ritz[i].real();
    info->ritz[2 * i + 1] = s.ritz[i].imag();
  }
}

}  // namespace qq
