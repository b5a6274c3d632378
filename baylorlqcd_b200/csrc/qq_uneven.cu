// Uneven batch: propagator solves on several lattices, gauge fields and kappa values in
// one call.  Each context (one lattice and its gauge field) keeps its own CUDA stream;
// the groups of one context run in the caller's order on one host thread, and the
// contexts run side by side, so the solves of a small lattice -- whose hop launches
// leave most of the 148 SMs idle -- overlap with those of the others on the GPU.
// Every group is exactly a qq_fermprop_batch call (same kernels, same graph-driven
// iteration); only the schedule differs.
#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include "qq_ctx.h"

namespace {

struct CtxWork {
  qq_ctx* ctx;
  std::vector<int> groups;  // indices into the caller's array, in its order
  int status = QQ_OK;
  std::string err;
};

int status_rank(int s) { return s == QQ_OK ? 0 : s == QQ_NOT_CONVERGED ? 1 : 2; }

void run_ctx(CtxWork& w, const qq_uneven_group* g, const qq_method* method) {
  for (int i : w.groups) {
    const qq_uneven_group& G = g[i];
    const int st = qq_fermprop_batch(G.ctx, G.nrhs, G.be, G.bo, G.kappa, method, G.xe, G.xo, G.infos);
    if (status_rank(st) > status_rank(w.status)) {
      w.status = st;
      if (st != QQ_NOT_CONVERGED) {
        w.err = "group " + std::to_string(i) + ": " + qq_last_error();
        return;  // a hard error stops this context's remaining groups
      }
    }
  }
}

}  // namespace

extern "C" int qq_fermprop_uneven(int ngroups, const qq_uneven_group* groups, const qq_method* method,
                                  int concurrent, double* seconds) {
  if (ngroups < 1 || !groups || !method) return qq::set_error(QQ_BAD_ARG, "bad arguments");
  std::vector<CtxWork> work;
  for (int i = 0; i < ngroups; ++i) {
    const qq_uneven_group& G = groups[i];
    if (!G.ctx || G.nrhs < 1 || !G.be || !G.bo || !G.xe || !G.xo)
      return qq::set_error(QQ_BAD_ARG, "group " + std::to_string(i) + ": null context, array or nrhs < 1");
    size_t w = 0;
    while (w < work.size() && work[w].ctx != G.ctx) ++w;
    if (w == work.size()) work.push_back(CtxWork{G.ctx, {}, QQ_OK, {}});
    work[w].groups.push_back(i);
  }
  const auto t0 = std::chrono::steady_clock::now();
  if (concurrent && work.size() > 1) {
    // every context's hop shapes are tuned here, one context at a time, so no autotuner
    // timing runs beside another context's solve (and the choice does not depend on the
    // schedule); the solves below then find every shape in their context's table
    for (int i = 0; i < ngroups; ++i) {
      const qq_uneven_group& G = groups[i];
      int st = cudaSetDevice(G.ctx->device) == cudaSuccess ? QQ_OK : QQ_CUDA_ERR;
      if (st == QQ_OK) st = qq::tune_batch_shapes(G.ctx, G.nrhs, G.kappa, method);
      if (st != QQ_OK) return qq::set_error(st, "group " + std::to_string(i) + ": " + qq_last_error());
    }
    std::vector<std::thread> th;
    th.reserve(work.size());
    for (auto& w : work) th.emplace_back(run_ctx, std::ref(w), groups, method);
    for (auto& t : th) t.join();
  } else {
    for (auto& w : work) run_ctx(w, groups, method);
  }
  const auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  int st = QQ_OK;
  std::string err;
  for (auto& w : work)
    if (status_rank(w.status) > status_rank(st)) {
      st = w.status;
      err = w.err;
    }
  if (st == QQ_OK) return QQ_OK;
  if (st == QQ_NOT_CONVERGED) return qq::set_error(st, "a solve stopped short of its tolerance");
  return qq::set_error(st, err);  // the worker's message, carried to the caller's thread
}
