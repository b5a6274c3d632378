// Eigenmodes of the Wilson operator M = 1 - kappa D and the eigenmode-subtracted loop
// estimators of the reference's Wilson loop driver (testFUNC, Q/disconloops.f90:1980-2569).
//
//   qq_eigmodes, kind 1   eigmodesofM (:1593-1937).  Ritz pairs of the even-odd operator
//       Mhat = Hdbletm (Hdouble for Wilson) from gmresdrEIGBS (Q/working.f90:48-907), a
//       GMRES-DR whose restart keeps the k harmonic Ritz vectors with the smallest
//       |theta| plus the common direction of their residuals, run a fixed number of
//       cycles from the unit source b(1,1,1,1,1) = 1.  Pairs theta, conj(theta) (to 1e-8)
//       are lifted to M: lambda = 1 - sqrt(1 - kappa^2 theta), odd half
//       kappa H_oe R_e / sqrt(1 - kappa^2 theta); the left vector of each mode is gamma5
//       times its partner's right vector, R is scaled so that <R, L> = 1; modes with
//       ||M R - lambda R|| < 1e-8 are kept, sorted by |lambda|.
//   qq_eigmodes, kind 2   eigmodesofMprime (:2573-2875).  Ritz pairs of the Hermitian
//       M gamma5 on the full lattice from gmresdr5EIG (Q/inverters.f90:1435-2070: the
//       restart keeps the least-squares residual instead, and zeroes the columns of the
//       new projected matrix below converged Ritz values), from the caller's start vector
//       (the reference draws a Z(4) noise); unit-norm modes with
//       ||M gamma5 R - Re(theta) R|| < 1e-5 are kept, sorted by |Re theta|; L = R.
//   qq_xigenerator        xigenerator (:465-838): xi(isub, j) = <L_j, S_isub R_j> with
//       S_1 = 0 and S_isub = sum_{n=0}^{isub+1} kappa^n H^n (gamma5 S for kind 2).
//   qq_eigaverage         eigaverage (:3239-3342): the loop operators of the cumulative
//       correction x'_j = sum_{i<=j} R_i s_i <L_i, z> (loopops; for kind 2
//       eigloopops_original :7919-8038, which is loopops of gamma5 x').  The operators are
//       linear in x', so each mode's trace T_i is evaluated once and the corrections are
//       prefix sums of s_i <L_i, z> T_i.
//   qq_generalaverage     generalaverage (:119-333), estimator styles 1-6 at imom = 1.
//
// The Krylov basis lives in HBM (FP64, GPU layout; a full-lattice vector is the even
// half followed by the odd half) and may hold up to 255 vectors: the multi-vector
// kernels run in chunks of 128 vectors, and the restart rotation is an out-of-place
// combination into a second basis.  The small dense problems (least squares, the
// harmonic eigenproblem, the QR of the restart matrix) run on the host in FP64.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "qq_ctx.h"

struct qq_eig {
  qq_ctx* ctx = nullptr;
  int kind = 0;
  int num = 0;
  std::vector<std::complex<double>> lam;  // eigenvalue of each kept mode (kind 2: real)
  qq::DevBuf R, L;                         // num full vectors each (kind 2: L unused, L = R)
  size_t half_nel = 0;                     // 12 vh elements of 16 bytes per half
  int cycles = 0, mvp = 0, nritz = 0;
  std::vector<std::complex<double>> ritz;  // Ritz values of the last cycle (k of them)
  void* r(int j) const { return static_cast<char*>(R.p) + (size_t)j * 2 * half_nel * 16; }
  void* l(int j) const { return kind == 2 ? r(j) : static_cast<char*>(L.p) + (size_t)j * 2 * half_nel * 16; }
};

namespace qq {

int loop_slices(qq_ctx* c, const double* ye, const double* yo, const double* be, const double* bo, int ksub,
                double* val, double* Jdev, double* J_host);

namespace {

using cd = std::complex<double>;
constexpr int kMaxEigBasis = 255;   // m + 1 <= 256
constexpr int kChunk = 128;         // vectors per multi-vector launch
constexpr int kCombineOut = 16;     // outputs per combine launch
constexpr double kPairTol = 1e-8;   // eigtol, Q/disconloops.f90:1638
constexpr double kResTolM = 1e-8;   // eigtoltemp, :1639
constexpr double kResTolMp = 1e-5;  // :2812
constexpr int kWsVal = 4096, kWsJ = 4097, kWsRef = 4098;  // context workspace ids

// out = gamma5 in on `nhalf` half fields (FP64, component-major: element q vh + s,
// q = 3 spin + colour); gamma5 = [[0, -i], [i, 0]] in 2 x 2 spin blocks.
__global__ void g5_kernel(int vh, int nhalf, const double2* in, double2* out) {
  const size_t n = (size_t)vh * 3 * nhalf;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const size_t h = t / ((size_t)3 * vh), r = t % ((size_t)3 * vh);
    const size_t base = h * 12 * (size_t)vh + r;  // spin 0, colour r / vh, site r % vh
    const double2 v0 = in[base], v1 = in[base + 3 * (size_t)vh], v2 = in[base + 6 * (size_t)vh],
                  v3 = in[base + 9 * (size_t)vh];
    out[base] = make_double2(v2.y, -v2.x);                   // -i v2
    out[base + 3 * (size_t)vh] = make_double2(v3.y, -v3.x);  // -i v3
    out[base + 6 * (size_t)vh] = make_double2(-v0.y, v0.x);  //  i v0
    out[base + 9 * (size_t)vh] = make_double2(-v1.y, v1.x);  //  i v1
  }
}

// W_j = sum_{i < nin} V_i Z(i, j0 + j) for j < nout (<= kCombineOut), out of place.
__global__ void __launch_bounds__(256) combine_kernel(const double2* V, size_t stride, size_t nel, int nin,
                                                      const double* Z, int ldz, int j0, int nout, double2* W) {
  __shared__ double2 zs[64][kCombineOut];
  const size_t e0 = (size_t)blockIdx.x * blockDim.x;
  for (size_t eb = e0; eb < nel; eb += (size_t)gridDim.x * blockDim.x) {  // block-uniform trip count
    const size_t e = eb + threadIdx.x;
    double2 acc[kCombineOut];
#pragma unroll
    for (int j = 0; j < kCombineOut; ++j) acc[j] = make_double2(0.0, 0.0);
    for (int i0 = 0; i0 < nin; i0 += 64) {
      const int ni = min(64, nin - i0);
      __syncthreads();
      for (int t = threadIdx.x; t < 64 * kCombineOut; t += blockDim.x) {
        const int i = t / kCombineOut, j = t % kCombineOut;
        if (i < ni && j < nout) {
          const size_t zi = 2 * ((size_t)(i0 + i) + (size_t)ldz * (j0 + j));
          zs[i][j] = make_double2(Z[zi], Z[zi + 1]);
        } else {
          zs[i][j] = make_double2(0.0, 0.0);
        }
      }
      __syncthreads();
      if (e < nel) {
        for (int i = 0; i < ni; ++i) {
          const double2 v = V[(size_t)(i0 + i) * stride + e];
#pragma unroll
          for (int j = 0; j < kCombineOut; ++j) {
            const double2 z = zs[i][j];
            acc[j].x += z.x * v.x - z.y * v.y;
            acc[j].y += z.x * v.y + z.y * v.x;
          }
        }
      }
    }
    if (e < nel)
#pragma unroll
      for (int j = 0; j < kCombineOut; ++j)
        if (j < nout) W[(size_t)j * stride + e] = acc[j];
  }
}

// A basis of up to kMaxEigBasis FP64 vectors of nel 16-byte elements.
struct Basis {
  DevBuf buf;
  size_t nel = 0;
  int cap = 0;
  int init(size_t nel_, int cap_) {
    nel = nel_;
    cap = cap_;
    QQ_CK(buf.alloc((size_t)cap * nel * 16));
    return QQ_OK;
  }
  void* v(int i) const { return static_cast<char*>(buf.p) + (size_t)i * nel * 16; }
  BasisArgs args(int i0) const { return BasisArgs{v(i0), nel, nel}; }
};

struct Scratch {
  DevBuf h1, h2, nrm, Z;  // dot columns, |w|^2, combine matrix
  int init(int m, int ncols) {
    QQ_CK(h1.alloc(sizeof(double) * 2 * (m + 2)));
    QQ_CK(h2.alloc(sizeof(double) * 2 * (m + 2)));
    QQ_CK(nrm.alloc(sizeof(double) * 4));
    QQ_CK(Z.alloc(sizeof(double) * 2 * (size_t)(m + 1) * ncols));
    return QQ_OK;
  }
};

// h = V[0..n)^H w on the device (h1), chunked.
int mdot(qq_ctx* c, const Basis& B, int n, const void* w, double* h) {
  double* part = c->partial.as<double>();
  for (int c0 = 0; c0 < n; c0 += kChunk) {
    const int nb = std::min(kChunk, n - c0);
    int ng = 0;
    QQ_CK(launch_multidot(P64, B.args(c0), nb, w, part, &ng, c->st));
    QQ_CK(launch_finalize(part, kRedBlocks, ng * 16, 2 * nb, h + 2 * c0, 0, c->st));
  }
  return QQ_OK;
}

// w -= V[0..n) h (h on the device); the partials of the last chunk hold |w|^2.
int maxpy(qq_ctx* c, const Basis& B, int n, const double* h, void* w) {
  double* part = c->partial.as<double>();
  for (int c0 = 0; c0 < n; c0 += kChunk) {
    const int nb = std::min(kChunk, n - c0);
    QQ_CK(launch_multiaxpy(P64, B.args(c0), nb, h + 2 * c0, 1.0, w, w, part, c->st));
  }
  return QQ_OK;
}

// W[0..nout) = V[0..nin) Z, Z host (nin x nout, column-major) uploaded to S.Z.
int combine(qq_ctx* c, const Basis& V, int nin, const dense::Mat& Z, int nout, Scratch& S, Basis& W, int w0 = 0) {
  std::vector<double> h(2 * (size_t)nin * nout);
  for (int j = 0; j < nout; ++j)
    for (int i = 0; i < nin; ++i) {
      h[2 * ((size_t)i + (size_t)nin * j)] = Z(i, j).real();
      h[2 * ((size_t)i + (size_t)nin * j) + 1] = Z(i, j).imag();
    }
  QQ_CK(S.Z.alloc(sizeof(double) * h.size()));
  QQ_CK(cudaMemcpyAsync(S.Z.p, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->st));
  for (int j0 = 0; j0 < nout; j0 += kCombineOut) {
    count_launch();
    combine_kernel<<<4 * 148, 256, 0, c->st>>>(static_cast<const double2*>(V.v(0)), V.nel, V.nel, nin,
                                                S.Z.as<double>(), nin, j0, std::min(kCombineOut, nout - j0),
                                                static_cast<double2*>(W.v(w0 + j0)));
    QQ_CK(cudaGetLastError());
  }
  QQ_CK(cudaStreamSynchronize(c->st));  // h goes out of scope
  return QQ_OK;
}

int g5(qq_ctx* c, const void* in, void* out, int nhalf) {
  count_launch();
  g5_kernel<<<4 * 148, 256, 0, c->st>>>(c->g.vh, nhalf, static_cast<const double2*>(in),
                                        static_cast<double2*>(out));
  QQ_CK(cudaGetLastError());
  return QQ_OK;
}

Spinor half_of(void* full, size_t half_nel, int parity) {
  return Spinor{static_cast<char*>(full) + (size_t)parity * half_nel * 16, nullptr, P64};
}

// The Krylov operator: kind 1 Hdbletm on the even half; kind 2 M gamma5 on the full
// lattice, (M y)_e = y_e - kappa H_eo y_o, (M y)_o = y_o - kappa H_oe y_e.
struct EigOp {
  qq_ctx* c;
  int kind;
  double kappa[2];
  size_t hn;  // half elements
  DevBuf tfull;
  int apply(void* out, const void* in) {
    if (kind == 1) {
      Tmp t(c, P64);
      return op_dbletm(c, Spinor{out, nullptr, P64}, Spinor{const_cast<void*>(in), nullptr, P64}, t.sp(), 0,
                       kappa);
    }
    if (!tfull.p) QQ_CK(tfull.alloc(2 * hn * 16));
    QQ_TRY(g5(c, in, tfull.p, 2));
    const Spinor te = half_of(tfull.p, hn, 0), to = half_of(tfull.p, hn, 1);
    const Spinor oe = half_of(out, hn, 0), oo = half_of(out, hn, 1);
    QQ_TRY(op_hsingle(c, oo, te, 0, 1));
    QQ_TRY(lin(c, oo, cimm(1.0), to, cimm(-kappa[0]), oo));
    QQ_TRY(op_hsingle(c, oe, to, 0, 0));
    QQ_TRY(lin(c, oe, cimm(1.0), te, cimm(-kappa[0]), oe));
    return QQ_OK;
  }
};

// Stable ascending order of keys (the reference's exchange sort, basics.f90:81-115).
std::vector<int> stable_order(const std::vector<double>& key) {
  std::vector<int> o(key.size());
  for (size_t i = 0; i < o.size(); ++i) o[i] = (int)i;
  std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return key[a] < key[b]; });
  return o;
}

// Complex square root, principal branch (Numerical Recipes' csqrt; basics.f90:286-343).
cd nr_sqrt(cd z) {
  const double a = z.real(), b = z.imag();
  if (a == 0.0 && b == 0.0) return cd(0.0, 0.0);
  double w;
  if (std::fabs(a) >= std::fabs(b)) {
    const double t = b / a;
    w = std::sqrt(std::fabs(a)) * std::sqrt((1.0 + std::sqrt(1.0 + t * t)) / 2.0);
  } else {
    const double t = a / b;
    w = std::sqrt(std::fabs(b)) * std::sqrt((std::fabs(t) + std::sqrt(1.0 + t * t)) / 2.0);
  }
  if (a >= 0.0) return cd(w, b / (2.0 * w));
  if (b >= 0.0) return cd(std::fabs(b) / (2.0 * w), w);
  return cd(std::fabs(b) / (2.0 * w), -w);
}

// 1 / z by Smith's method (basics.f90:48-77).
cd nr_inv(cd z) {
  const double a = z.real(), b = z.imag();
  if (std::fabs(a) >= std::fabs(b)) {
    const double t = b / a, d = t * b + a;
    return cd(1.0 / d, -t / d);
  }
  const double t = a / b, d = t * a + b;
  return cd(t / d, -1.0 / d);
}

// The deflated-restart eigen-iteration shared by gmresdrEIGBS (variant 1) and
// gmresdr5EIG (variant 2).  On return evec holds the k Ritz vectors of the last cycle
// (V_m times the harmonic Ritz eigenvectors, ordered by increasing Ritz residual) and
// eval their harmonic Ritz values.
int eig_gmresdr(qq_ctx* c, EigOp& op, int variant, const void* b, int m, int k, int ncycles, Basis& evec,
                std::vector<cd>& eval, int* cycles_done, int* mvp) {
  const size_t nel = (op.kind == 1 ? 1 : 2) * op.hn;
  Basis V, W;
  QQ_TRY(V.init(nel, m + 1));
  QQ_TRY(W.init(nel, m + 1));
  QQ_TRY(evec.init(nel, k));
  Scratch S;
  QQ_TRY(S.init(m, k + 1));
  DevBuf H;
  QQ_CK(H.alloc(sizeof(double) * 2 * (size_t)(m + 1) * m));
  double* nrm2 = S.nrm.as<double>();
  double* part = c->partial.as<double>();
  // v_1 = b / ||b||, c = (||b||, 0, ...)
  QQ_CK(cudaMemcpyAsync(V.v(0), b, nel * 16, cudaMemcpyDeviceToDevice, c->st));
  QQ_TRY(mdot(c, V, 1, V.v(0), S.h1.as<double>()));
  double bb[2];
  QQ_TRY(read_scalars(c, S.h1.as<double>(), 2, bb));
  const double rninit = std::sqrt(bb[0]);
  if (!(rninit > 0.0) || !std::isfinite(rninit)) return set_error(QQ_BAD_ARG, "start vector is zero or not finite");
  QQ_CK(cudaMemcpyAsync(nrm2, bb, sizeof(double), cudaMemcpyHostToDevice, c->st));
  QQ_CK(launch_normalize(P64, nel, V.v(0), V.v(0), nrm2, c->st));
  QQ_CK(cudaMemsetAsync(H.p, 0, H.bytes, c->st));
  std::vector<cd> cv(m + 1, 0.0);
  cv[0] = rninit;
  int j0 = 0;
  *mvp = 0;
  std::vector<double> hh(2 * (size_t)(m + 1) * m);
  for (int icycle = 1; icycle <= ncycles; ++icycle) {
    for (int j = j0; j < m; ++j) {
      QQ_TRY(op.apply(V.v(j + 1), V.v(j)));
      *mvp += 1;
      void* w = V.v(j + 1);
      double* hcol = H.as<double>() + 2 * (size_t)(m + 1) * j;
      QQ_TRY(mdot(c, V, j + 1, w, hcol));
      QQ_TRY(maxpy(c, V, j + 1, hcol, w));
      QQ_TRY(mdot(c, V, j + 1, w, S.h2.as<double>()));
      QQ_TRY(maxpy(c, V, j + 1, S.h2.as<double>(), w));
      QQ_CK(launch_finalize(part, kRedBlocks, 3, 1, nrm2, 0, c->st));
      QQ_CK(launch_hcol_update(H.as<double>(), m + 1, j, S.h2.as<double>(), j + 1, nrm2, c->st));
      QQ_CK(launch_normalize(P64, nel, w, w, nrm2, c->st));
    }
    QQ_CK(cudaMemcpyAsync(hh.data(), H.p, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    dense::Mat Hb(m + 1, m);
    for (int jj = 0; jj < m; ++jj)
      for (int i = 0; i <= m; ++i)
        Hb(i, jj) = {hh[2 * ((size_t)i + (size_t)(m + 1) * jj)], hh[2 * ((size_t)i + (size_t)(m + 1) * jj) + 1]};
    if (!std::isfinite(std::abs(Hb(m, m - 1)))) return set_error(QQ_NAN, "NaN in the Arnoldi process");
    // least squares and its residual (the linear system of the cycle)
    std::vector<cd> d, srv;
    dense::hess_lsq(Hb, cv, m, d, srv);
    double rn = 0.0;
    for (const cd& s : srv) rn += std::norm(s);
    rn = std::sqrt(rn);
    const bool last = icycle == ncycles || !(rn / rninit > 1e-160);
    // harmonic Ritz pairs: eig(H_m + h^2 f e_m^T), f = H_m^{-H} e_m
    dense::Mat Hm(m, m), HmH(m, m);
    for (int jj = 0; jj < m; ++jj)
      for (int i = 0; i < m; ++i) {
        Hm(i, jj) = Hb(i, jj);
        HmH(jj, i) = std::conj(Hb(i, jj));
      }
    std::vector<cd> f(m, 0.0);
    f[m - 1] = 1.0;
    if (!dense::lu_solve(HmH, f)) return set_error(QQ_SINGULAR, "singular projected matrix");
    const cd hl = Hb(m, m - 1);
    dense::Mat A = Hm;
    for (int i = 0; i < m; ++i) A(i, m - 1) += hl * hl * f[i];
    std::vector<cd> dd;
    dense::Mat gg;
    if (!dense::eig_vectors(A, dd, gg)) return set_error(QQ_SINGULAR, "harmonic Ritz eigenproblem failed");
    std::vector<double> mag(m);
    for (int i = 0; i < m; ++i) mag[i] = std::norm(dd[i]);
    const std::vector<int> om = stable_order(mag);
    std::vector<double> rna(k);
    for (int i = 0; i < k; ++i) {
      const int col = om[i];
      cd rho = 0.0;
      std::vector<cd> tv(m, 0.0);
      for (int r = 0; r < m; ++r) {
        cd s = 0.0;
        for (int l = 0; l < m; ++l) s += Hm(r, l) * gg(l, col);
        tv[r] = s;
        rho += std::conj(gg(r, col)) * s;
      }
      double t2 = 0.0;
      for (int r = 0; r < m; ++r) t2 += std::norm(tv[r] - rho * gg(r, col));
      rna[i] = std::sqrt(t2 + std::norm(hl) * std::norm(gg(m - 1, col)));
    }
    const std::vector<int> orr = stable_order(rna);
    dense::Mat P(m + 1, k + 1);
    for (int i = 0; i < k; ++i)
      for (int r = 0; r < m; ++r) P(r, i) = gg(r, om[orr[i]]);
    if (variant == 1) {  // the harmonic residual direction [-h f; 1]
      for (int r = 0; r < m; ++r) P(r, k) = -hl * f[r];
      P(m, k) = 1.0;
    } else {  // the least-squares residual
      for (int r = 0; r <= m; ++r) P(r, k) = srv[r];
    }
    dense::Mat Q;
    dense::house_q(P, Q);
    dense::Mat Hk(k + 1, k);
    {
      dense::Mat T(m + 1, k);
      for (int jj = 0; jj < k; ++jj)
        for (int i = 0; i <= m; ++i) {
          cd s = 0.0;
          for (int l = 0; l < m; ++l) s += Hb(i, l) * Q(l, jj);
          T(i, jj) = s;
        }
      for (int jj = 0; jj < k; ++jj)
        for (int i = 0; i <= k; ++i) {
          cd s = 0.0;
          for (int l = 0; l <= m; ++l) s += std::conj(Q(l, i)) * T(l, jj);
          Hk(i, jj) = s;
        }
    }
    // gmresdr5EIG zeroes the subdiagonal part of column i while the i-th Ritz residual in
    // |theta| order is below 1e-12 (the columns themselves are in residual order),
    // Q/inverters.f90:1895-1899
    if (variant == 2)
      for (int i = 0; i < k && rna[i] < 1e-12; ++i)
        for (int r = i + 1; r <= k; ++r) Hk(r, i) = 0.0;
    if (last) {
      dense::Mat G(m, k);
      for (int i = 0; i < k; ++i)
        for (int r = 0; r < m; ++r) G(r, i) = P(r, i);
      QQ_TRY(combine(c, V, m, G, k, S, evec));
      eval.resize(k);
      for (int i = 0; i < k; ++i) eval[i] = dd[om[orr[i]]];
      *cycles_done = icycle;
      break;
    }
    // restart: V_{k+1} = V_{m+1} Q, H = [Hk; 0], c = Q^H srv
    std::fill(cv.begin(), cv.end(), cd(0.0, 0.0));
    for (int i = 0; i <= k; ++i) {
      cd s = 0.0;
      for (int l = 0; l <= m; ++l) s += std::conj(Q(l, i)) * srv[l];
      cv[i] = s;
    }
    QQ_TRY(combine(c, V, m + 1, Q, k + 1, S, W));
    std::swap(V.buf.p, W.buf.p);
    std::swap(V.buf.bytes, W.buf.bytes);
    // one more orthogonalisation of v_{k+1} against v_1..v_k, then normalise
    QQ_TRY(mdot(c, V, k, V.v(k), S.h1.as<double>()));
    QQ_TRY(maxpy(c, V, k, S.h1.as<double>(), V.v(k)));
    QQ_CK(launch_finalize(part, kRedBlocks, 3, 1, nrm2, 0, c->st));
    QQ_CK(launch_normalize(P64, nel, V.v(k), V.v(k), nrm2, c->st));
    std::vector<double> hk(2 * (size_t)(m + 1) * m, 0.0);
    for (int jj = 0; jj < k; ++jj)
      for (int i = 0; i <= k; ++i) {
        hk[2 * ((size_t)i + (size_t)(m + 1) * jj)] = Hk(i, jj).real();
        hk[2 * ((size_t)i + (size_t)(m + 1) * jj) + 1] = Hk(i, jj).imag();
      }
    QQ_CK(cudaMemcpyAsync(H.p, hk.data(), sizeof(double) * hk.size(), cudaMemcpyHostToDevice, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    j0 = k;
    *cycles_done = icycle;
  }
  return QQ_OK;
}

int dot_full(qq_ctx* c, const void* a, const void* b, size_t hn, cd* out) {
  cd d0, d1;
  QQ_TRY(dot_host(c, half_of(const_cast<void*>(a), hn, 0), half_of(const_cast<void*>(b), hn, 0), &d0, nullptr));
  QQ_TRY(dot_host(c, half_of(const_cast<void*>(a), hn, 1), half_of(const_cast<void*>(b), hn, 1), &d1, nullptr));
  *out = d0 + d1;
  return QQ_OK;
}

// out = a * x (full vectors, complex a)
int scale_full(qq_ctx* c, void* out, cd a, const void* x, size_t hn) {
  for (int p = 0; p < 2; ++p)
    QQ_TRY(lin(c, half_of(out, hn, p), cimm(a.real(), a.imag()), half_of(const_cast<void*>(x), hn, p)));
  return QQ_OK;
}

// eigmodesofM's lift of the paired Ritz vectors of Mhat to modes of M.
int modes_of_m(qq_ctx* c, qq_eig* E, const Basis& ev, const std::vector<cd>& th, double kappa) {
  const size_t hn = E->half_nel;
  const int k = (int)th.size();
  std::vector<int> pos, neg, ind;
  for (int i = 0; i < k; ++i) {
    if (std::fabs(th[i].imag()) < kPairTol) continue;  // real: not handled by the reference
    (th[i].imag() > 0 ? pos : neg).push_back(i);
  }
  for (int p : pos)
    for (int q : neg)
      if (std::abs(th[p] - std::conj(th[q])) <= kPairTol) {
        ind.push_back(p);
        ind.push_back(q);
        break;
      }
  const int np = (int)ind.size();
  Basis Rt, Lt;
  QQ_TRY(Rt.init(2 * hn, std::max(np, 1)));
  QQ_TRY(Lt.init(2 * hn, std::max(np, 1)));
  std::vector<cd> lam(np);
  for (int e = 0; e < np; ++e) {
    const cd t = 1.0 - kappa * kappa * th[ind[e]];
    const cd s = nr_sqrt(t);
    lam[e] = 1.0 - s;
    QQ_CK(cudaMemcpyAsync(Rt.v(e), ev.v(ind[e]), hn * 16, cudaMemcpyDeviceToDevice, c->st));
    const Spinor ro = half_of(Rt.v(e), hn, 1);
    QQ_TRY(op_hsingle(c, ro, half_of(Rt.v(e), hn, 0), 0, 1));
    const cd a = kappa * nr_inv(s);
    QQ_TRY(lin(c, ro, cimm(a.real(), a.imag()), ro));
  }
  // left vectors: gamma5 times the partner's right vector
  for (int e = 0; e + 1 < np; e += 2) {
    QQ_TRY(g5(c, Rt.v(e + 1), Lt.v(e), 2));
    QQ_TRY(g5(c, Rt.v(e), Lt.v(e + 1), 2));
  }
  // <R, L> = 1, then the residual test on M
  std::vector<int> keep;
  Tmp xe(c, P64), xo(c, P64);
  for (int e = 0; e < np; ++e) {
    cd rl;
    QQ_TRY(dot_full(c, Rt.v(e), Lt.v(e), hn, &rl));
    QQ_TRY(scale_full(c, Rt.v(e), std::conj(nr_inv(rl)), Rt.v(e), hn));
    const Spinor re = half_of(Rt.v(e), hn, 0), ro = half_of(Rt.v(e), hn, 1);
    QQ_TRY(op_hsingle(c, xo.sp(), re, 0, 1));
    QQ_TRY(op_hsingle(c, xe.sp(), ro, 0, 0));
    const cd ml = -lam[e];
    QQ_TRY(lin(c, xe.sp(), cimm(1.0 + ml.real(), ml.imag()), re, cimm(-kappa), xe.sp()));
    QQ_TRY(lin(c, xo.sp(), cimm(1.0 + ml.real(), ml.imag()), ro, cimm(-kappa), xo.sp()));
    double n0, n1;
    QQ_TRY(norm2_host(c, xe.sp(), &n0));
    QQ_TRY(norm2_host(c, xo.sp(), &n1));
    if (std::sqrt(n0 + n1) < kResTolM) keep.push_back(e);
  }
  std::vector<double> mag(keep.size());
  for (size_t i = 0; i < keep.size(); ++i) mag[i] = std::abs(lam[keep[i]]);
  const std::vector<int> o = stable_order(mag);
  E->num = (int)keep.size();
  E->lam.resize(E->num);
  QQ_CK(E->R.alloc(std::max<size_t>(1, E->num) * 2 * hn * 16));
  QQ_CK(E->L.alloc(std::max<size_t>(1, E->num) * 2 * hn * 16));
  for (int i = 0; i < E->num; ++i) {
    const int e = keep[o[i]];
    E->lam[i] = lam[e];
    QQ_CK(cudaMemcpyAsync(E->r(i), Rt.v(e), 2 * hn * 16, cudaMemcpyDeviceToDevice, c->st));
    QQ_CK(cudaMemcpyAsync(E->l(i), Lt.v(e), 2 * hn * 16, cudaMemcpyDeviceToDevice, c->st));
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

// eigmodesofMprime's selection of the Ritz vectors of M gamma5.
int modes_of_mprime(qq_ctx* c, qq_eig* E, EigOp& op, Basis& ev, const std::vector<cd>& th) {
  const size_t hn = E->half_nel;
  const int k = (int)th.size();
  Basis X;
  QQ_TRY(X.init(2 * hn, 1));
  std::vector<int> keep;
  for (int i = 0; i < k; ++i) {
    double n0, n1;
    QQ_TRY(norm2_host(c, half_of(ev.v(i), hn, 0), &n0));
    QQ_TRY(norm2_host(c, half_of(ev.v(i), hn, 1), &n1));
    QQ_TRY(scale_full(c, ev.v(i), cd(1.0 / std::sqrt(n0 + n1), 0.0), ev.v(i), hn));
    QQ_TRY(op.apply(X.v(0), ev.v(i)));
    for (int p = 0; p < 2; ++p)
      QQ_TRY(lin(c, half_of(X.v(0), hn, p), cimm(1.0), half_of(X.v(0), hn, p), cimm(-th[i].real()), half_of(ev.v(i), hn, p)));
    QQ_TRY(norm2_host(c, half_of(X.v(0), hn, 0), &n0));
    QQ_TRY(norm2_host(c, half_of(X.v(0), hn, 1), &n1));
    if (std::sqrt(n0 + n1) < kResTolMp) keep.push_back(i);
  }
  std::vector<double> mag(keep.size());
  for (size_t i = 0; i < keep.size(); ++i) mag[i] = std::fabs(th[keep[i]].real());
  const std::vector<int> o = stable_order(mag);
  E->num = (int)keep.size();
  E->lam.resize(E->num);
  QQ_CK(E->R.alloc(std::max<size_t>(1, E->num) * 2 * hn * 16));
  for (int i = 0; i < E->num; ++i) {
    const int e = keep[o[i]];
    E->lam[i] = cd(th[e].real(), 0.0);
    QQ_CK(cudaMemcpyAsync(E->r(i), ev.v(e), 2 * hn * 16, cudaMemcpyDeviceToDevice, c->st));
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

// Loop traces T_j (2 nt x 9 per mode, no kappa) of each mode's R_j (kind 1) or gamma5 R_j
// (kind 2) against the noise z, and the projections <L_j, z>; z in reference layout on
// the device.
int mode_traces(qq_ctx* c, const qq_eig* E, const double* ze, const double* zo, std::vector<double>& T,
                std::vector<cd>& proj) {
  const size_t hn = E->half_nel, nv = c->ref_doubles();
  const int nt = c->g.n[3], V = 2 * c->g.vh, n = E->num;
  void *val = nullptr, *Jd = nullptr, *ref = nullptr;
  QQ_CK(ws_get(c, kWsVal, sizeof(double) * 18 * (size_t)V, &val));
  QQ_CK(ws_get(c, kWsJ, sizeof(double) * 18 * (size_t)nt, &Jd));
  QQ_CK(ws_get(c, kWsRef, sizeof(double) * 2 * nv, &ref));
  double* ye = static_cast<double*>(ref);
  double* yo = ye + nv;
  Tmp zfe(c, P64), zfo(c, P64), g5e(c, P64), g5o(c, P64);
  QQ_TRY(ref_to_field(c, ze, 0, zfe.sp()));
  QQ_TRY(ref_to_field(c, zo, 1, zfo.sp()));
  T.assign((size_t)n * 18 * nt, 0.0);
  proj.assign(n, 0.0);
  for (int j = 0; j < n; ++j) {
    cd p0, p1;
    QQ_TRY(dot_host(c, half_of(E->l(j), hn, 0), zfe.sp(), &p0, nullptr));
    QQ_TRY(dot_host(c, half_of(E->l(j), hn, 1), zfo.sp(), &p1, nullptr));
    proj[j] = p0 + p1;
    Spinor re = half_of(E->r(j), hn, 0), ro = half_of(E->r(j), hn, 1);
    if (E->kind == 2) {
      QQ_TRY(g5(c, re.data, g5e.sp().data, 1));
      QQ_TRY(g5(c, ro.data, g5o.sp().data, 1));
      re = g5e.sp();
      ro = g5o.sp();
    }
    QQ_TRY(field_to_ref(c, re, 0, ye));
    QQ_TRY(field_to_ref(c, ro, 1, yo));
    QQ_TRY(loop_slices(c, ye, yo, ze, zo, 0, static_cast<double*>(val), static_cast<double*>(Jd),
                       T.data() + (size_t)j * 18 * nt));
  }
  return QQ_OK;
}

// eigaverage from the mode traces: Jtime(2, nt, n, 9) for scalar multipliers s.
void compose_eigaverage(const std::vector<double>& T, const std::vector<cd>& proj, const double* s, int n,
                        int nt, int eigstart, int eigstep, double kappa, double* J) {
  std::memset(J, 0, sizeof(double) * 2 * (size_t)nt * n * 9);
  std::vector<cd> acc((size_t)9 * nt, 0.0);
  for (int e = 1; e <= n; ++e) {
    const cd cj = proj[e - 1] * cd(s[2 * (e - 1)], s[2 * (e - 1) + 1]);
    const double* t = T.data() + (size_t)(e - 1) * 18 * nt;
    for (int iop = 0; iop < 9; ++iop)
      for (int it = 0; it < nt; ++it)
        acc[(size_t)iop * nt + it] += cj * cd(t[((size_t)iop * nt + it) * 2], t[((size_t)iop * nt + it) * 2 + 1]);
    const bool pick = e == eigstart || (e > eigstart && (e - eigstart) % eigstep == 0) || e == n;
    if (!pick) continue;
    for (int iop = 0; iop < 9; ++iop) {
      const double f = iop < 4 ? kappa : 1.0;
      for (int it = 0; it < nt; ++it) {
        const cd v = acc[(size_t)iop * nt + it];
        const size_t o = ((((size_t)iop * n) + (e - 1)) * nt + it) * 2;
        J[o] = f * v.real();
        J[o + 1] = f * v.imag();
      }
    }
  }
}

// (M y)_e = y_e - kappa H_eo y_o, (M y)_o = y_o - kappa H_oe y_e on full vectors.
int apply_m(qq_ctx* c, void* out, const void* in, double kappa, size_t hn) {
  const Spinor ie = half_of(const_cast<void*>(in), hn, 0), io = half_of(const_cast<void*>(in), hn, 1);
  const Spinor oe = half_of(out, hn, 0), oo = half_of(out, hn, 1);
  QQ_TRY(op_hsingle(c, oe, io, 0, 0));
  QQ_TRY(lin(c, oe, cimm(1.0), ie, cimm(-kappa), oe));
  QQ_TRY(op_hsingle(c, oo, ie, 0, 1));
  QQ_TRY(lin(c, oo, cimm(1.0), io, cimm(-kappa), oo));
  return QQ_OK;
}

// The least-squares polynomials of ppaverage (p = 5), ppaverage1 (p = 8) and ppaverage2
// (p = 11), Q/disconloops.f90:6885-7434, 6290-6883, 5740-6288: the terms (coefficient
// index, power index, both 1-based: co_c M^(v-1) b) added at levels isub = 2..6.  The
// p = 5 form reuses its fifth coefficient on the powers 6, 7, 8 (:7217-7293).
struct PolyTerm {
  int co, v;
};
const std::vector<PolyTerm>& poly_terms(int p, int isub) {
  static const std::vector<PolyTerm> none;
  static const std::vector<PolyTerm> t11[7] = {{}, {}, {{1, 1}, {2, 2}, {3, 3}, {4, 4}}, {{5, 5}}, {{6, 6}}, {{7, 7}},
                                               {{8, 8}, {9, 9}, {10, 10}, {11, 11}}};
  static const std::vector<PolyTerm> t8[7] = {{}, {}, {{1, 1}, {2, 2}, {3, 3}, {4, 4}}, {{5, 5}}, {{6, 6}}, {{7, 7}},
                                              {{8, 8}}};
  static const std::vector<PolyTerm> t5[7] = {{}, {}, {{1, 1}, {2, 2}, {3, 3}, {4, 4}}, {{5, 5}}, {{5, 6}}, {{5, 7}},
                                              {{5, 8}}};
  if (isub < 1 || isub > 6) return none;
  return p == 11 ? t11[isub] : p == 8 ? t8[isub] : t5[isub];
}
int poly_powers(int p) { return p == 11 ? 12 : p == 8 ? 9 : 8; }  // vectors M^0 b .. kept

// P[i] = M^i b for i < n (full vectors)
int krylov_powers(qq_ctx* c, const void* b, double kappa, size_t hn, int n, Basis& P) {
  QQ_TRY(P.init(2 * hn, n));
  QQ_CK(cudaMemcpyAsync(P.v(0), b, 2 * hn * 16, cudaMemcpyDeviceToDevice, c->st));
  for (int i = 1; i < n; ++i) QQ_TRY(apply_m(c, P.v(i), P.v(i - 1), kappa, hn));
  return QQ_OK;
}

// sub_isub accumulated in place: sub += sum over the level's terms co_c P[v-1]
int poly_accumulate(qq_ctx* c, void* sub, const Basis& P, const double* co, int p, int isub, size_t hn) {
  for (const PolyTerm& t : poly_terms(p, isub)) {
    const cd a(co[2 * (t.co - 1)], co[2 * (t.co - 1) + 1]);
    for (int h = 0; h < 2; ++h)
      QQ_TRY(lin(c, half_of(sub, hn, h), cimm(1.0), half_of(sub, hn, h), cimm(a.real(), a.imag()),
                 half_of(P.v(t.v - 1), hn, h)));
  }
  return QQ_OK;
}

int load_full(qq_ctx* c, const double* e, const double* o, void* full, size_t hn) {
  const double* d = nullptr;
  QQ_TRY(stage_in(c, 0, e, c->ref_doubles(), &d));
  QQ_TRY(ref_to_field(c, d, 0, half_of(full, hn, 0)));
  QQ_TRY(stage_in(c, 1, o, c->ref_doubles(), &d));
  QQ_TRY(ref_to_field(c, d, 1, half_of(full, hn, 1)));
  return QQ_OK;
}

// ppaverage*: Jtime(2, nt, nsub, 9) at imom = 1 (Fortran order), x and b full vectors in
// GPU layout, b also in reference layout on the device (be_ref, bo_ref).
int ppaverage_dev(qq_ctx* c, int p, const double* co, const void* b, const double* be_ref, const double* bo_ref,
                  const void* x, double kappa, int nsub, double* J) {
  const size_t hn = (size_t)12 * c->g.vh, nv = c->ref_doubles();
  const int nt = c->g.n[3], V = 2 * c->g.vh;
  Basis P, Y;
  QQ_TRY(krylov_powers(c, b, kappa, hn, poly_powers(p), P));
  QQ_TRY(Y.init(2 * hn, 2));  // sub and y
  QQ_CK(cudaMemsetAsync(Y.v(0), 0, 2 * hn * 16, c->st));
  void *val = nullptr, *Jd = nullptr, *ref = nullptr;
  QQ_CK(ws_get(c, kWsVal, sizeof(double) * 18 * (size_t)V, &val));
  QQ_CK(ws_get(c, kWsJ, sizeof(double) * 18 * (size_t)nt, &Jd));
  QQ_CK(ws_get(c, kWsRef, sizeof(double) * 2 * nv, &ref));
  double* ye = static_cast<double*>(ref);
  std::vector<double> T((size_t)18 * nt);
  std::memset(J, 0, sizeof(double) * 2 * (size_t)nt * nsub * 9);
  for (int isub = 1; isub <= nsub; ++isub) {
    QQ_TRY(poly_accumulate(c, Y.v(0), P, co, p, isub, hn));
    for (int h = 0; h < 2; ++h)
      QQ_TRY(lin(c, half_of(Y.v(1), hn, h), cimm(1.0), half_of(const_cast<void*>(x), hn, h), cimm(-1.0),
                 half_of(Y.v(0), hn, h)));
    QQ_TRY(field_to_ref(c, half_of(Y.v(1), hn, 0), 0, ye));
    QQ_TRY(field_to_ref(c, half_of(Y.v(1), hn, 1), 1, ye + nv));
    QQ_TRY(loop_slices(c, ye, ye + nv, be_ref, bo_ref, isub == 1 ? 0 : 1, static_cast<double*>(val),
                       static_cast<double*>(Jd), T.data()));
    for (int iop = 0; iop < 9; ++iop)
      for (int it = 0; it < nt; ++it)
        for (int ri = 0; ri < 2; ++ri)
          J[((((size_t)iop * nsub) + (isub - 1)) * nt + it) * 2 + ri] =
              (iop < 4 ? kappa : 1.0) * T[((size_t)iop * nt + it) * 2 + ri];
  }
  return QQ_OK;
}

// xipolygenerator: xiinv(2, 6, n) = <L_j, gamma5 sub_isub(R_j)> with the p = 8 terms.
int xipoly_dev(qq_ctx* c, const qq_eig* e, double kappa, const double* co, double* xiinv) {
  const size_t hn = e->half_nel;
  Basis Y;
  QQ_TRY(Y.init(2 * hn, 2));
  for (int j = 0; j < e->num; ++j) {
    Basis P;
    QQ_TRY(krylov_powers(c, e->r(j), kappa, hn, poly_powers(8), P));
    QQ_CK(cudaMemsetAsync(Y.v(0), 0, 2 * hn * 16, c->st));
    for (int isub = 1; isub <= 6; ++isub) {
      QQ_TRY(poly_accumulate(c, Y.v(0), P, co, 8, isub, hn));
      QQ_TRY(g5(c, Y.v(0), Y.v(1), 2));
      cd x;
      QQ_TRY(dot_full(c, e->l(j), Y.v(1), hn, &x));
      xiinv[2 * ((size_t)(isub - 1) + 6 * (size_t)j)] = x.real();
      xiinv[2 * ((size_t)(isub - 1) + 6 * (size_t)j) + 1] = x.imag();
    }
  }
  return QQ_OK;
}

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_eigmodes(qq_ctx* c, int kind, const int nGMRES[2], int ncycles, const double kappa[2],
                           const double* se, const double* so, qq_eig** out, int* numEV, double* evals) {
  if (!c || !nGMRES || !kappa || !out) return set_error(QQ_BAD_ARG, "null argument");
  *out = nullptr;
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  if (kind != 1 && kind != 2) return set_error(QQ_BAD_ARG, "kind must be 1 (M) or 2 (M gamma5)");
  const int m = nGMRES[0], k = nGMRES[1];
  if (m < 2 || k < 1 || k >= m || m + 1 > kMaxEigBasis + 1 || m > kMaxEigBasis)
    return set_error(QQ_BAD_ARG, "nGMRES out of range (k < m <= 255)");
  if (ncycles < 1) return set_error(QQ_BAD_ARG, "ncycles must be positive");
  if (kind == 2 && (!se || !so)) return set_error(QQ_BAD_ARG, "kind 2 needs a start vector");
  QQ_CK(cudaSetDevice(c->device));
  std::unique_ptr<qq_eig> E(new qq_eig());
  E->ctx = c;
  E->kind = kind;
  E->half_nel = (size_t)12 * c->g.vh;
  const size_t hn = E->half_nel;
  EigOp op{c, kind, {kappa[0], kappa[1]}, hn, {}};
  // start vector: the unit source b(1,1,1,1,1) = 1 (kind 1) or the caller's pair
  DevBuf b;
  QQ_CK(b.alloc((kind == 1 ? 1 : 2) * hn * 16));
  QQ_CK(cudaMemsetAsync(b.p, 0, b.bytes, c->st));
  if (kind == 1) {
    const size_t nv = c->ref_doubles();
    std::vector<double> u(nv, 0.0);
    u[0] = 1.0;
    const double* d = nullptr;
    QQ_TRY(stage_in(c, 0, u.data(), nv, &d));
    QQ_TRY(ref_to_field(c, d, 0, half_of(b.p, hn, 0)));
    QQ_CK(cudaStreamSynchronize(c->st));
  } else {
    const double* d = nullptr;
    QQ_TRY(stage_in(c, 0, se, c->ref_doubles(), &d));
    QQ_TRY(ref_to_field(c, d, 0, half_of(b.p, hn, 0)));
    QQ_TRY(stage_in(c, 1, so, c->ref_doubles(), &d));
    QQ_TRY(ref_to_field(c, d, 1, half_of(b.p, hn, 1)));
  }
  Basis ev;
  std::vector<cd> th;
  QQ_TRY(eig_gmresdr(c, op, kind, b.p, m, k, ncycles, ev, th, &E->cycles, &E->mvp));
  E->ritz = th;
  E->nritz = k;
  if (kind == 1)
    QQ_TRY(modes_of_m(c, E.get(), ev, th, kappa[0]));
  else
    QQ_TRY(modes_of_mprime(c, E.get(), op, ev, th));
  if (numEV) *numEV = E->num;
  if (evals)
    for (int i = 0; i < E->num; ++i) {
      evals[2 * i] = E->lam[i].real();
      evals[2 * i + 1] = E->lam[i].imag();
    }
  *out = E.release();
  return QQ_OK;
}

extern "C" int qq_eig_destroy(qq_eig* e) {
  if (!e) return QQ_OK;
  cudaSetDevice(e->ctx->device);
  delete e;
  return QQ_OK;
}

extern "C" int qq_eig_info(const qq_eig* e, int* kind, int* numEV, int* cycles, int* mvp, double* evals,
                           double* ritz) {
  if (!e) return set_error(QQ_BAD_ARG, "null handle");
  if (kind) *kind = e->kind;
  if (numEV) *numEV = e->num;
  if (cycles) *cycles = e->cycles;
  if (mvp) *mvp = e->mvp;
  if (evals)
    for (int i = 0; i < e->num; ++i) {
      evals[2 * i] = e->lam[i].real();
      evals[2 * i + 1] = e->lam[i].imag();
    }
  if (ritz)
    for (int i = 0; i < e->nritz; ++i) {
      ritz[2 * i] = e->ritz[i].real();
      ritz[2 * i + 1] = e->ritz[i].imag();
    }
  return QQ_OK;
}

extern "C" int qq_eig_vector(const qq_eig* e, int j, int left, double* ve, double* vo) {
  if (!e || !ve || !vo) return set_error(QQ_BAD_ARG, "null argument");
  if (j < 0 || j >= e->num) return set_error(QQ_BAD_ARG, "no such mode");
  qq_ctx* c = e->ctx;
  QQ_CK(cudaSetDevice(c->device));
  void* f = left ? e->l(j) : e->r(j);
  const size_t nv = c->ref_doubles();
  for (int p = 0; p < 2; ++p) {
    double* out = p == 0 ? ve : vo;
    double* d = nullptr;
    QQ_TRY(stage_out_begin(c, 2 + p, out, nv, &d));
    QQ_TRY(field_to_ref(c, half_of(f, e->half_nel, p), p, d));
    QQ_TRY(stage_out_end(c, 2 + p, out, nv, d));
  }
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

extern "C" int qq_xigenerator(qq_ctx* c, const qq_eig* e, double kappa, double* xiinv) {
  if (!c || !e || !xiinv) return set_error(QQ_BAD_ARG, "null argument");
  if (e->ctx != c) return set_error(QQ_BAD_ARG, "handle belongs to another context");
  QQ_CK(cudaSetDevice(c->device));
  const size_t hn = e->half_nel;
  Tmp s1e(c, P64), s1o(c, P64), s2e(c, P64), s2o(c, P64), se(c, P64), so(c, P64), ge(c, P64), go(c, P64);
  auto H = [&](const Tmp& out, Spinor in, int pout) { return op_hsingle(c, out.sp(), in, 0, pout); };
  auto axpy = [&](const Tmp& y, double a, const Tmp& x) {
    return lin(c, y.sp(), cimm(1.0), y.sp(), cimm(a), x.sp());
  };
  for (int j = 0; j < e->num; ++j) {
    const Spinor be = half_of(e->r(j), hn, 0), bo = half_of(e->r(j), hn, 1);
    const Spinor le = half_of(e->l(j), hn, 0), lo = half_of(e->l(j), hn, 1);
    for (int isub = 1; isub <= 6; ++isub) {
      if (isub == 1) {
        QQ_TRY(zero_field(c, se.sp()));
        QQ_TRY(zero_field(c, so.sp()));
      } else if (isub == 2) {  // O(kappa) .. O(kappa^3)
        QQ_TRY(H(s1e, bo, 0));
        QQ_TRY(H(s1o, be, 1));
        QQ_TRY(copy_field(c, se.sp(), be));
        QQ_TRY(copy_field(c, so.sp(), bo));
        QQ_TRY(axpy(se, kappa, s1e));
        QQ_TRY(axpy(so, kappa, s1o));
        QQ_TRY(H(s2e, s1o.sp(), 0));
        QQ_TRY(H(s2o, s1e.sp(), 1));
        QQ_TRY(axpy(se, kappa * kappa, s2e));
        QQ_TRY(axpy(so, kappa * kappa, s2o));
        QQ_TRY(H(s1e, s2o.sp(), 0));
        QQ_TRY(H(s1o, s2e.sp(), 1));
        QQ_TRY(axpy(se, kappa * kappa * kappa, s1e));
        QQ_TRY(axpy(so, kappa * kappa * kappa, s1o));
      } else {  // O(kappa^(isub+1)), the scratch pairs alternating
        const double xk = std::pow(kappa, isub + 1);
        if (isub % 2 == 1) {
          QQ_TRY(H(s2e, s1o.sp(), 0));
          QQ_TRY(H(s2o, s1e.sp(), 1));
          QQ_TRY(axpy(se, xk, s2e));
          QQ_TRY(axpy(so, xk, s2o));
        } else {
          QQ_TRY(H(s1e, s2o.sp(), 0));
          QQ_TRY(H(s1o, s2e.sp(), 1));
          QQ_TRY(axpy(se, xk, s1e));
          QQ_TRY(axpy(so, xk, s1o));
        }
      }
      Spinor te = se.sp(), to = so.sp();
      if (e->kind == 2) {
        QQ_TRY(g5(c, te.data, ge.sp().data, 1));
        QQ_TRY(g5(c, to.data, go.sp().data, 1));
        te = ge.sp();
        to = go.sp();
      }
      cd d0, d1;
      QQ_TRY(dot_host(c, le, te, &d0, nullptr));
      QQ_TRY(dot_host(c, lo, to, &d1, nullptr));
      const cd x = d0 + d1;
      xiinv[2 * ((size_t)(isub - 1) + 6 * (size_t)j)] = x.real();
      xiinv[2 * ((size_t)(isub - 1) + 6 * (size_t)j) + 1] = x.imag();
    }
  }
  return QQ_OK;
}

extern "C" int qq_eigaverage(qq_ctx* c, const qq_eig* e, const double* ze, const double* zo, double kappa,
                             const double* scal, int eigstart, int eigstep, double* Jtime) {
  if (!c || !e || !ze || !zo || !scal || !Jtime) return set_error(QQ_BAD_ARG, "null argument");
  if (e->ctx != c) return set_error(QQ_BAD_ARG, "handle belongs to another context");
  if (eigstart < 1 || eigstep < 1) return set_error(QQ_BAD_ARG, "eigstart and eigstep must be positive");
  QQ_CK(cudaSetDevice(c->device));
  const size_t nv = c->ref_doubles();
  DevBuf z;
  QQ_CK(z.alloc(sizeof(double) * 2 * nv));
  QQ_CK(cudaMemcpyAsync(z.p, ze, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(z.as<double>() + nv, zo, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  std::vector<double> T;
  std::vector<cd> proj;
  QQ_TRY(mode_traces(c, e, z.as<double>(), z.as<double>() + nv, T, proj));
  std::vector<double> out(2 * (size_t)c->g.n[3] * std::max(1, e->num) * 9);
  compose_eigaverage(T, proj, scal, e->num, c->g.n[3], eigstart, eigstep, kappa, out.data());
  QQ_CK(cudaMemcpy(Jtime, out.data(), sizeof(double) * 2 * (size_t)c->g.n[3] * e->num * 9, cudaMemcpyDefault));
  return QQ_OK;
}

extern "C" int qq_ppcoeffs(qq_ctx* c, const double* be, const double* bo, double kappa, int p, double* co) {
  if (!c || !be || !bo || !co) return set_error(QQ_BAD_ARG, "null argument");
  if (p < 1 || p > 16) return set_error(QQ_BAD_ARG, "p must be 1..16");
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  QQ_CK(cudaSetDevice(c->device));
  const size_t hn = (size_t)12 * c->g.vh;
  DevBuf b, h;
  QQ_CK(b.alloc(2 * hn * 16));
  QQ_CK(h.alloc(sizeof(double) * 2 * (p + 1)));
  QQ_TRY(load_full(c, be, bo, b.p, hn));
  Basis P;
  QQ_TRY(krylov_powers(c, b.p, kappa, hn, p + 1, P));
  // normal equations G co = r, G(a, b) = <M^a b, M^b b>, r(a) = <M^a b, b> (a, b = 1..p)
  dense::Mat G(p, p);
  std::vector<dense::cd> r(p);
  std::vector<double> hv(2 * (p + 1));
  for (int bb = 0; bb <= p; ++bb) {
    QQ_TRY(mdot(c, P, p + 1, P.v(bb), h.as<double>()));
    QQ_TRY(read_scalars(c, h.as<double>(), 2 * (p + 1), hv.data()));
    for (int a = 1; a <= p; ++a) {
      const dense::cd v(hv[2 * a], hv[2 * a + 1]);
      if (bb == 0)
        r[a - 1] = v;
      else
        G(a - 1, bb - 1) = v;
    }
  }
  if (!dense::lu_solve(G, r)) return set_error(QQ_SINGULAR, "singular normal equations");
  for (int a = 0; a < p; ++a) {
    co[2 * a] = r[a].real();
    co[2 * a + 1] = r[a].imag();
  }
  return QQ_OK;
}

extern "C" int qq_ppaverage(qq_ctx* c, int p, const double* co, const double* be, const double* bo, const double* xe,
                            const double* xo, double kappa, int nsub, double* Jtime) {
  if (!c || !co || !be || !bo || !xe || !xo || !Jtime) return set_error(QQ_BAD_ARG, "null argument");
  if (p != 5 && p != 8 && p != 11) return set_error(QQ_BAD_ARG, "p must be 5, 8 or 11");
  if (nsub < 1 || nsub > 6) return set_error(QQ_BAD_ARG, "nsub must be 1..6");
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  QQ_CK(cudaSetDevice(c->device));
  const size_t hn = (size_t)12 * c->g.vh, nv = c->ref_doubles();
  DevBuf bx, bref;
  QQ_CK(bx.alloc(2 * 2 * hn * 16));
  QQ_CK(bref.alloc(sizeof(double) * 2 * nv));
  void* b = bx.p;
  void* x = static_cast<char*>(bx.p) + 2 * hn * 16;
  QQ_TRY(load_full(c, be, bo, b, hn));
  QQ_CK(cudaMemcpyAsync(bref.p, be, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(bref.as<double>() + nv, bo, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_TRY(load_full(c, xe, xo, x, hn));
  std::vector<double> J(2 * (size_t)c->g.n[3] * nsub * 9);
  QQ_TRY(ppaverage_dev(c, p, co, b, bref.as<double>(), bref.as<double>() + nv, x, kappa, nsub, J.data()));
  QQ_CK(cudaMemcpy(Jtime, J.data(), sizeof(double) * J.size(), cudaMemcpyDefault));
  return QQ_OK;
}

extern "C" int qq_xipolygenerator(qq_ctx* c, const qq_eig* e, double kappa, const double* co, double* xiinv) {
  if (!c || !e || !co || !xiinv) return set_error(QQ_BAD_ARG, "null argument");
  if (e->ctx != c) return set_error(QQ_BAD_ARG, "handle belongs to another context");
  QQ_CK(cudaSetDevice(c->device));
  std::vector<double> xi(2 * 6 * (size_t)std::max(1, e->num));
  QQ_TRY(xipoly_dev(c, e, kappa, co, xi.data()));
  QQ_CK(cudaMemcpy(xiinv, xi.data(), sizeof(double) * 12 * (size_t)e->num, cudaMemcpyDefault));
  return QQ_OK;
}

extern "C" int qq_generalaverage(qq_ctx* c, const qq_eig* m, const qq_eig* mp, const double* ze, const double* zo,
                                 const double* xe, const double* xo, double kappa, int eigstart, int eigstep,
                                 const double* co11, const double* co8, const double* co5, const double* copoly,
                                 double* Jave) {
  if (!c || !m || !mp || !ze || !zo || !xe || !xo || !co11 || !co8 || !co5 || !copoly || !Jave)
    return set_error(QQ_BAD_ARG, "null argument");
  if (m->ctx != c || mp->ctx != c) return set_error(QQ_BAD_ARG, "handle belongs to another context");
  if (m->kind != 1 || mp->kind != 2) return set_error(QQ_BAD_ARG, "need the modes of M (kind 1) and of M gamma5 (kind 2)");
  if (eigstart < 1 || eigstep < 1) return set_error(QQ_BAD_ARG, "eigstart and eigstep must be positive");
  QQ_CK(cudaSetDevice(c->device));
  const int nt = c->g.n[3], nsub = 6, nsty = 10;
  const size_t hn = (size_t)12 * c->g.vh, nv = c->ref_doubles();
  const int n1 = m->num, n2 = mp->num, nmax = std::max(n1, n2);
  // device copies: z and x (reference layout), z and a zero solution (GPU layout)
  DevBuf zr, zx, zero;
  QQ_CK(zr.alloc(sizeof(double) * 4 * nv));
  double* zref = zr.as<double>();
  QQ_CK(cudaMemcpyAsync(zref, ze, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(zref + nv, zo, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(zref + 2 * nv, xe, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(cudaMemcpyAsync(zref + 3 * nv, xo, sizeof(double) * nv, cudaMemcpyDefault, c->st));
  QQ_CK(zx.alloc(2 * hn * 16));
  QQ_CK(zero.alloc(2 * hn * 16));
  QQ_CK(cudaMemsetAsync(zero.p, 0, zero.bytes, c->st));
  QQ_TRY(ref_to_field(c, zref, 0, half_of(zx.p, hn, 0)));
  QQ_TRY(ref_to_field(c, zref + nv, 1, half_of(zx.p, hn, 1)));
  // NS: loop operators of the solution, operators 1..4 times kappa
  std::vector<double> NS((size_t)18 * nt);
  {
    void *val = nullptr, *Jd = nullptr;
    QQ_CK(ws_get(c, kWsVal, sizeof(double) * 18 * (size_t)2 * c->g.vh, &val));
    QQ_CK(ws_get(c, kWsJ, sizeof(double) * 18 * (size_t)nt, &Jd));
    QQ_TRY(loop_slices(c, zref + 2 * nv, zref + 3 * nv, zref, zref + nv, 0, static_cast<double*>(val),
                       static_cast<double*>(Jd), NS.data()));
    for (int iop = 0; iop < 4; ++iop)
      for (int k = 0; k < 2 * nt; ++k) NS[(size_t)iop * 2 * nt + k] *= kappa;
  }
  // PS = -average(z, 0); PP = -ppaverage2(0), PP4 = -ppaverage(0), PP7 = -ppaverage1(0)
  std::vector<double> PS((size_t)2 * nt * nsub * 9), PP(PS.size()), PP4(PS.size()), PP7(PS.size());
  {
    DevBuf zref0;
    QQ_CK(zref0.alloc(sizeof(double) * nv));
    QQ_CK(cudaMemsetAsync(zref0.p, 0, zref0.bytes, c->st));
    QQ_TRY(qq_average(c, zref, zref + nv, zref0.as<double>(), zref0.as<double>(), kappa, nsub, 1, 9, nullptr,
                      PS.data()));
  }
  QQ_TRY(ppaverage_dev(c, 11, co11, zx.p, zref, zref + nv, zero.p, kappa, nsub, PP.data()));
  QQ_TRY(ppaverage_dev(c, 5, co5, zx.p, zref, zref + nv, zero.p, kappa, nsub, PP4.data()));
  QQ_TRY(ppaverage_dev(c, 8, co8, zx.p, zref, zref + nv, zero.p, kappa, nsub, PP7.data()));
  for (size_t i = 0; i < PS.size(); ++i) {
    PS[i] = -PS[i];
    PP[i] = -PP[i];
    PP4[i] = -PP4[i];
    PP7[i] = -PP7[i];
  }
  // the eigenmode corrections from each mode's traces
  std::vector<double> T1, T2;
  std::vector<cd> p1, p2;
  QQ_TRY(mode_traces(c, m, zref, zref + nv, T1, p1));
  QQ_TRY(mode_traces(c, mp, zref, zref + nv, T2, p2));
  std::vector<double> s1(2 * (size_t)std::max(1, n1)), s2(2 * (size_t)std::max(1, n2));
  for (int j = 0; j < n1; ++j) {
    const cd v = nr_inv(m->lam[j]);
    s1[2 * j] = v.real();
    s1[2 * j + 1] = v.imag();
  }
  for (int j = 0; j < n2; ++j) {
    s2[2 * j] = 1.0 / mp->lam[j].real();
    s2[2 * j + 1] = 0.0;
  }
  std::vector<double> xi1(12 * (size_t)std::max(1, n1)), xi2(12 * (size_t)std::max(1, n2)),
      xip(12 * (size_t)std::max(1, n2));
  QQ_TRY(qq_xigenerator(c, m, kappa, xi1.data()));
  QQ_TRY(qq_xigenerator(c, mp, kappa, xi2.data()));
  QQ_TRY(xipoly_dev(c, mp, kappa, copoly, xip.data()));
  const size_t blk1 = (size_t)2 * nt * std::max(1, n1) * 9, blk2 = (size_t)2 * nt * std::max(1, n2) * 9;
  std::vector<double> ES(blk1), HFES(blk2), ESPS(blk1 * nsub), HFESPS(blk2 * nsub), HFESPOLY(blk2 * nsub);
  compose_eigaverage(T1, p1, s1.data(), n1, nt, eigstart, eigstep, kappa, ES.data());
  compose_eigaverage(T2, p2, s2.data(), n2, nt, eigstart, eigstep, kappa, HFES.data());
  std::vector<double> sc(2 * (size_t)std::max(n1, n2) + 2);
  for (int isub = 0; isub < nsub; ++isub) {
    for (int j = 0; j < n1; ++j) {
      sc[2 * j] = xi1[2 * ((size_t)isub + 6 * j)];
      sc[2 * j + 1] = xi1[2 * ((size_t)isub + 6 * j) + 1];
    }
    compose_eigaverage(T1, p1, sc.data(), n1, nt, eigstart, eigstep, kappa, ESPS.data() + isub * blk1);
    for (int j = 0; j < n2; ++j) {
      sc[2 * j] = xi2[2 * ((size_t)isub + 6 * j)];
      sc[2 * j + 1] = xi2[2 * ((size_t)isub + 6 * j) + 1];
    }
    compose_eigaverage(T2, p2, sc.data(), n2, nt, eigstart, eigstep, kappa, HFESPS.data() + isub * blk2);
    for (int j = 0; j < n2; ++j) {
      sc[2 * j] = xip[2 * ((size_t)isub + 6 * j)];
      sc[2 * j + 1] = xip[2 * ((size_t)isub + 6 * j) + 1];
    }
    compose_eigaverage(T2, p2, sc.data(), n2, nt, eigstart, eigstep, kappa, HFESPOLY.data() + isub * blk2);
  }
  // generalaverage's styles at imom = 1 (Q/disconloops.f90:283-329); a mode count beyond
  // one side's modes reads that side's (zero) entries, as the reference's arrays do
  auto ns = [&](int iop, int t, int ri) { return NS[((size_t)iop * nt + t) * 2 + ri]; };
  auto lvl = [&](const std::vector<double>& A, int iop, int isub, int t, int ri) {
    return A[((((size_t)iop * nsub) + isub) * nt + t) * 2 + ri];
  };
  auto eg = [&](const std::vector<double>& A, int n, size_t off, int iop, int e, int t, int ri) {
    return e < n ? A[off + ((((size_t)iop * n) + e) * nt + t) * 2 + ri] : 0.0;
  };
  const size_t total = (size_t)2 * nt * nsub * std::max(1, nmax) * nsty * 9;
  std::vector<double> out(total, 0.0);
  for (int iop = 0; iop < 9; ++iop)
    for (int sty = 1; sty <= nsty; ++sty)
      for (int e = 0; e < nmax; ++e)
        for (int isub = 0; isub < nsub; ++isub)
          for (int t = 0; t < nt; ++t)
            for (int ri = 0; ri < 2; ++ri) {
              const double N = ns(iop, t, ri);
              double v = 0.0;
              bool set = true;
              switch (sty) {
                case 1: set = e == 0 && isub == 0; v = N; break;
                case 2: set = e == 0; v = N - lvl(PS, iop, isub, t, ri); break;
                case 3: set = isub == 0; v = N - eg(ES, n1, 0, iop, e, t, ri); break;
                case 4: set = isub == 0; v = N - eg(HFES, n2, 0, iop, e, t, ri); break;
                case 5:
                  v = N - eg(ES, n1, 0, iop, e, t, ri) -
                      (lvl(PS, iop, isub, t, ri) - eg(ESPS, n1, isub * blk1, iop, e, t, ri));
                  break;
                case 6:
                  v = N - eg(HFES, n2, 0, iop, e, t, ri) -
                      (lvl(PS, iop, isub, t, ri) - eg(HFESPS, n2, isub * blk2, iop, e, t, ri));
                  break;
                case 7: set = e == 0; v = N - lvl(PP, iop, isub, t, ri); break;
                case 8: set = e == 0; v = N - lvl(PP4, iop, isub, t, ri); break;
                case 9: set = e == 0; v = N - lvl(PP7, iop, isub, t, ri); break;
                default:
                  v = N - eg(HFES, n2, 0, iop, e, t, ri) -
                      (lvl(PP7, iop, isub, t, ri) - eg(HFESPOLY, n2, isub * blk2, iop, e, t, ri));
                  break;
              }
              if (!set) continue;
              out[((((((size_t)iop * nsty) + (sty - 1)) * std::max(1, nmax) + e) * nsub + isub) * nt + t) * 2 + ri] = v;
            }
  QQ_CK(cudaMemcpy(Jave, out.data(), sizeof(double) * out.size(), cudaMemcpyDefault));
  return QQ_OK;
}
