// extern "C" entry points of libqqcd_gpu.so (declared in include/qqcd_gpu.h).
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "qq_ctx.h"

namespace qq {
const char* last_error();
int sources_z(qq_ctx* c, double* be, double* bo, bool z4);
int sources_point(qq_ctx* c, double* be, double* bo, const int src[4], int icsrc, int idsrc);
int lagfib_init(int myid, int iseed);
int lagfib_rnds(int m, double* rn);
int batch_solve(qq_ctx* c, int nrhs, const double* be, const double* bo, const double kappa[2],
                const qq_method* method, double* xe, double* xo, qq_solve_info* infos);
int traces_level0(qq_ctx* c, const double* be, const double* bo, const double* xe,
                  const double* xo, double kappa, double delta, int dobndry, double* J);
}  // namespace qq

using namespace qq;

namespace {

struct Timer {
  qq_ctx* c;
  explicit Timer(qq_ctx* c_) : c(c_) { cudaEventRecord(c->ev0, c->st); }
  double seconds() {
    cudaEventRecord(c->ev1, c->st);
    cudaEventSynchronize(c->ev1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    return ms * 1e-3;
  }
};

int check_ctx(const qq_ctx* c) {
  if (!c) return set_error(QQ_BAD_ARG, "null context");
  return QQ_OK;
}

int set_device(qq_ctx* c) {
  QQ_CK(cudaSetDevice(c->device));
  return QQ_OK;
}

// Load the reference half-vector `ref` (host or device) into field f (parity p).
int load_half(qq_ctx* c, int slot, const double* ref, int parity, Spinor f) {
  const double* d = nullptr;
  QQ_TRY(stage_in(c, slot, ref, c->ref_doubles(), &d));
  return ref_to_field(c, d, parity, f);
}

int store_half(qq_ctx* c, int slot, Spinor f, int parity, double* ref) {
  double* d = nullptr;
  QQ_TRY(stage_out_begin(c, slot, ref, c->ref_doubles(), &d));
  QQ_TRY(field_to_ref(c, f, parity, d));
  QQ_TRY(stage_out_end(c, slot, ref, c->ref_doubles(), d));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

int check_iflag(int iflag) {
  if (iflag != -1) return set_error(QQ_BAD_ARG, "only iflag = -1 (Wilson / twisted mass) is supported");
  return QQ_OK;
}

}  // namespace

extern "C" {

const char* qq_last_error(void) { return qq::last_error(); }

int qq_ctx_create(const qq_geom* geom, int device, qq_ctx** out) {
  if (!geom || !out) return set_error(QQ_BAD_ARG, "null argument");
  *out = nullptr;
  const int n[4] = {geom->nx, geom->ny, geom->nz, geom->nt};
  for (int mu = 0; mu < 4; ++mu) {
    if (n[mu] <= 0 || n[mu] % 4) return set_error(QQ_BAD_ARG, "lattice extents must be positive multiples of 4");
    if (geom->bc[mu] < -1 || geom->bc[mu] > 1) return set_error(QQ_BAD_ARG, "bc must be 1, -1 or 0");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(QQ_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return set_error(QQ_BAD_ARG, "bad device index");
  auto* c = new qq_ctx();
  c->device = device;
  if (const char* f = std::getenv("QQ_FORCE_TPS")) c->forced_tps = std::atoi(f);  // testing
  if (c->forced_tps < 0 || c->forced_tps > kShapeMax) c->forced_tps = 0;
  for (int mu = 0; mu < 4; ++mu) {
    c->g.n[mu] = n[mu];
    c->g.bc[mu] = geom->bc[mu];
    c->c1[mu] = geom->c1[mu];
    c->c2[mu] = geom->c2[mu];
  }
  const long long V = (long long)n[0] * n[1] * n[2] * n[3];
  geom_finish(c->g);  // vh, nxh, float/double bc, fast divisors
  const int nvhalf = (int)(V / 32);
  int nbmax = 0;
  for (int mu = 0; mu < 4; ++mu) nbmax = std::max(nbmax, 2 * nvhalf / n[mu]);
  c->rd.nvhalf = nvhalf;
  c->rd.ntotal = nvhalf + nbmax;
  int st = set_device(c);
  if (st == QQ_OK && cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) st = QQ_CUDA_ERR;
  if (st == QQ_OK && cudaEventCreate(&c->ev0) != cudaSuccess) st = QQ_CUDA_ERR;
  if (st == QQ_OK && cudaEventCreate(&c->ev1) != cudaSuccess) st = QQ_CUDA_ERR;
  if (st == QQ_OK && cudaEventCreate(&c->tev0) != cudaSuccess) st = QQ_CUDA_ERR;
  if (st == QQ_OK && cudaEventCreate(&c->tev1) != cudaSuccess) st = QQ_CUDA_ERR;
  if (st == QQ_OK && c->partial.alloc(sizeof(double) * kRedBlocks * 16 * 16) != cudaSuccess) st = QQ_CUDA_ERR;
  if (st == QQ_OK && c->scal.alloc(sizeof(double) * 1024) != cudaSuccess) st = QQ_CUDA_ERR;
  if (st == QQ_OK && cudaMallocHost(&c->hpin, sizeof(double) * 3072) != cudaSuccess) st = QQ_CUDA_ERR;
  if (st != QQ_OK) {
    qq_ctx_destroy(c);
    return set_error(QQ_CUDA_ERR, "context allocation failed");
  }
  *out = c;
  return QQ_OK;
}

int qq_ctx_destroy(qq_ctx* c) {
  if (!c) return QQ_OK;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  for (auto& p : c->pool) p.clear();
  c->ws.clear();
  if (c->aux_st) cudaStreamDestroy(c->aux_st);
  if (c->hpin) cudaFreeHost(c->hpin);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->tev0) cudaEventDestroy(c->tev0);
  if (c->tev1) cudaEventDestroy(c->tev1);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return QQ_OK;
}

int qq_ctx_dims(const qq_ctx* c, int* nvhalf, int* ntotal) {
  QQ_TRY(check_ctx(c));
  if (nvhalf) *nvhalf = c->rd.nvhalf;
  if (ntotal) *ntotal = c->rd.ntotal;
  return QQ_OK;
}

int qq_set_coact(qq_ctx* c, const double c1[4], const double c2[4]) {
  QQ_TRY(check_ctx(c));
  for (int mu = 0; mu < 4; ++mu) {
    c->c1[mu] = c1[mu];
    c->c2[mu] = c2[mu];
  }
  return QQ_OK;
}

int qq_gauge_upload(qq_ctx* c, const double* u_ref, int recon) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (recon != 0 && recon != 12 && recon != 18) return set_error(QQ_BAD_ARG, "recon must be 0, 12 or 18");
  const size_t nu = (size_t)18 * c->rd.ntotal * 4 * 2 * 16;
  const double* d = nullptr;
  QQ_TRY(stage_in(c, 0, u_ref, nu, &d));
  QQ_CK(launch_su3_defect(c->g, c->rd, d, c->partial.as<double>(), c->st));
  std::vector<double> part(kRedBlocks);
  QQ_CK(cudaMemcpyAsync(part.data(), c->partial.p, sizeof(double) * kRedBlocks, cudaMemcpyDeviceToHost, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  double defect = 0.0;
  for (double v : part) defect = std::max(defect, v);
  if (!std::isfinite(defect)) return set_error(QQ_NAN, "NaN in gauge field");
  if (recon == 0) recon = defect < 1e-12 ? 12 : 18;
  const int vh = c->g.vh;
  QQ_CK(c->gauge64.alloc((size_t)2 * 4 * (recon == 18 ? 9 : 6) * vh * 16));
  QQ_CK(launch_gauge_from_ref(c->g, c->rd, d, c->gauge64.p, P64, recon, c->st));
  QQ_CK(c->gauge32.alloc((size_t)2 * 4 * 3 * vh * 16));
  QQ_CK(launch_gauge_from_ref(c->g, c->rd, d, c->gauge32.p, P32, 12, c->st));
  QQ_CK(cudaStreamSynchronize(c->st));
  c->recon64 = recon;
  c->have_gauge = true;
  return QQ_OK;
}

int qq_hsingle(qq_ctx* c, double* gout, const double* gin, int idag, int gblclr) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (gblclr != 1 && gblclr != 2) return set_error(QQ_BAD_ARG, "gblclr must be 1 or 2");
  if (idag != 0 && idag != 1) return set_error(QQ_BAD_ARG, "idag must be 0 or 1");
  if (!gout || !gin) return set_error(QQ_BAD_ARG, "null array");
  Tmp in(c, P64), out(c, P64);
  const int pout = gblclr - 1;
  QQ_TRY(load_half(c, 1, gin, 1 - pout, in.sp()));
  QQ_TRY(op_hsingle(c, out.sp(), in.sp(), idag, pout));
  return store_half(c, 2, out.sp(), pout, gout);
}

int qq_hdouble(qq_ctx* c, double* he, const double* ge, int idag, double kappa) {
  const double k2[2] = {kappa, 0.0};
  return qq_hdbletm(c, he, ge, idag, k2, -1);
}

int qq_hdbletm(qq_ctx* c, double* he, const double* ge, int idag, const double kappa[2], int iflag) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  QQ_TRY(check_iflag(iflag));
  if (!he || !ge || !kappa) return set_error(QQ_BAD_ARG, "null argument");
  if (idag != 0 && idag != 1) return set_error(QQ_BAD_ARG, "idag must be 0 or 1");
  Tmp in(c, P64), out(c, P64), tmp(c, P64);
  QQ_TRY(load_half(c, 1, ge, 0, in.sp()));
  QQ_TRY(op_dbletm(c, out.sp(), in.sp(), tmp.sp(), idag, kappa));
  return store_half(c, 2, out.sp(), 0, he);
}

// twMshift: h_e = g_e + t J g_e - fac1 J (H_eo g_o), h_o likewise; J = i gamma5 and
// t = -1/(2 kappa mu), fac1 = 1/(2 mu)  (Q/diracops.f90:1880-1925).
int qq_twmshift(qq_ctx* c, double* hwhole, const double* gwhole, int idag, const double kappa[2],
                int iflag) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  QQ_TRY(check_iflag(iflag));
  if (!hwhole || !gwhole || !kappa) return set_error(QQ_BAD_ARG, "null argument");
  const size_t nv = c->ref_doubles();
  Tmp ge(c, P64), go(c, P64), he(c, P64), ho(c, P64);
  QQ_TRY(load_half(c, 1, gwhole, 0, ge.sp()));
  QQ_TRY(load_half(c, 2, gwhole + nv, 1, go.sp()));
  const double fac1 = 1.0 / (2.0 * kappa[1]);
  const double fac2 = 1.0 / (2.0 * kappa[0] * kappa[1]);
  Tmp h(c, P64);
  QQ_TRY(op_hsingle(c, h.sp(), go.sp(), idag, 0));
  QQ_CK(launch_spinmix(c->g.vh, ge.sp(), h.sp(), he.sp(), 1.0, -fac2, 0.0, -fac1, P64, c->st));
  QQ_TRY(op_hsingle(c, h.sp(), ge.sp(), idag, 1));
  QQ_CK(launch_spinmix(c->g.vh, go.sp(), h.sp(), ho.sp(), 1.0, -fac2, 0.0, -fac1, P64, c->st));
  QQ_TRY(store_half(c, 3, he.sp(), 0, hwhole));
  return store_half(c, 3, ho.sp(), 1, hwhole + nv);
}

// gamma5mult (Q/diracops.f90:1750-1860): he = -i gamma5 Hdbletm'(ge) / (2 kappa mu), with
// Hdbletm' the twisted form for every mu /= 0.  iflag must be -1 (the reference stops on
// the clover flag).
int qq_gamma5mult(qq_ctx* c, double* he, const double* ge, int idag, const double kappa[2], int iflag) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (iflag != -1) return set_error(QQ_BAD_ARG, "gamma5mult: iflag must be -1 (no clover term)");
  if (!he || !ge || !kappa) return set_error(QQ_BAD_ARG, "null argument");
  if (idag != 0 && idag != 1) return set_error(QQ_BAD_ARG, "idag must be 0 or 1");
  Tmp in(c, P64), out(c, P64), tmp(c, P64);
  QQ_TRY(load_half(c, 1, ge, 0, in.sp()));
  QQ_TRY(op_g5mult(c, out.sp(), in.sp(), tmp.sp(), idag, kappa, 0.0));
  return store_half(c, 2, out.sp(), 0, he);
}

// gmresdrshift (Q/inverters.f90:6041-7179) with the shifts as an argument.
int qq_gmresdrshift(qq_ctx* c, const double* b, double* xshift, int nshifts, const double* sigma,
                    const int GMRES[2], double resmax, int itermin, const double kappa[2], int iflag,
                    double* resid, qq_solve_info* info) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (iflag != -1) return set_error(QQ_BAD_ARG, "gmresdrshift: iflag must be -1 (no clover term)");
  if (!b || !xshift || !sigma || !GMRES || !kappa || !resid) return set_error(QQ_BAD_ARG, "null argument");
  if (nshifts < 1 || nshifts > 512) return set_error(QQ_BAD_ARG, "nshifts must be in 1..512");
  for (int q = 0; q < nshifts; ++q)
    if (!std::isfinite(sigma[q])) return set_error(QQ_BAD_ARG, "shift is not finite");
  const double t = 2.0 * kappa[0] * kappa[1];
  if (!(t != 0.0) || !std::isfinite(1.0 / t)) return set_error(QQ_BAD_ARG, "gmresdrshift needs kappa*mu /= 0");
  Tmp fb(c, P64);
  QQ_TRY(load_half(c, 1, b, 0, fb.sp()));
  std::vector<std::unique_ptr<Tmp>> fx, fr;
  std::vector<Spinor> xs, rs;
  for (int q = 0; q < nshifts; ++q) {
    fx.emplace_back(new Tmp(c, P64));
    fr.emplace_back(new Tmp(c, P64));
    xs.push_back(fx.back()->sp());
    rs.push_back(fr.back()->sp());
  }
  Timer tm(c);
  SolveStats st;
  int status = gmresdrshift_fp64(c, fb.sp(), xs, rs, sigma, GMRES[0], GMRES[1], resmax, itermin, kappa,
                                 resid, &st);
  const double sec = tm.seconds();
  fill_info(info, status, st, sec);
  if (status != QQ_OK && status != QQ_NOT_CONVERGED) return status;
  const size_t nv = c->ref_doubles();
  for (int q = 0; q < nshifts; ++q) QQ_TRY(store_half(c, 3, xs[q], 0, xshift + (size_t)q * nv));
  return status;
}

int qq_vecdot(qq_ctx* c, const double* a, const double* b, double adb[2]) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (!a || !b || !adb) return set_error(QQ_BAD_ARG, "null argument");
  Tmp fa(c, P64), fb(c, P64);
  QQ_TRY(load_half(c, 1, a, 0, fa.sp()));
  QQ_TRY(load_half(c, 2, b, 0, fb.sp()));
  std::complex<double> d;
  QQ_TRY(dot_host(c, fa.sp(), fb.sp(), &d, nullptr));
  adb[0] = d.real();
  adb[1] = d.imag();
  return QQ_OK;
}

int qq_defl_create(qq_ctx* c, int nmax, int kmax, qq_defl** out) {
  QQ_TRY(check_ctx(c));
  if (!out || nmax < 2 || kmax < 1 || kmax >= nmax) return set_error(QQ_BAD_ARG, "bad deflation sizes");
  auto* d = new qq_defl();
  d->ctx = c;
  d->nmax = nmax;
  d->kmax = kmax;
  *out = d;
  return QQ_OK;
}

int qq_defl_destroy(qq_defl* d) {
  delete d;
  return QQ_OK;
}

int qq_defl_size(const qq_defl* d) { return d ? d->space.k : 0; }

int qq_defl_vector(const qq_defl* d, int j, double* v) {
  if (!d || !v) return set_error(QQ_BAD_ARG, "null argument");
  if (j < 0 || j > d->space.k || d->space.k == 0) return set_error(QQ_BAD_ARG, "no such deflation vector");
  qq_ctx* c = d->ctx;
  QQ_TRY(set_device(c));
  const Spinor f{static_cast<char*>(d->space.V.p) + (size_t)j * d->space.nel * 16, nullptr, d->space.pb};
  double* o = nullptr;
  const size_t nv = c->ref_doubles();
  QQ_TRY(stage_out_begin(c, 2, v, nv, &o));
  if (d->space.pb == P64) {
    QQ_TRY(field_to_ref(c, f, 0, o));
  } else {  // a reduced-precision space: through an FP64 temporary
    Tmp t(c, P64);
    QQ_TRY(lin(c, t.sp(), cimm(1.0), f));
    QQ_TRY(field_to_ref(c, t.sp(), 0, o));
  }
  QQ_TRY(stage_out_end(c, 2, v, nv, o));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

int qq_gmresdr(qq_ctx* c, const double* phi, double* x, const int GMRES[2], double resmax,
               int itermin, const double kappa[2], int iflag, qq_defl* defl, qq_solve_info* info) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  QQ_TRY(check_iflag(iflag));
  if (!phi || !x || !GMRES || !kappa) return set_error(QQ_BAD_ARG, "null argument");
  Tmp fphi(c, P64), fx(c, P64);
  QQ_TRY(load_half(c, 1, phi, 0, fphi.sp()));
  QQ_TRY(load_half(c, 2, x, 0, fx.sp()));
  Timer t(c);
  SolveStats s;
  int status = gmresdr_fp64(c, fphi.sp(), fx.sp(), GMRES[0], GMRES[1], resmax, itermin, kappa,
                            defl ? &defl->space : nullptr, &s);
  const double sec = t.seconds();
  fill_info(info, status, s, sec);
  if (status != QQ_OK && status != QQ_NOT_CONVERGED) return status;
  QQ_TRY(store_half(c, 3, fx.sp(), 0, x));
  return status;
}

int qq_gmresproj(qq_ctx* c, const double* b, double* x, const int GMRES[2], double resmax,
                 int itermin, const double kappa[2], int iflag, const qq_defl* defl,
                 qq_solve_info* info) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  QQ_TRY(check_iflag(iflag));
  if (!b || !x || !GMRES || !kappa || !defl) return set_error(QQ_BAD_ARG, "null argument");
  Tmp fb(c, P64), fx(c, P64);
  QQ_TRY(load_half(c, 1, b, 0, fb.sp()));
  Timer t(c);
  SolveStats s;
  int status = gmresproj_fp64(c, fb.sp(), fx.sp(), GMRES[0], GMRES[1], resmax, itermin, kappa,
                              defl->space, &s);
  const double sec = t.seconds();
  fill_info(info, status, s, sec);
  if (status != QQ_OK && status != QQ_NOT_CONVERGED) return status;
  QQ_TRY(store_half(c, 3, fx.sp(), 0, x));
  return status;
}

int qq_psc(qq_ctx* c, const double* b, double* x, const int GMRES[2], double resmax, int itermin,
           const double kappa[2], int iflag, int isignal, qq_defl* defl, qq_solve_info* info) {
  if (!defl || !GMRES) return set_error(QQ_BAD_ARG, "psc needs a deflation handle");
  if (isignal == 1) return qq_gmresdr(c, b, x, GMRES, resmax, itermin, kappa, iflag, defl, info);
  if (isignal != 2) return set_error(QQ_BAD_ARG, "isignal must be 1 or 2");
  const int gp[2] = {GMRES[0] - GMRES[1], GMRES[1]};
  const double projresmax = 1.0e-8;  // Q/inverters.f90:4442
  (void)resmax;
  return qq_gmresproj(c, b, x, gp, projresmax, itermin, kappa, iflag, defl, info);
}

int qq_bicgstab(qq_ctx* c, const double* phi, double* x, double resmax, int itermin,
                const double kappa[2], int iflag, int maxiter, qq_solve_info* info) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  QQ_TRY(check_iflag(iflag));
  if (!phi || !x || !kappa) return set_error(QQ_BAD_ARG, "null argument");
  Tmp fphi(c, P64), fx(c, P64);
  QQ_TRY(load_half(c, 1, phi, 0, fphi.sp()));
  QQ_TRY(load_half(c, 2, x, 0, fx.sp()));
  Timer t(c);
  SolveStats s;
  int status = bicgstab_fp64(c, fphi.sp(), fx.sp(), resmax, itermin, maxiter, kappa, &s);
  const double sec = t.seconds();
  fill_info(info, status, s, sec);
  if (status != QQ_OK && status != QQ_NOT_CONVERGED) return status;
  QQ_TRY(store_half(c, 3, fx.sp(), 0, x));
  return status;
}

// fermprop, nkappa = -1 (Q/quark.f90:595-618 source, :645-694 dispatch,
// :787-830 reconstruction and twisted-basis rotation).
int qq_fermprop(qq_ctx* c, const double* be, const double* bo, const double kappa[2], int inverter,
                double resmax, int itermin, const int nGMRES[2], double* xe, double* xo,
                int ntmqcd, int isignal, qq_defl* defl, qq_solve_info* info) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (!be || !bo || !kappa || !xe || !xo) return set_error(QQ_BAD_ARG, "null argument");
  if (inverter != 0 && inverter != 5 && inverter != 6) return set_error(QQ_BAD_ARG, "inverter must be 0, 5 or 6");
  if ((inverter == 5 || inverter == 6) && !nGMRES) return set_error(QQ_BAD_ARG, "nGMRES needed");
  if (inverter == 6 && !defl) return set_error(QQ_BAD_ARG, "psc needs a deflation handle");
  Tmp fbe(c, P64), fbo(c, P64), src(c, P64), h(c, P64), fxe(c, P64), fxo(c, P64);
  QQ_TRY(load_half(c, 1, be, 0, fbe.sp()));
  QQ_TRY(load_half(c, 2, bo, 1, fbo.sp()));
  const double tk = 2.0 * kappa[0] * kappa[1];
  // vecsrc_o = (1 - 2 i kappa mu gamma5) b_o ; vecsrc_e = b_e/kappa^2 + H_eo vecsrc_o * fac2
  QQ_CK(launch_spinmix(c->g.vh, fbo.sp(), Spinor{nullptr, nullptr, P64}, src.sp(), 1.0, -tk, 0.0, 0.0, P64, c->st));
  QQ_TRY(op_hsingle(c, h.sp(), src.sp(), 0, 0));
  const double fac1 = 1.0 / (kappa[0] * kappa[0]);
  const double fac2 = 1.0 / (kappa[0] * (1.0 + tk * tk));
  QQ_TRY(lin(c, src.sp(), cimm(fac1), fbe.sp(), cimm(fac2), h.sp()));
  if (inverter > 3) {
    QQ_TRY(zero_field(c, fxe.sp()));
  } else {
    QQ_TRY(load_half(c, 3, xe, 0, fxe.sp()));
  }
  Timer t(c);
  SolveStats s;
  int status;
  if (inverter == 0) {
    status = bicgstab_fp64(c, src.sp(), fxe.sp(), resmax, itermin, 0, kappa, &s);
  } else if (inverter == 5 || (inverter == 6 && isignal == 1)) {
    status = gmresdr_fp64(c, src.sp(), fxe.sp(), nGMRES[0], nGMRES[1], resmax, itermin, kappa,
                          defl ? &defl->space : nullptr, &s);
  } else {
    status = gmresproj_fp64(c, src.sp(), fxe.sp(), nGMRES[0] - nGMRES[1], nGMRES[1], 1.0e-8,
                            itermin, kappa, defl->space, &s);
  }
  const double sec = t.seconds();
  fill_info(info, status, s, sec);
  if (status != QQ_OK && status != QQ_NOT_CONVERGED) return status;
  // x_o = (1 - 2 i kappa mu gamma5)(b_o + kappa H_oe x_e) / (1 + 4 kappa^2 mu^2)
  QQ_TRY(op_hsingle(c, h.sp(), fxe.sp(), 0, 1));
  const double f = 1.0 / (1.0 + tk * tk);
  QQ_CK(launch_spinmix(c->g.vh, fbo.sp(), h.sp(), fxo.sp(), f, -tk * f, f * kappa[0], -tk * f * kappa[0], P64, c->st));
  if (ntmqcd != 0 && std::fabs(kappa[1]) > 0.0001) {
    const double fac = 1.0 / std::sqrt(2.0);
    const double sgn = ntmqcd > 0 ? 1.0 : -1.0;
    Spinor none{nullptr, nullptr, P64};
    QQ_CK(launch_spinmix(c->g.vh, fxo.sp(), none, fxo.sp(), fac, sgn * fac, 0.0, 0.0, P64, c->st));
    QQ_CK(launch_spinmix(c->g.vh, fxe.sp(), none, fxe.sp(), fac, sgn * fac, 0.0, 0.0, P64, c->st));
  }
  QQ_TRY(store_half(c, 1, fxe.sp(), 0, xe));
  QQ_TRY(store_half(c, 2, fxo.sp(), 1, xo));
  return status;
}

int qq_pointsource(qq_ctx* c, double* be, double* bo, const int src[4], int icsrc, int idsrc) {
  QQ_TRY(check_ctx(c));
  if (!be || !bo || !src) return set_error(QQ_BAD_ARG, "null argument");
  if (icsrc < 1 || icsrc > 3 || idsrc < 1 || idsrc > 4) return set_error(QQ_BAD_ARG, "bad colour/spin index");
  return sources_point(c, be, bo, src, icsrc, idsrc);
}

int qq_initlagfib(int myid, int iseed) { return lagfib_init(myid, iseed); }
int qq_rnds(int m, double* rn) {
  if (m < 0 || (m > 0 && !rn)) return set_error(QQ_BAD_ARG, "bad rnds arguments");
  return lagfib_rnds(m, rn);
}
int qq_z2source(qq_ctx* c, double* be, double* bo) {
  QQ_TRY(check_ctx(c));
  if (!be || !bo) return set_error(QQ_BAD_ARG, "null argument");
  return sources_z(c, be, bo, false);
}
int qq_z4source(qq_ctx* c, double* be, double* bo) {
  QQ_TRY(check_ctx(c));
  if (!be || !bo) return set_error(QQ_BAD_ARG, "null argument");
  return sources_z(c, be, bo, true);
}

int qq_fermprop_batch(qq_ctx* c, int nrhs, const double* be, const double* bo, const double kappa[2],
                      const qq_method* method, double* xe, double* xo, qq_solve_info* infos) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (nrhs < 1 || !be || !bo || !kappa || !method || !xe || !xo) return set_error(QQ_BAD_ARG, "bad arguments");
  return batch_solve(c, nrhs, be, bo, kappa, method, xe, xo, infos);
}

int qq_twaverage_level0(qq_ctx* c, const double* be, const double* bo, const double* xe,
                        const double* xo, double kappa, double delta, int dobndry, double* J) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (!be || !bo || !xe || !xo || !J) return set_error(QQ_BAD_ARG, "null argument");
  return traces_level0(c, be, bo, xe, xo, kappa, delta, dobndry, J);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Kernel-only timing of the hopping term (see qqcd_gpu.h).
// ---------------------------------------------------------------------------
namespace {
__global__ void fill_kernel(double2* p, size_t n, unsigned seed) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned h = (unsigned)(i * 2654435761u) ^ seed;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    p[i] = make_double2((double)(h & 0xffff) / 65536.0 - 0.5, (double)(h >> 16) / 65536.0 - 0.5);
  }
}
}  // namespace

namespace qq {
int hsingle_block(qq_ctx* c, int prec, int nrhs, int shape, double* gout, const double* gin, int idag,
                  int pout);
}

extern "C" int qq_hsingle_block(qq_ctx* c, int precision, int nrhs, int shape, double* gout,
                                const double* gin, int idag, int gblclr) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  const int prec = precision == 32 ? P32 : precision == 16 ? P16 : precision == -16 ? PB16 : -1;
  if (prec < 0) return set_error(QQ_BAD_ARG, "precision must be 32, 16 or -16 (BF16)");
  if (nrhs < 1 || nrhs > kMaxBatch) return set_error(QQ_BAD_ARG, "nrhs must be 1..32");
  if (shape < 0 || shape > kShapeMax) return set_error(QQ_BAD_ARG, "bad kernel shape");
  if (gblclr != 1 && gblclr != 2) return set_error(QQ_BAD_ARG, "gblclr must be 1 or 2");
  if (idag != 0 && idag != 1) return set_error(QQ_BAD_ARG, "idag must be 0 or 1");
  if (!gout || !gin) return set_error(QQ_BAD_ARG, "null array");
  return hsingle_block(c, prec, nrhs, shape, gout, gin, idag, gblclr - 1);
}

extern "C" int qq_hop_tuned_shape(qq_ctx* c, int precision, int nrhs, int* shape) {
  QQ_TRY(check_ctx(c));
  if (!shape) return set_error(QQ_BAD_ARG, "null argument");
  const int prec = prec_of_code(precision);
  if (prec < 0 || nrhs < 1 || nrhs > kMaxBatch) return set_error(QQ_BAD_ARG, "bad precision or nrhs");
  HopArgs a;
  std::memset(&a, 0, sizeof(a));
  a.nrhs = nrhs;
  a.blk = nrhs > 1 ? 1 : 0;
  for (int epi : {EPI_STORE, EPI_TWIST, EPI_DBLE}) {  // the first hop of Hdbletm, Wilson or twisted
    auto it = c->hop_tune.find(hop_tune_key(c, a, prec, epi));
    if (it != c->hop_tune.end()) {
      *shape = it->second;
      return QQ_OK;
    }
  }
  return set_error(QQ_BAD_ARG, "no hopping launch of that kind has been tuned yet");
}

extern "C" int qq_bench_hsingle(qq_ctx* c, int precision, int nrhs, int tps, int niter,
                                int flush_l2, double* ms_per_call, double* bytes_per_call) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (!c->have_gauge) return set_error(QQ_BAD_ARG, "no gauge field uploaded");
  const int prec = prec_of_code(precision);
  if (prec < 0 || nrhs < 1 || nrhs > kMaxBatch || niter < 1 || tps < 0 || tps > kShapeMax)
    return set_error(QQ_BAD_ARG, "bad benchmark arguments");
  const int vh = c->g.vh;
  // nrhs > 1: one RHS-interleaved block field of nrhs right-hand sides (the layout of
  // the batched solver), random FP64 content converted to the target precision
  Field in, out;
  in.prec = out.prec = prec;
  QQ_CK(in.data.alloc(field_bytes(prec, vh) * nrhs));
  QQ_CK(out.data.alloc(field_bytes(prec, vh) * nrhs));
  if (has_norm(prec)) {
    QQ_CK(in.norm.alloc(sizeof(float) * vh * nrhs));
    QQ_CK(out.norm.alloc(sizeof(float) * vh * nrhs));
  }
  {
    Field t;
    t.prec = P64;
    QQ_CK(t.data.alloc(field_bytes(P64, vh) * nrhs));
    fill_kernel<<<592, 256, 0, c->st>>>(static_cast<double2*>(t.data.p), (size_t)12 * vh * nrhs, 17u);
    QQ_CK(cudaGetLastError());
    LinArgs L;
    std::memset(&L, 0, sizeof(L));
    L.vh = vh * nrhs;  // a block field is a field of vh * nrhs sites
    L.x = t.sp();
    L.y = L.z = Spinor{nullptr, nullptr, P64};
    L.out = in.sp();
    L.a = cimm(1.0);
    L.b = L.c = cimm(0.0);
    QQ_CK(launch_lincomb(L, P64, P64, P64, prec, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
  }
  DevBuf flush;
  const size_t flush_bytes = (size_t)512 << 20;
  if (flush_l2) QQ_CK(flush.alloc(flush_bytes));
  HopArgs a;
  std::memset(&a, 0, sizeof(a));
  a.g = c->g;
  a.c = make_hopcoef(c->c1, c->c2, 0);
  a.pout = 1;
  a.gauge = prec == P64 ? c->gauge64.p : c->gauge32.p;
  a.nrhs = nrhs;
  a.blk = nrhs > 1 ? 1 : 0;
  a.in[0] = in.data.p;
  a.in_norm[0] = in.norm.as<float>();
  a.out[0] = out.data.p;
  a.out_norm[0] = out.norm.as<float>();
  const int recon = prec == P64 ? c->recon64 : 12;
  if (tps == 0) {  // the autotuned choice the solvers use
    QQ_TRY(launch_hop_tuned(c, a, prec, EPI_STORE));
    tps = c->hop_tune.at(hop_tune_key(c, a, prec, EPI_STORE));
  }
  for (int w = 0; w < 3; ++w) QQ_CK(launch_hop(a, prec, recon, EPI_STORE, tps, c->st));
  double total = 0.0;
  for (int it = 0; it < niter; ++it) {
    if (flush_l2) QQ_CK(cudaMemsetAsync(flush.p, it & 0xff, flush_bytes, c->st));
    QQ_CK(cudaEventRecord(c->ev0, c->st));
    QQ_CK(launch_hop(a, prec, recon, EPI_STORE, tps, c->st));
    QQ_CK(cudaEventRecord(c->ev1, c->st));
    QQ_CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    QQ_CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    total += ms;
  }
  const double link_bytes = prec == P64 ? (recon == 18 ? 144.0 : 96.0) : 48.0;
  const double spinor_bytes = prec == P64 ? 192.0 : prec == P32 ? 96.0 : 52.0;  // 16-bit: + the norm
  if (ms_per_call) *ms_per_call = total / niter;
  if (bytes_per_call) *bytes_per_call = (double)vh * (8.0 * link_bytes + nrhs * 2.0 * spinor_bytes);
  return QQ_OK;
}

namespace qq {
int heatbath_generate(qq_ctx* c, double beta, int nsweeps, unsigned long long seed, double* u_ref,
                      double* plaq);
}

extern "C" int qq_heatbath(qq_ctx* c, double beta, int nsweeps, unsigned long long seed,
                           double* u_ref, double* plaq) {
  QQ_TRY(check_ctx(c));
  QQ_TRY(set_device(c));
  if (!(beta > 0.0) || nsweeps < 0) return set_error(QQ_BAD_ARG, "beta must be > 0, nsweeps >= 0");
  const size_t nu = (size_t)18 * c->rd.ntotal * 4 * 2 * 16;
  DevBuf own;
  double* dst = u_ref;
  if (!dst) {
    QQ_CK(own.alloc(nu * sizeof(double)));
    dst = own.as<double>();
  }
  QQ_TRY(heatbath_generate(c, beta, nsweeps, seed, dst, plaq));
  return qq_gauge_upload(c, dst, 12);
}

extern "C" int qq_ctx_stream(const qq_ctx* c, void** stream) {
  QQ_TRY(check_ctx(c));
  if (!stream) return set_error(QQ_BAD_ARG, "null argument");
  *stream = (void*)c->st;
  return QQ_OK;
}

extern "C" long long qq_launch_count(void) { return qq::launch_count(); }

extern "C" int qq_profile_hop(qq_ctx* c, int enable) {
  QQ_TRY(check_ctx(c));
  QQ_CK(cudaStreamSynchronize(c->st));
  c->prof_hop = enable != 0;
  if (c->prof_hop) c->prof_used = 0;
  return QQ_OK;
}

extern "C" int qq_profile_hop_read(qq_ctx* c, long long* launches, double* ms_total,
                                   double* bytes_total) {
  QQ_TRY(check_ctx(c));
  QQ_CK(cudaStreamSynchronize(c->st));
  double ms = 0.0, by = 0.0;
  for (size_t i = 0; i < c->prof_used; ++i) {
    float t = 0.f;
    QQ_CK(cudaEventElapsedTime(&t, c->prof_events[i].first, c->prof_events[i].second));
    ms += t;
    by += c->prof_bytes[i];
  }
  if (launches) *launches = (long long)c->prof_used;
  if (ms_total) *ms_total = ms;
  if (bytes_total) *bytes_total = by;
  return QQ_OK;
}

extern "C" int qq_profile_hop_select(qq_ctx* c, int precision, int nrhs, long long* launches, double* ms_total,
                                     double* bytes_total, double* flops_total) {
  QQ_TRY(check_ctx(c));
  QQ_CK(cudaStreamSynchronize(c->st));
  long long n = 0;
  double ms = 0.0, by = 0.0, fl = 0.0;
  for (size_t i = 0; i < c->prof_used; ++i) {
    const int p = c->prof_shape[i] / 1000, r = c->prof_shape[i] % 1000;  // storage enum, RHS
    if ((precision && p != prec_of_code(precision)) || (nrhs && r != nrhs)) continue;
    float t = 0.f;
    QQ_CK(cudaEventElapsedTime(&t, c->prof_events[i].first, c->prof_events[i].second));
    ++n;
    ms += t;
    by += c->prof_bytes[i];
    fl += 1320.0 * (double)c->g.vh * r;  // spin-projected hop: 1320 flops per output site and RHS
  }
  if (launches) *launches = n;
  if (ms_total) *ms_total = ms;
  if (bytes_total) *bytes_total = by;
  if (flops_total) *flops_total = fl;
  return QQ_OK;
}
