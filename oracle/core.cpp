// CPU oracle (test infrastructure): geometry tables, lagged-Fibonacci RNG, sources,
// the Dirac operator family and vecdot, restated from the qqcd Fortran sources.
// Parity unpinned against the Fortran (no compiler, no golden vectors): see oracle.h.
#include "oracle_impl.h"
#ifdef _OPENMP
#include <omp.h>
#endif

#include <algorithm>
#include <cmath>
#include <cstring>

using namespace oq;

// ------------------------------------------------------------------------------------
// Geometry: G/lattice.f90 siteindex (:140-294), setblk (:298-331), gblchker (:335-354)
// for a single process (ip = 0, ldiv = .false.).  basics.f90:20-31 for the sizes.
// ------------------------------------------------------------------------------------
extern "C" oq_geom* oq_geom_create(int nx, int ny, int nz, int nt, const int bc[4],
                                   const double c1[4], const double c2[4]) {
  if (nx % 4 || ny % 4 || nz % 4 || nt % 4) return nullptr;  // latdims.f90:11-13
  auto* g = new oq_geom();
  g->n[0] = nx; g->n[1] = ny; g->n[2] = nz; g->n[3] = nt;
  for (int mu = 0; mu < 4; ++mu) {
    g->bc[mu] = bc[mu];
    g->c1[mu] = c1[mu];
    g->c2[mu] = c2[mu];
  }
  const int nxyzt = nx * ny * nz * nt;
  g->nvhalf = nxyzt / 32;
  int nbmax = 0;
  for (int mu = 0; mu < 4; ++mu) nbmax = std::max(nbmax, 2 * g->nvhalf / g->n[mu]);
  g->nbmax = nbmax;
  g->ntotal = g->nvhalf + nbmax;
  const int nvhalf = g->nvhalf;
  g->lv.assign((size_t)nvhalf * 8, 0);
  g->lvbc.assign((size_t)nvhalf * 8, 0);
  g->ib.assign((size_t)nbmax * 16, 0);

  int ns[4];
  for (int mu = 0; mu < 4; ++mu) ns[mu] = g->n[mu] / 2;
  auto atoc = [&](int ia, int* ic) {  // lattice.f90 atoc :104-118
    ic[0] = ia % ns[0];
    ic[1] = (ia / ns[0]) % ns[1];
    ic[2] = (ia / (ns[0] * ns[1])) % ns[2];
    ic[3] = (ia / (ns[0] * ns[1] * ns[2])) % ns[3];
  };
  auto ctoa = [&](const int* ic) {  // lattice.f90 ctoa :122-136
    return ic[0] + ic[1] * ns[0] + ic[2] * ns[1] * ns[0] + ic[3] * ns[2] * ns[1] * ns[0];
  };
  // PART II: local site index isg().
  std::vector<int> isg(2 * nvhalf);
  int iseo[2] = {0, 0};
  for (int iv = 1; iv <= 2 * nvhalf; ++iv) {
    int is[4];
    atoc(iv - 1, is);
    int ig = is[0] + is[1] + is[2] + is[3];
    int ieo = ig % 2 + 1;
    iseo[ieo - 1] += 1;
    isg[iv - 1] = iseo[ieo - 1];
  }
  // PART III: neighbours in the +mu direction and boundary lists.
  iseo[0] = iseo[1] = 0;
  int imin[2][4] = {{0}}, imax[2][4] = {{0}};
  for (int iv = 1; iv <= 2 * nvhalf; ++iv) {
    int is[4];
    atoc(iv - 1, is);
    int ig = is[0] + is[1] + is[2] + is[3];
    int ieo = ig % 2 + 1;
    iseo[ieo - 1] += 1;
    const int me = iseo[ieo - 1];
    for (int mu = 1; mu <= 4; ++mu) {
      if (bc[mu - 1] != 1) {  // single process, non-periodic fermion boundary
        if (is[mu - 1] < ns[mu - 1] - 1) {
          int save = is[mu - 1];
          is[mu - 1] += 1;
          int k = ctoa(is);
          g->LV(me, mu, ieo) = isg[k];
          g->LVBC(me, mu, ieo) = isg[k];
          is[mu - 1] = save;
        } else {
          int save = is[mu - 1];
          is[mu - 1] = 0;
          int k = ctoa(is);
          g->LV(me, mu, ieo) = isg[k];
          is[mu - 1] = save;
          imax[ieo - 1][mu - 1] += 1;
          g->LVBC(me, mu, ieo) = nvhalf + imax[ieo - 1][mu - 1];
          g->IB(imax[ieo - 1][mu - 1], mu, 2, ieo) = me;
        }
        if (is[mu - 1] == 0) {
          imin[ieo - 1][mu - 1] += 1;
          g->IB(imin[ieo - 1][mu - 1], mu, 1, ieo) = me;
        }
      } else {  // single process, periodic
        int save = is[mu - 1];
        is[mu - 1] = (is[mu - 1] + 1) % ns[mu - 1];
        int k = ctoa(is);
        g->LV(me, mu, ieo) = isg[k];
        g->LVBC(me, mu, ieo) = isg[k];
        is[mu - 1] = save;
      }
    }
  }
  for (int mu = 0; mu < 4; ++mu) g->nms[mu] = nvhalf / ns[mu];  // PART IV
  // setblk
  int ib0 = 0;
  for (int ibt = 1; ibt <= 2; ++ibt)
    for (int ibz = 1; ibz <= 2; ++ibz)
      for (int iby = 1; iby <= 2; ++iby)
        for (int ibx = 1; ibx <= 2; ++ibx) {
          ib0 += 1;
          g->lbd[ib0 - 1][0] = ibx == 1;
          g->lbd[ib0 - 1][1] = iby == 1;
          g->lbd[ib0 - 1][2] = ibz == 1;
          g->lbd[ib0 - 1][3] = ibt == 1;
          g->iblv[ib0 - 1][0] = ib0 + 3 - 2 * ibx;
          g->iblv[ib0 - 1][1] = ib0 + 2 * (3 - 2 * iby);
          g->iblv[ib0 - 1][2] = ib0 + 4 * (3 - 2 * ibz);
          g->iblv[ib0 - 1][3] = ib0 + 8 * (3 - 2 * ibt);
        }
  // gblchker
  static const int vb1[8] = {1, 4, 6, 7, 10, 11, 13, 16};
  static const int vb2[8] = {2, 3, 5, 8, 9, 12, 14, 15};
  static const int vi1[16] = {1, 2, 2, 1, 2, 1, 1, 2, 2, 1, 1, 2, 1, 2, 2, 1};
  static const int vi2[16] = {1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8};
  for (int i = 0; i < 8; ++i) {
    g->vecbl[0][i] = vb1[i];
    g->vecbl[1][i] = vb2[i];
  }
  for (int i = 0; i < 16; ++i) {
    g->vecblinv[0][i] = vi1[i];
    g->vecblinv[1][i] = vi2[i];
  }
  return g;
}

extern "C" void oq_geom_destroy(oq_geom* g) { delete g; }
extern "C" int oq_nvhalf(const oq_geom* g) { return g->nvhalf; }
extern "C" int oq_ntotal(const oq_geom* g) { return g->ntotal; }
extern "C" int oq_nbmax(const oq_geom* g) { return g->nbmax; }
extern "C" void oq_set_coact(oq_geom* g, const double c1[4], const double c2[4]) {
  for (int mu = 0; mu < 4; ++mu) {
    g->c1[mu] = c1[mu];
    g->c2[mu] = c2[mu];
  }
}

extern "C" void oq_tables(const oq_geom* g, int* lv, int* lvbc, int* ib, int* nms,
                          int* lbd, int* iblv, int* vecbl, int* vecblinv) {
  const int nvhalf = g->nvhalf;
  if (lv) std::memcpy(lv, g->lv.data(), sizeof(int) * nvhalf * 8);
  if (lvbc) std::memcpy(lvbc, g->lvbc.data(), sizeof(int) * nvhalf * 8);
  if (ib) std::memcpy(ib, g->ib.data(), sizeof(int) * g->nbmax * 16);
  if (nms)
    for (int mu = 0; mu < 4; ++mu) nms[mu] = g->nms[mu];
  for (int mu = 0; mu < 4; ++mu)
    for (int b = 0; b < 16; ++b) {
      if (lbd) lbd[b + 16 * mu] = g->lbd[b][mu] ? 1 : 0;
      if (iblv) iblv[b + 16 * mu] = g->iblv[b][mu];
    }
  for (int i = 0; i < 8; ++i)
    for (int c = 0; c < 2; ++c)
      if (vecbl) vecbl[c + 2 * i] = g->vecbl[c][i];
  for (int i = 0; i < 16; ++i)
    for (int c = 0; c < 2; ++c)
      if (vecblinv) vecblinv[c + 2 * i] = g->vecblinv[c][i];
}

// Q/quark.f90:70-105 (pointsource) with src = x + 1.
extern "C" void oq_site_of_coords(const oq_geom* g, const int x[4], int* isite, int* ieo,
                                  int* ibl, int* gblclr, int* ibleo) {
  int srcbit[4];
  for (int mu = 0; mu < 4; ++mu) srcbit[mu] = x[mu] + 1;
  const int nx = g->n[0], ny = g->n[1], nz = g->n[2];
  int intx = (srcbit[0] - 1) / 4, inty = (srcbit[1] - 1) / 2, intz = (srcbit[2] - 1) / 2,
      intt = (srcbit[3] - 1) / 2;
  *isite = 1 + intx + inty * nx / 4 + intz * nx * ny / 8 + intt * nx * ny * nz / 16;
  int e = 1, b = 1;
  for (int mu = 0; mu < 4; ++mu) {
    if (srcbit[mu] % 4 == 3 || srcbit[mu] % 4 == 0) e = 3 - e;
    if (srcbit[mu] % 2 == 0) b = g->iblv[b - 1][mu];
  }
  *ieo = e;
  *ibl = b;
  *gblclr = g->vecblinv[0][b - 1];
  *ibleo = g->vecblinv[1][b - 1];
}

// ------------------------------------------------------------------------------------
// Lagged Fibonacci generator: G/lagfib.f90 initlagfib :80-92, initbirep :96-146,
// bigdelay :150-215, rnds :219-259.  Integer arithmetic is the reference's 32-bit
// signed (two's complement wrap), ishft is a logical shift.
// ------------------------------------------------------------------------------------
namespace {
constexpr int IP = 521, IQ = 32;
int32_t iwlagfib[IP];
int jrlagfib = 0, krlagfib = 0;

inline int32_t lshr(int32_t v, int s) { return (int32_t)((uint32_t)v >> s); }

void initbirep() {
  int32_t ib[IP];
  uint32_t ix = 1;
  for (int i = 0; i < IP; ++i) {
    ix = ix * 69069u;
    ib[i] = lshr((int32_t)ix, 31);
  }
  jrlagfib = 0;
  krlagfib = IP - IQ;
  for (int j = 0; j < IP; ++j) {
    uint32_t iwork = 0;
    for (int i = 0; i < 32; ++i) {
      iwork = 2u * iwork + (uint32_t)ib[jrlagfib];
      ib[jrlagfib] = ib[jrlagfib] ^ ib[krlagfib];
      jrlagfib += 1;
      if (jrlagfib == IP) jrlagfib = 0;
      krlagfib += 1;
      if (krlagfib == IP) krlagfib = 0;
    }
    iwlagfib[j] = lshr((int32_t)iwork, 1);
  }
}

void bigdelay(int ndelay) {
  const int mu = 40;
  std::vector<int32_t> iwk(2 * IP - 1);
  std::vector<int32_t> c(2 * IP);
  std::vector<int32_t> ib(IP + 32);
  for (int i = 0; i < IP; ++i) iwk[i] = iwlagfib[i];
  for (int i = IP; i <= 2 * IP - 2; ++i) iwk[i] = iwk[i - IP] ^ iwk[i - IQ];
  for (int i = 0; i < mu; ++i) ib[i] = 0;
  int m = ndelay;
  int nb = mu - 1;
  while (m > IP - 1) {
    nb += 1;
    ib[nb] = m % 2;
    m = m / 2;
  }
  for (int i = 0; i < IP; ++i) c[i] = 0;
  c[m] = 1;
  for (int j = nb; j >= 0; --j) {
    for (int i = IP - 1; i >= 0; --i) {
      c[2 * i + ib[j]] = c[i];
      c[2 * i + 1 - ib[j]] = 0;
    }
    for (int i = 2 * IP - 1; i >= IP; --i) {
      c[i - IP] = c[i - IP] ^ c[i];
      c[i - IQ] = c[i - IQ] ^ c[i];
    }
  }
  for (int j = 0; j < IP; ++j) {
    int32_t iwork = 0;
    for (int i = 0; i < IP; ++i) iwork = iwork ^ (int32_t)((uint32_t)c[i] * (uint32_t)iwk[j + i]);
    iwlagfib[j] = iwork;
  }
}
}  // namespace

extern "C" void oq_initlagfib(int myid, int iseed) {
  initbirep();
  bigdelay(myid + iseed);
}

extern "C" void oq_rnds(int m, double* rn) {
  // fnorm is a default-real (single precision) literal promoted into the product.
  const double fnorm = (double)0.465661e-9f;
  for (int i = 0; i < m; ++i) {
    for (;;) {
      iwlagfib[jrlagfib] = iwlagfib[jrlagfib] ^ iwlagfib[krlagfib];
      rn[i] = (double)iwlagfib[jrlagfib] * fnorm;
      if (rn[i] != 0.0) break;
    }
    jrlagfib += 1;
    if (jrlagfib >= IP) jrlagfib -= IP;
    krlagfib += 1;
    if (krlagfib >= IP) krlagfib -= IP;
  }
}

extern "C" void oq_lagfib_state(int* iw, int* jr, int* kr) {
  for (int i = 0; i < IP; ++i) iw[i] = iwlagfib[i];
  *jr = jrlagfib;
  *kr = krlagfib;
}
extern "C" void oq_lagfib_set_state(const int* iw, int jr, int kr) {
  for (int i = 0; i < IP; ++i) iwlagfib[i] = iw[i];
  jrlagfib = jr;
  krlagfib = kr;
}

// ------------------------------------------------------------------------------------
// Sources: Q/quark.f90:46-108 pointsource; Q/disconloops.f90:4518-4570 z4source
// (the active branch), :4583-4649 z2source.
// ------------------------------------------------------------------------------------
extern "C" void oq_pointsource(const oq_geom* g, double* be, double* bo, const int src[4],
                               int icsrc, int idsrc) {
  const size_t nv = g->vsize();
  std::fill(be, be + nv, 0.0);
  std::fill(bo, bo + nv, 0.0);
  int x[4];
  for (int mu = 0; mu < 4; ++mu) x[mu] = src[mu] - 1;
  int isite, ieo, ibl, gblclr, ibleo;
  oq_site_of_coords(g, x, &isite, &ieo, &ibl, &gblclr, &ibleo);
  if (gblclr == 1)
    be[g->gi(2 * icsrc - 1, isite, idsrc, ieo, ibleo)] = 1.0;
  else
    bo[g->gi(2 * icsrc - 1, isite, idsrc, ieo, ibleo)] = 1.0;
}

static void noise_half(const oq_geom* g, double* b, bool z4) {
  const int nvhalf = g->nvhalf;
  std::fill(b, b + g->vsize(), 0.0);
  std::vector<double> rn((size_t)192 * nvhalf);
  oq_rnds(192 * nvhalf, rn.data());
  size_t icount = 0;
  for (int ic = 1; ic <= 3; ++ic) {
    int icri = 2 * ic - 1;
    for (int isite = 1; isite <= nvhalf; ++isite)
      for (int id = 1; id <= 4; ++id)
        for (int ieo = 1; ieo <= 2; ++ieo)
          for (int ibl = 1; ibl <= 8; ++ibl) {
            double r = rn[icount++];
            if (z4) {
              if (r > 0.75)
                b[g->gi(icri, isite, id, ieo, ibl)] = 1.0;
              else if (0.5 < r && r < 0.75)
                b[g->gi(icri, isite, id, ieo, ibl)] = -1.0;
              else if (0.25 < r && r < 0.5)
                b[g->gi(icri + 1, isite, id, ieo, ibl)] = 1.0;
              else
                b[g->gi(icri + 1, isite, id, ieo, ibl)] = -1.0;
            } else {
              b[g->gi(icri, isite, id, ieo, ibl)] = r > 0.5 ? 1.0 : -1.0;
            }
          }
  }
}

extern "C" void oq_z2source(const oq_geom* g, double* be, double* bo) {
  noise_half(g, be, false);
  noise_half(g, bo, false);
}
extern "C" void oq_z4source(const oq_geom* g, double* be, double* bo) {
  noise_half(g, be, true);
  noise_half(g, bo, true);
}

// ------------------------------------------------------------------------------------
// Dirac operator: Q/diracops.f90 Hsingle :554-599, mulbac :950-1159,
// mulfor :1163-1391, setmvf :1395-1437, mv/mdv/mvg/mdvg :1441-1637,
// setvector :1641-1697, slidevector :1701-1747 (single process: the send/receive is
// absent, only the local copy and the boundary sign remain).
// ------------------------------------------------------------------------------------
namespace {

// w(i) = y(i) * v(j(i)) ; j == nullptr means j(i) = i  (mv / mvg)
inline void mvg(int n, const double* y, const double* v, double* w, const int* j) {
  OQ_PAR_FOR
  for (int i = 0; i < n; ++i) {
    const double* Y = y + 18 * (size_t)i;
    const double* V = v + 6 * (size_t)(j ? j[i] - 1 : i);
    double* W = w + 6 * (size_t)i;
    W[0] = Y[0] * V[0] - Y[1] * V[1] + Y[2] * V[2] - Y[3] * V[3] + Y[4] * V[4] - Y[5] * V[5];
    W[1] = Y[0] * V[1] + Y[1] * V[0] + Y[2] * V[3] + Y[3] * V[2] + Y[4] * V[5] + Y[5] * V[4];
    W[2] = Y[6] * V[0] - Y[7] * V[1] + Y[8] * V[2] - Y[9] * V[3] + Y[10] * V[4] - Y[11] * V[5];
    W[3] = Y[6] * V[1] + Y[7] * V[0] + Y[8] * V[3] + Y[9] * V[2] + Y[10] * V[5] + Y[11] * V[4];
    W[4] = Y[12] * V[0] - Y[13] * V[1] + Y[14] * V[2] - Y[15] * V[3] + Y[16] * V[4] - Y[17] * V[5];
    W[5] = Y[12] * V[1] + Y[13] * V[0] + Y[14] * V[3] + Y[15] * V[2] + Y[16] * V[5] + Y[17] * V[4];
  }
}

// w(i) = y(i)^dagger * v(i)  (mdv)
inline void mdv(int n, const double* y, const double* v, double* w) {
  OQ_PAR_FOR
  for (int i = 0; i < n; ++i) {
    const double* Y = y + 18 * (size_t)i;
    const double* V = v + 6 * (size_t)i;
    double* W = w + 6 * (size_t)i;
    W[0] = Y[0] * V[0] + Y[1] * V[1] + Y[6] * V[2] + Y[7] * V[3] + Y[12] * V[4] + Y[13] * V[5];
    W[1] = Y[0] * V[1] - Y[1] * V[0] + Y[6] * V[3] - Y[7] * V[2] + Y[12] * V[5] - Y[13] * V[4];
    W[2] = Y[2] * V[0] + Y[3] * V[1] + Y[8] * V[2] + Y[9] * V[3] + Y[14] * V[4] + Y[15] * V[5];
    W[3] = Y[2] * V[1] - Y[3] * V[0] + Y[8] * V[3] - Y[9] * V[2] + Y[14] * V[5] - Y[15] * V[4];
    W[4] = Y[4] * V[0] + Y[5] * V[1] + Y[10] * V[2] + Y[11] * V[3] + Y[16] * V[4] + Y[17] * V[5];
    W[5] = Y[4] * V[1] - Y[5] * V[0] + Y[10] * V[3] - Y[11] * V[2] + Y[16] * V[5] - Y[17] * V[4];
  }
}

// Accumulate h += [c1 -/+ c2 gamma_mu] wx, in the reference's term order.
// sgn = -1 : c1 - c2*gamma_mu ; sgn = +1 : c1 + c2*gamma_mu.
void accumulate(const oq_geom* g, double* h, const double* wx, int ldw, int mu, int sgn,
                int ieo, int ibleo) {
  const int nvhalf = g->nvhalf;
  const double c1 = g->c1[mu - 1], c2 = g->c2[mu - 1];
  double* h1 = h + g->gi(1, 1, 1, ieo, ibleo);
  double* h2 = h + g->gi(1, 1, 2, ieo, ibleo);
  double* h3 = h + g->gi(1, 1, 3, ieo, ibleo);
  double* h4 = h + g->gi(1, 1, 4, ieo, ibleo);
  const double* w1 = wx;
  const double* w2 = wx + (size_t)6 * ldw;
  const double* w3 = wx + (size_t)12 * ldw;
  const double* w4 = wx + (size_t)18 * ldw;
  // s = +1 means the "minus gamma" form of the reference (c1 - c2 gamma).
  const bool minus = sgn < 0;
  switch (mu) {
    case 1:
      OQ_PAR_FOR
      for (int i = 0; i < nvhalf; ++i)
        for (int ir = 0; ir < 6; ++ir) {
          size_t k = 6 * (size_t)i + ir;
          if (minus) {
            h1[k] = h1[k] + c1 * w1[k] - c2 * w4[k];
            h2[k] = h2[k] + c1 * w2[k] - c2 * w3[k];
            h3[k] = h3[k] + c1 * w3[k] - c2 * w2[k];
            h4[k] = h4[k] + c1 * w4[k] - c2 * w1[k];
          } else {
            h1[k] = h1[k] + c1 * w1[k] + c2 * w4[k];
            h2[k] = h2[k] + c1 * w2[k] + c2 * w3[k];
            h3[k] = h3[k] + c1 * w3[k] + c2 * w2[k];
            h4[k] = h4[k] + c1 * w4[k] + c2 * w1[k];
          }
        }
      break;
    case 2:
      OQ_PAR_FOR
      for (int i = 0; i < nvhalf; ++i)
        for (int ir = 0; ir < 6; ir += 2) {
          size_t k = 6 * (size_t)i + ir;
          if (minus) {
            h1[k] = h1[k] + c1 * w1[k] - c2 * w4[k + 1];
            h1[k + 1] = h1[k + 1] + c1 * w1[k + 1] + c2 * w4[k];
            h2[k] = h2[k] + c1 * w2[k] + c2 * w3[k + 1];
            h2[k + 1] = h2[k + 1] + c1 * w2[k + 1] - c2 * w3[k];
            h3[k] = h3[k] + c1 * w3[k] - c2 * w2[k + 1];
            h3[k + 1] = h3[k + 1] + c1 * w3[k + 1] + c2 * w2[k];
            h4[k] = h4[k] + c1 * w4[k] + c2 * w1[k + 1];
            h4[k + 1] = h4[k + 1] + c1 * w4[k + 1] - c2 * w1[k];
          } else {
            h1[k] = h1[k] + c1 * w1[k] + c2 * w4[k + 1];
            h1[k + 1] = h1[k + 1] + c1 * w1[k + 1] - c2 * w4[k];
            h2[k] = h2[k] + c1 * w2[k] - c2 * w3[k + 1];
            h2[k + 1] = h2[k + 1] + c1 * w2[k + 1] + c2 * w3[k];
            h3[k] = h3[k] + c1 * w3[k] + c2 * w2[k + 1];
            h3[k + 1] = h3[k + 1] + c1 * w3[k + 1] - c2 * w2[k];
            h4[k] = h4[k] + c1 * w4[k] - c2 * w1[k + 1];
            h4[k + 1] = h4[k + 1] + c1 * w4[k + 1] + c2 * w1[k];
          }
        }
      break;
    case 3:
      OQ_PAR_FOR
      for (int i = 0; i < nvhalf; ++i)
        for (int ir = 0; ir < 6; ++ir) {
          size_t k = 6 * (size_t)i + ir;
          if (minus) {
            h1[k] = h1[k] + c1 * w1[k] - c2 * w3[k];
            h2[k] = h2[k] + c1 * w2[k] + c2 * w4[k];
            h3[k] = h3[k] + c1 * w3[k] - c2 * w1[k];
            h4[k] = h4[k] + c1 * w4[k] + c2 * w2[k];
          } else {
            h1[k] = h1[k] + c1 * w1[k] + c2 * w3[k];
            h2[k] = h2[k] + c1 * w2[k] - c2 * w4[k];
            h3[k] = h3[k] + c1 * w3[k] + c2 * w1[k];
            h4[k] = h4[k] + c1 * w4[k] - c2 * w2[k];
          }
        }
      break;
    case 4:
      OQ_PAR_FOR
      for (int i = 0; i < nvhalf; ++i)
        for (int ir = 0; ir < 6; ++ir) {
          size_t k = 6 * (size_t)i + ir;
          if (minus) {
            h1[k] = h1[k] + (c1 - c2) * w1[k];
            h2[k] = h2[k] + (c1 - c2) * w2[k];
            h3[k] = h3[k] + (c1 + c2) * w3[k];
            h4[k] = h4[k] + (c1 + c2) * w4[k];
          } else {
            h1[k] = h1[k] + (c1 + c2) * w1[k];
            h2[k] = h2[k] + (c1 + c2) * w2[k];
            h3[k] = h3[k] + (c1 - c2) * w3[k];
            h4[k] = h4[k] + (c1 - c2) * w4[k];
          }
        }
      break;
  }
}

// mulbac: h(x) += (c1 -/+ c2 gamma_mu) U_mu(x) g(x+mu)
void mulbac(const oq_geom* g, double* h, const double* u, double* gin, int mu, int idag,
            int gblclr, std::vector<double>& wx) {
  const int nvhalf = g->nvhalf;
  wx.resize((size_t)24 * nvhalf);
  for (int ieo = 1; ieo <= 2; ++ieo) {
    const int jeo = 3 - ieo;
    for (int ibleo = 1; ibleo <= 8; ++ibleo) {
      const int ibl = g->vecbl[gblclr - 1][ibleo - 1];
      const int jbl = g->iblv[ibl - 1][mu - 1];
      const int jbleo = g->vecblinv[1][jbl - 1];
      const double* a = u + g->ui(1, 1, mu, ieo, ibl);
      for (int id = 1; id <= 4; ++id) {
        double* c = wx.data() + (size_t)6 * nvhalf * (id - 1);
        if (g->lbd[ibl - 1][mu - 1]) {
          mvg(nvhalf, a, gin + g->gi(1, 1, id, ieo, jbleo), c, nullptr);
        } else {
          double* b = gin + g->gi(1, 1, id, jeo, jbleo);
          if (g->bc[mu - 1] != 1) {  // setvector
            const double fbc = (double)g->bc[mu - 1];
            for (int i = 1; i <= g->nms[mu - 1]; ++i) {
              const int src = g->IB(i, mu, 1, jeo);
              for (int a6 = 0; a6 < 6; ++a6)
                b[6 * (size_t)(nvhalf + i - 1) + a6] = b[6 * (size_t)(src - 1) + a6];
            }
            for (int i = 1; i <= g->nms[mu - 1]; ++i)
              for (int a6 = 0; a6 < 6; ++a6)
                b[6 * (size_t)(nvhalf + i - 1) + a6] = fbc * b[6 * (size_t)(nvhalf + i - 1) + a6];
          }
          mvg(nvhalf, a, b, c, &g->LVBC(1, mu, ieo));
        }
      }
      accumulate(g, h, wx.data(), nvhalf, mu, idag == 0 ? -1 : +1, ieo, ibleo);
    }
  }
}

// mulfor: h(x) += (c1 +/- c2 gamma_mu) U_mu^dagger(x-mu) g(x-mu)
void mulfor(const oq_geom* g, double* h, const double* u, const double* gin, int mu,
            int idag, int gblclr, std::vector<double>& wx, std::vector<double>& wy) {
  const int nvhalf = g->nvhalf, ntotal = g->ntotal;
  wx.resize((size_t)24 * ntotal);
  wy.resize((size_t)6 * nvhalf);
  for (int ieo = 1; ieo <= 2; ++ieo) {
    for (int ibleo = 1; ibleo <= 8; ++ibleo) {
      const int ibl = g->vecbl[gblclr - 1][ibleo - 1];
      const int jbl = g->iblv[ibl - 1][mu - 1];
      const int jbleo = g->vecblinv[1][jbl - 1];
      const int jeo = g->lbd[jbl - 1][mu - 1] ? ieo : 3 - ieo;
      for (int id = 1; id <= 4; ++id) {
        double* w = wx.data() + (size_t)6 * ntotal * (id - 1);
        mdv(nvhalf, u + g->ui(1, 1, mu, jeo, jbl), gin + g->gi(1, 1, id, jeo, jbleo),
            wy.data());
        if (g->lbd[jbl - 1][mu - 1]) {
          std::memcpy(w, wy.data(), sizeof(double) * 6 * nvhalf);
        } else {
          OQ_PAR_FOR
          for (int j = 1; j <= nvhalf; ++j) {
            const int t = g->LVBC(j, mu, jeo);
            for (int a6 = 0; a6 < 6; ++a6)
              w[6 * (size_t)(t - 1) + a6] = wy[6 * (size_t)(j - 1) + a6];
          }
          if (g->bc[mu - 1] != 1) {  // slidevector
            const double fbc = (double)g->bc[mu - 1];
            for (int i = 1; i <= g->nms[mu - 1]; ++i)
              for (int a6 = 0; a6 < 6; ++a6)
                w[6 * (size_t)(nvhalf + i - 1) + a6] = fbc * w[6 * (size_t)(nvhalf + i - 1) + a6];
            for (int i = 1; i <= g->nms[mu - 1]; ++i) {
              const int dst = g->IB(i, mu, 1, ieo);
              for (int a6 = 0; a6 < 6; ++a6)
                w[6 * (size_t)(dst - 1) + a6] = w[6 * (size_t)(nvhalf + i - 1) + a6];
            }
          }
        }
      }
      accumulate(g, h, wx.data(), ntotal, mu, idag == 0 ? +1 : -1, ieo, ibleo);
    }
  }
}
}  // namespace

namespace oq {
void hsingle(const oq_geom* g, double* gout, const double* u, double* gin, int idag,
             int gblclr) {
  std::vector<double> wx, wy;
  std::fill(gout, gout + g->vsize(), 0.0);
  for (int mu = 1; mu <= 4; ++mu) {
    mulbac(g, gout, u, gin, mu, idag, gblclr, wx);
    mulfor(g, gout, u, gin, mu, idag, gblclr, wx, wy);
  }
}

// Hdouble Q/diracops.f90:264-346
void hdouble(const oq_geom* g, double* he, const double* u, double* ge, int idag,
             double kappa) {
  std::vector<double> htmp(g->vsize());
  hsingle(g, htmp.data(), u, ge, idag, 2);
  hsingle(g, he, u, htmp.data(), idag, 1);
  const double fac1 = 1.0 / (kappa * kappa);
  g->for_interior([&](size_t k) { he[k] = fac1 * ge[k] - he[k]; });
}

// Hdbletm Q/diracops.f90:435-550 (Wilson branch, iflag = -1)
void hdbletm(const oq_geom* g, double* he, const double* u, double* ge, int idag,
             const double kappa[2]) {
  if (kappa[1] < 0.00000001) {
    hdouble(g, he, u, ge, idag, kappa[0]);
    return;
  }
  std::vector<double> htmp(g->vsize(), 0.0);
  hsingle(g, he, u, ge, idag, 2);
  double fac1 = 2.0 * kappa[0] * kappa[1];
  g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
    htmp[s1] = he[s1] - fac1 * he[s3];
    htmp[s2] = he[s2] - fac1 * he[s4];
    htmp[s3] = he[s3] + fac1 * he[s1];
    htmp[s4] = he[s4] + fac1 * he[s2];
  });
  hsingle(g, he, u, htmp.data(), idag, 1);
  fac1 = 1.0 / (kappa[0] * kappa[0]);
  const double fac2 = 2.0 * kappa[1] / kappa[0];
  const double t = 2.0 * kappa[0] * kappa[1];
  const double fac3 = 1.0 / (1.0 + t * t);
  g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
    const double g1 = ge[s1], g2 = ge[s2], g3 = ge[s3], g4 = ge[s4];
    he[s1] = fac1 * g1 + fac2 * g3 - fac3 * he[s1];
    he[s2] = fac1 * g2 + fac2 * g4 - fac3 * he[s2];
    he[s3] = fac1 * g3 - fac2 * g1 - fac3 * he[s3];
    he[s4] = fac1 * g4 - fac2 * g2 - fac3 * he[s4];
  });
}

double vecdot_re(const oq_geom* g, const double* a, const double* b, double* im) {
  double adb[2];
  oq_vecdot(g, a, b, adb);
  if (im) *im = adb[1];
  return adb[0];
}
}  // namespace oq

extern "C" void oq_hsingle(const oq_geom* g, double* gout, const double* u, double* gin,
                           int idag, int gblclr) {
  oq::hsingle(g, gout, u, gin, idag, gblclr);
}
extern "C" void oq_hdouble(const oq_geom* g, double* he, const double* u, double* ge,
                           int idag, double kappa) {
  oq::hdouble(g, he, u, ge, idag, kappa);
}
extern "C" void oq_hdbletm(const oq_geom* g, double* he, const double* u, double* ge,
                           int idag, const double kappa[2]) {
  oq::hdbletm(g, he, u, ge, idag, kappa);
}

// twMshift Q/diracops.f90:1863-1995 (iflag = -1): full twisted operator on
// gwhole(...,1:2); output hwhole(...,1:2).  Each half has g->vsize() doubles.
extern "C" void oq_twmshift(const oq_geom* g, double* hwhole, const double* u,
                            double* gwhole, int idag, const double kappa[2]) {
  const size_t nv = g->vsize();
  std::vector<double> hx(nv), htmp(nv, 0.0);
  const double basekappa = kappa[0], basemu = kappa[1];
  const double fac1 = 1.0 / (2.0 * basemu);
  const double fac2 = 1.0 / (2.0 * basekappa * basemu);
  for (int half = 0; half < 2; ++half) {
    double* gin = gwhole + (half == 0 ? nv : 0);       // other half
    const double* gsame = gwhole + (half == 0 ? 0 : nv);
    double* hout = hwhole + (half == 0 ? 0 : nv);
    oq::hsingle(g, hx.data(), u, gin, idag, half == 0 ? 1 : 2);
    g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
      htmp[s1] = -fac1 * hx[s3];
      htmp[s2] = -fac1 * hx[s4];
      htmp[s3] = fac1 * hx[s1];
      htmp[s4] = fac1 * hx[s2];
    });
    g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
      hout[s1] = gsame[s1] - fac2 * gsame[s3] + htmp[s1];
      hout[s2] = gsame[s2] - fac2 * gsame[s4] + htmp[s2];
      hout[s3] = gsame[s3] + fac2 * gsame[s1] + htmp[s3];
      hout[s4] = gsame[s4] + fac2 * gsame[s2] + htmp[s4];
    });
  }
}

// gamma5mult Q/diracops.f90:1750-1860 (iflag = -1): the even-odd twisted operator
// multiplied by -i gamma5 / (2 kappa mu),
//   he = ge/kappa^2 + fac4 J'[ ge/kappa^2 - fac3 H_eo (1 - 2 i kappa mu gamma5) H_oe ge ],
// with J'(v) = (-v3, -v4, v1, v2), fac3 = 1/(1 + 4 kappa^2 mu^2), fac4 = 1/(2 kappa mu),
// in the reference's expression order.
namespace oq {
void gamma5mult(const oq_geom* g, double* he, const double* u, double* ge, int idag,
                const double kappa[2]) {
  const size_t nv = g->vsize();
  std::vector<double> hx(nv, 0.0), htmp(nv, 0.0);
  const double basekappa = kappa[0], basemu = kappa[1];
  oq::hsingle(g, hx.data(), u, ge, idag, 2);
  const double f = 2.0 * basekappa * basemu;
  g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
    htmp[s1] = hx[s1] - f * hx[s3];
    htmp[s2] = hx[s2] - f * hx[s4];
    htmp[s3] = hx[s3] + f * hx[s1];
    htmp[s4] = hx[s4] + f * hx[s2];
  });
  oq::hsingle(g, hx.data(), u, htmp.data(), idag, 1);
  const double fac1 = 1.0 / (basekappa * basekappa);
  const double fac3 = 1.0 / (1.0 + (2.0 * basekappa * basemu) * (2.0 * basekappa * basemu));
  const double fac4 = 1.0 / (2.0 * basekappa * basemu);
  g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
    const double h1 = hx[s1], h2 = hx[s2], h3 = hx[s3], h4 = hx[s4];
    he[s1] = -fac4 * fac1 * ge[s3] + fac1 * ge[s1] + fac4 * fac3 * h3;
    he[s2] = -fac4 * fac1 * ge[s4] + fac1 * ge[s2] + fac4 * fac3 * h4;
    he[s3] = fac4 * fac1 * ge[s1] + fac1 * ge[s3] - fac4 * fac3 * h1;
    he[s4] = fac4 * fac1 * ge[s2] + fac1 * ge[s4] - fac4 * fac3 * h2;
  });
}
}  // namespace oq

extern "C" void oq_gamma5mult(const oq_geom* g, double* he, const double* u, double* ge,
                              int idag, const double kappa[2]) {
  oq::gamma5mult(g, he, u, ge, idag, kappa);
}

// gam5x C/basics.f90:408-454
extern "C" void oq_gam5x(const oq_geom* g, double* a) {
  std::vector<double> b(a, a + g->vsize());
  g->for_spin_interior([&](size_t s1, size_t s2, size_t s3, size_t s4) {
    // s* index the real part of one colour component; +1 is the imaginary part.
    a[s1] = b[s3 + 1];
    a[s1 + 1] = -b[s3];
    a[s2] = b[s4 + 1];
    a[s2 + 1] = -b[s4];
    a[s3] = -b[s1 + 1];
    a[s3 + 1] = b[s1];
    a[s4] = -b[s2 + 1];
    a[s4 + 1] = b[s2];
  }, /*complex_stride=*/true);
}

// gamma5vector Q/quark.f90:3484-3548 (twisted-basis rotation), loops over ntotal sites.
extern "C" void oq_gamma5vector(const oq_geom* g, double* a, int ntmqcd) {
  const double fac = 1.0 / std::sqrt(2.0);
  if (ntmqcd == 0) return;
  const double sgn = ntmqcd > 0 ? 1.0 : -1.0;
  g->for_spin_all([&](size_t s1, size_t s2, size_t s3, size_t s4) {
    const double t1 = a[s1], t2 = a[s2];
    a[s1] = a[s1] + sgn * a[s3];
    a[s2] = a[s2] + sgn * a[s4];
    a[s3] = a[s3] - sgn * t1;
    a[s4] = a[s4] - sgn * t2;
  });
  const size_t nv = g->vsize();
  for (size_t k = 0; k < nv; ++k) a[k] = fac * a[k];
}

// vecdot Q/inverters.f90:13485-13530
// Host threads of the timing build (liboracle_omp.so); the default build is serial and
// ignores it.
extern "C" void oq_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
extern "C" int oq_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

extern "C" void oq_vecdot(const oq_geom* g, const double* a, const double* b, double* adb) {
  double re = 0.0, im = 0.0;
  OQ_PAR_SUM3
  for (int ibleo = 1; ibleo <= 8; ++ibleo)
    for (int ieo = 1; ieo <= 2; ++ieo)
      for (int id = 1; id <= 4; ++id)
        for (int isite = 1; isite <= g->nvhalf; ++isite) {
          const double* A = a + g->gi(1, isite, id, ieo, ibleo);
          const double* B = b + g->gi(1, isite, id, ieo, ibleo);
          re = re + (A[0] * B[0] + A[1] * B[1] + A[2] * B[2] + A[3] * B[3] + A[4] * B[4] +
                     A[5] * B[5]);
          im = im + (A[0] * B[1] - A[1] * B[0] + A[2] * B[3] - A[3] * B[2] + A[4] * B[5] -
                     A[5] * B[4]);
        }
  adb[0] = re;
  adb[1] = im;
}

// ------------------------------------------------------------------------------------
// Gauge helpers: cold start (all links = identity) and the average plaquette
// (G/gaugetools.f90 aveplaq :1436-1474 computes (1/3) Re Tr of the plaquettes),
// evaluated here from global coordinates.
// ------------------------------------------------------------------------------------
extern "C" void oq_coldstart(const oq_geom* g, double* u) {
  const size_t n = (size_t)18 * g->ntotal * 4 * 2 * 16;
  std::fill(u, u + n, 0.0);
  for (int ibl = 1; ibl <= 16; ++ibl)
    for (int ieo = 1; ieo <= 2; ++ieo)
      for (int mu = 1; mu <= 4; ++mu)
        for (int s = 1; s <= g->ntotal; ++s) {
          double* U = u + g->ui(1, s, mu, ieo, ibl);
          U[0] = U[8] = U[16] = 1.0;
        }
}

namespace {
void link_at(const oq_geom* g, const double* u, const int* x, int mu, double* out) {
  int isite, ieo, ibl, gblclr, ibleo;
  oq_site_of_coords(g, x, &isite, &ieo, &ibl, &gblclr, &ibleo);
  const double* U = u + g->ui(1, isite, mu, ieo, ibl);
  std::memcpy(out, U, sizeof(double) * 18);
}
void mm(const double* a, const double* b, double* c) {  // c = a b
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double re = 0, im = 0;
      for (int k = 0; k < 3; ++k) {
        const double ar = a[2 * (3 * i + k)], ai = a[2 * (3 * i + k) + 1];
        const double br = b[2 * (3 * k + j)], bi = b[2 * (3 * k + j) + 1];
        re += ar * br - ai * bi;
        im += ar * bi + ai * br;
      }
      c[2 * (3 * i + j)] = re;
      c[2 * (3 * i + j) + 1] = im;
    }
}
void dag(const double* a, double* c) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      c[2 * (3 * i + j)] = a[2 * (3 * j + i)];
      c[2 * (3 * i + j) + 1] = -a[2 * (3 * j + i) + 1];
    }
}
}  // namespace

extern "C" double oq_aveplaq(const oq_geom* g, const double* u) {
  double sum = 0.0;
  long count = 0;
  int x[4];
  for (x[3] = 0; x[3] < g->n[3]; ++x[3])
    for (x[2] = 0; x[2] < g->n[2]; ++x[2])
      for (x[1] = 0; x[1] < g->n[1]; ++x[1])
        for (x[0] = 0; x[0] < g->n[0]; ++x[0])
          for (int mu = 1; mu <= 4; ++mu)
            for (int nu = mu + 1; nu <= 4; ++nu) {
              double a[18], b[18], c[18], d[18], t1[18], t2[18], t3[18], bd[18], dd[18];
              int y[4];
              link_at(g, u, x, mu, a);
              std::memcpy(y, x, sizeof y);
              y[mu - 1] = (y[mu - 1] + 1) % g->n[mu - 1];
              link_at(g, u, y, nu, b);
              std::memcpy(y, x, sizeof y);
              y[nu - 1] = (y[nu - 1] + 1) % g->n[nu - 1];
              link_at(g, u, y, mu, c);
              link_at(g, u, x, nu, d);
              dag(c, bd);
              dag(d, dd);
              mm(a, b, t1);
              mm(t1, bd, t2);
              mm(t2, dd, t3);
              sum += (t3[0] + t3[8] + t3[16]) / 3.0;
              ++count;
            }
  return sum / (double)count;
}
