// Gauge-configuration and propagator files in the reference's formats (host code).
//
// Both are Fortran unformatted sequential files: every WRITE statement is one record,
// framed by a 4-byte little-endian length before and after the data; reals are
// 8 bytes and integers 4 (U/kinds.f90).
//   * GFwrite / GFread (G/gaugetools.f90:1260-1334): after re-unitarising the links
//     (fixsu3 :1338-1432), rows 1 and 2 of every link (icri = 1..12) are written as
//     one 8-double record per (icri, isite, ibl), in that loop order, holding
//     (u(icri,isite,mu,1,ibl), u(icri,isite,mu,2,ibl), mu = 1..4); then one record of
//     gaction(4), beta, alat(4), tad(4), icfgsave, myid.  Reading completes row 3 with
//     fixsu3.
//   * FPwrite / FPread (Q/quark.f90:3379-3481): one 8-double record per
//     (isite, ibl, icri) holding (x(icri,isite,id,1,ibleo), x(icri,isite,id,2,ibleo),
//     id = 1..4) from xe when block ibl is globally even (vecblinv(1,ibl) = 1) and from
//     xo otherwise, ibleo = vecblinv(2,ibl); then one record of kappa, tmqcd, cSW,
//     icsrc, idsrc, icfg, myid.
// Arrays are host memory in the reference layouts: u(18,ntotal,4,2,16) and
// x(6,ntotal,4,2,8).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "qq_ctx.h"

namespace qq {
namespace {

// G/lattice.f90:351-352
constexpr int kVecblinv[2][16] = {{1, 2, 2, 1, 2, 1, 1, 2, 2, 1, 1, 2, 1, 2, 2, 1},
                                  {1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8}};

inline size_t ui(int a, int isite, int mu, int ieo, int ibl, int ntotal) {
  return (size_t)(a - 1) +
         18 * ((size_t)(isite - 1) + (size_t)ntotal * ((size_t)(mu - 1) + 4 * ((size_t)(ieo - 1) + 2 * (size_t)(ibl - 1))));
}
inline size_t gi(int a, int isite, int id, int ieo, int ibleo, int ntotal) {
  return (size_t)(a - 1) +
         6 * ((size_t)(isite - 1) + (size_t)ntotal * ((size_t)(id - 1) + 4 * ((size_t)(ieo - 1) + 2 * (size_t)(ibleo - 1))));
}

// fixsu3, G/gaugetools.f90:1338-1432, in its operation order.
void fixsu3(double* u, int nvhalf, int ntotal) {
  for (int ieo = 1; ieo <= 2; ++ieo)
    for (int mu = 1; mu <= 4; ++mu)
      for (int isite = 1; isite <= nvhalf; ++isite)
        for (int ibl = 1; ibl <= 16; ++ibl) {
          double* w = u + ui(1, isite, mu, ieo, ibl, ntotal);  // w[i - 1] = u(i,isite,mu,ieo,ibl)
          double c1r = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2] + w[3] * w[3] + w[4] * w[4] + w[5] * w[5]);
          for (int i = 0; i < 6; ++i) w[i] = w[i] / c1r;
          c1r = w[6] * w[0] + w[7] * w[1] + w[8] * w[2] + w[9] * w[3] + w[10] * w[4] + w[11] * w[5];
          const double c1i = w[7] * w[0] - w[6] * w[1] + w[9] * w[2] - w[8] * w[3] + w[11] * w[4] - w[10] * w[5];
          w[6] = w[6] - c1r * w[0] + c1i * w[1];
          w[7] = w[7] - c1r * w[1] - c1i * w[0];
          w[8] = w[8] - c1r * w[2] + c1i * w[3];
          w[9] = w[9] - c1r * w[3] - c1i * w[2];
          w[10] = w[10] - c1r * w[4] + c1i * w[5];
          w[11] = w[11] - c1r * w[5] - c1i * w[4];
          c1r = std::sqrt(w[6] * w[6] + w[7] * w[7] + w[8] * w[8] + w[9] * w[9] + w[10] * w[10] + w[11] * w[11]);
          for (int i = 6; i < 12; ++i) w[i] = w[i] / c1r;
          w[16] = w[0] * w[8] - w[1] * w[9] - w[2] * w[6] + w[3] * w[7];
          w[14] = w[4] * w[6] - w[5] * w[7] - w[0] * w[10] + w[1] * w[11];
          w[12] = w[2] * w[10] - w[3] * w[11] - w[4] * w[8] + w[5] * w[9];
          w[17] = -w[0] * w[9] - w[1] * w[8] + w[2] * w[7] + w[3] * w[6];
          w[15] = -w[4] * w[7] - w[5] * w[6] + w[0] * w[11] + w[1] * w[10];
          w[13] = -w[2] * w[11] - w[3] * w[10] + w[4] * w[9] + w[5] * w[8];
        }
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

bool put_record(FILE* f, const void* data, int32_t n) {
  return std::fwrite(&n, 4, 1, f) == 1 && std::fwrite(data, 1, (size_t)n, f) == (size_t)n &&
         std::fwrite(&n, 4, 1, f) == 1;
}

bool get_record(FILE* f, void* data, int32_t n) {
  int32_t a = 0, b = 0;
  return std::fread(&a, 4, 1, f) == 1 && a == n && std::fread(data, 1, (size_t)n, f) == (size_t)n &&
         std::fread(&b, 4, 1, f) == 1 && b == n;
}

int check_dims(int nvhalf, int ntotal) {
  if (nvhalf < 1 || ntotal < nvhalf) return set_error(QQ_BAD_ARG, "need 1 <= nvhalf <= ntotal");
  return QQ_OK;
}

#pragma pack(push, 1)
struct GfTrailer {
  int32_t gaction[4];
  double beta, alat[4], tad[4];
  int32_t icfgsave, myid;
};
struct FpTrailer {
  double kappa, tmqcd, csw;
  int32_t icsrc, idsrc, icfg, myid;
};
#pragma pack(pop)
static_assert(sizeof(GfTrailer) == 96, "GFwrite trailer record");
static_assert(sizeof(FpTrailer) == 40, "FPwrite trailer record");

}  // namespace
}  // namespace qq

using namespace qq;

extern "C" int qq_gfwrite(const char* path, double* u, int nvhalf, int ntotal, const int gaction[4],
                          double beta, const double alat[4], const double tad[4], int icfgsave, int myid) {
  if (!path || !u || !gaction || !alat || !tad) return set_error(QQ_BAD_ARG, "null argument");
  QQ_TRY(check_dims(nvhalf, ntotal));
  fixsu3(u, nvhalf, ntotal);  // as GFwrite, in place
  File F;
  F.f = std::fopen(path, "wbx");  // status="new"
  if (!F.f) return set_error(QQ_BAD_ARG, std::string("cannot create ") + path + " (it must not exist)");
  double rec[8];
  for (int icri = 1; icri <= 12; ++icri)
    for (int isite = 1; isite <= nvhalf; ++isite)
      for (int ibl = 1; ibl <= 16; ++ibl) {
        for (int mu = 1; mu <= 4; ++mu) {
          rec[2 * (mu - 1)] = u[ui(icri, isite, mu, 1, ibl, ntotal)];
          rec[2 * (mu - 1) + 1] = u[ui(icri, isite, mu, 2, ibl, ntotal)];
        }
        if (!put_record(F.f, rec, sizeof(rec))) return set_error(QQ_BAD_ARG, "write failed");
      }
  GfTrailer t;
  for (int i = 0; i < 4; ++i) {
    t.gaction[i] = gaction[i];
    t.alat[i] = alat[i];
    t.tad[i] = tad[i];
  }
  t.beta = beta;
  t.icfgsave = icfgsave;
  t.myid = myid;
  if (!put_record(F.f, &t, sizeof(t))) return set_error(QQ_BAD_ARG, "write failed");
  return QQ_OK;
}

extern "C" int qq_gfread(const char* path, double* u, int nvhalf, int ntotal, int gaction[4], double* beta,
                         double alat[4], double tad[4], int* icfgsave, int* myid) {
  if (!path || !u || !gaction || !beta || !alat || !tad || !icfgsave || !myid)
    return set_error(QQ_BAD_ARG, "null argument");
  QQ_TRY(check_dims(nvhalf, ntotal));
  File F;
  F.f = std::fopen(path, "rb");
  if (!F.f) return set_error(QQ_BAD_ARG, std::string("cannot open ") + path);
  double rec[8];
  for (int icri = 1; icri <= 12; ++icri)
    for (int isite = 1; isite <= nvhalf; ++isite)
      for (int ibl = 1; ibl <= 16; ++ibl) {
        if (!get_record(F.f, rec, sizeof(rec)))
          return set_error(QQ_BAD_ARG, "not a gauge file of this lattice size (record framing)");
        for (int mu = 1; mu <= 4; ++mu) {
          u[ui(icri, isite, mu, 1, ibl, ntotal)] = rec[2 * (mu - 1)];
          u[ui(icri, isite, mu, 2, ibl, ntotal)] = rec[2 * (mu - 1) + 1];
        }
      }
  GfTrailer t;
  if (!get_record(F.f, &t, sizeof(t))) return set_error(QQ_BAD_ARG, "gauge file trailer record");
  for (int i = 0; i < 4; ++i) {
    gaction[i] = t.gaction[i];
    alat[i] = t.alat[i];
    tad[i] = t.tad[i];
  }
  *beta = t.beta;
  *icfgsave = t.icfgsave;
  *myid = t.myid;
  fixsu3(u, nvhalf, ntotal);  // completes row 3
  return QQ_OK;
}

extern "C" int qq_fpwrite(const char* path, const double* xe, const double* xo, int nvhalf, int ntotal,
                          double kappa, double tmqcd, double csw, int icsrc, int idsrc, int icfg, int myid) {
  if (!path || !xe || !xo) return set_error(QQ_BAD_ARG, "null argument");
  QQ_TRY(check_dims(nvhalf, ntotal));
  File F;
  F.f = std::fopen(path, "wb");  // status="replace"
  if (!F.f) return set_error(QQ_BAD_ARG, std::string("cannot create ") + path);
  double rec[8];
  for (int isite = 1; isite <= nvhalf; ++isite)
    for (int ibl = 1; ibl <= 16; ++ibl) {
      const double* x = kVecblinv[0][ibl - 1] == 1 ? xe : xo;
      const int ibleo = kVecblinv[1][ibl - 1];
      for (int icri = 1; icri <= 6; ++icri) {
        for (int id = 1; id <= 4; ++id) {
          rec[2 * (id - 1)] = x[gi(icri, isite, id, 1, ibleo, ntotal)];
          rec[2 * (id - 1) + 1] = x[gi(icri, isite, id, 2, ibleo, ntotal)];
        }
        if (!put_record(F.f, rec, sizeof(rec))) return set_error(QQ_BAD_ARG, "write failed");
      }
    }
  const FpTrailer t{kappa, tmqcd, csw, icsrc, idsrc, icfg, myid};
  if (!put_record(F.f, &t, sizeof(t))) return set_error(QQ_BAD_ARG, "write failed");
  return QQ_OK;
}

extern "C" int qq_fpread(const char* path, double* xe, double* xo, int nvhalf, int ntotal, double* kappa,
                         double* tmqcd, double* csw, int* icsrc, int* idsrc, int* icfg, int* myid) {
  if (!path || !xe || !xo || !kappa || !tmqcd || !csw || !icsrc || !idsrc || !icfg || !myid)
    return set_error(QQ_BAD_ARG, "null argument");
  QQ_TRY(check_dims(nvhalf, ntotal));
  File F;
  F.f = std::fopen(path, "rb");
  if (!F.f) return set_error(QQ_BAD_ARG, std::string("cannot open ") + path);
  double rec[8];
  for (int isite = 1; isite <= nvhalf; ++isite)
    for (int ibl = 1; ibl <= 16; ++ibl) {
      double* x = kVecblinv[0][ibl - 1] == 1 ? xe : xo;
      const int ibleo = kVecblinv[1][ibl - 1];
      for (int icri = 1; icri <= 6; ++icri) {
        if (!get_record(F.f, rec, sizeof(rec)))
          return set_error(QQ_BAD_ARG, "not a propagator file of this lattice size (record framing)");
        for (int id = 1; id <= 4; ++id) {
          x[gi(icri, isite, id, 1, ibleo, ntotal)] = rec[2 * (id - 1)];
          x[gi(icri, isite, id, 2, ibleo, ntotal)] = rec[2 * (id - 1) + 1];
        }
      }
    }
  FpTrailer t;
  if (!get_record(F.f, &t, sizeof(t))) return set_error(QQ_BAD_ARG, "propagator file trailer record");
  *kappa = t.kappa;
  *tmqcd = t.tmqcd;
  *csw = t.csw;
  *icsrc = t.icsrc;
  *idsrc = t.idsrc;
  *icfg = t.icfg;
  *myid = t.myid;
  return QQ_OK;
}
