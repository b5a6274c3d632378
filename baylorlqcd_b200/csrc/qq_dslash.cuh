// Wilson hopping term H_eo / H_oe (the reference's Hsingle, Q/diracops.f90:554-599,
// with mulbac :950-1159 and mulfor :1163-1391) for the B200.
//
// One thread per output site.  For every direction the thread gathers the two
// neighbour spinors with the periodic / antiperiodic / fixed boundary factor folded
// into the hop coefficient (the MPI halo exchange of setvector/slidevector becomes
// in-kernel neighbour indexing), spin-projects them with (1 -/+ gamma_mu) in the
// reference gamma basis (so only two colour vectors are multiplied by the link),
// multiplies by U or U^dagger and accumulates in registers.  Links are read once per
// site and applied to NRHS right-hand sides.  The epilogue fuses the twisted-mass /
// Schur-complement axpys of Hdouble (:264-346) and Hdbletm (:435-550).
#pragma once
#include "qq_fields.cuh"

namespace qq {

enum Epilogue : int {
  EPI_STORE = 0,  // out = H in
  EPI_TWIST = 1,  // out = (1 - i a gamma5) H in           (Hdbletm :483-490)
  EPI_DBLE = 2,   // out = f1*g + f2*J(g) - f3 * H in      (Hdbletm :496-514, Hdouble :340-343)
};

constexpr int kMaxRhs = 8;

struct HopArgs {
  Geom g;
  HopCoef c;
  int pout;                    // output parity (0 = gblclr 1, 1 = gblclr 2)
  int nrhs;
  const void* gauge;
  const void* in[kMaxRhs];
  const float* in_norm[kMaxRhs];
  void* out[kMaxRhs];
  float* out_norm[kMaxRhs];
  const void* aux[kMaxRhs];    // g of EPI_DBLE (same precision as out)
  const float* aux_norm[kMaxRhs];
  double a;                    // EPI_TWIST: 2 kappa mu
  double f1, f2, f3;           // EPI_DBLE factors
};

template <class R>
__device__ inline void matvec(const Su3<R>& u, const cplx<R>* h, cplx<R>* w) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cplx<R> t = cmul(u.e[a][0], h[0]);
    t = cadd(t, cmul(u.e[a][1], h[1]));
    t = cadd(t, cmul(u.e[a][2], h[2]));
    w[a] = t;
  }
}
template <class R>
__device__ inline void matvec_dag(const Su3<R>& u, const cplx<R>* h, cplx<R>* w) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cplx<R> t = cmulconj(u.e[0][a], h[0]);
    t = cadd(t, cmulconj(u.e[1][a], h[1]));
    t = cadd(t, cmulconj(u.e[2][a], h[2]));
    w[a] = t;
  }
}

// Half-spinor projection (1 + S gamma_MU) psi = reconstruct(h0, h1), MU = 0..3 for
// gamma_1..gamma_4 of Q/diracops.f90:61-71; S = -1 or +1.
template <int MU, int S, class R>
__device__ inline void project(const cplx<R>* psi, R coef, cplx<R>* h) {
  const R s = (R)S;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    cplx<R> h0, h1;
    if (MU == 0) {
      h0 = cadd(psi[0 + c], cscale(s, psi[9 + c]));
      h1 = cadd(psi[3 + c], cscale(s, psi[6 + c]));
    } else if (MU == 1) {
      h0 = csub(psi[0 + c], cscale(s, ctimesi(psi[9 + c])));
      h1 = cadd(psi[3 + c], cscale(s, ctimesi(psi[6 + c])));
    } else if (MU == 2) {
      h0 = cadd(psi[0 + c], cscale(s, psi[6 + c]));
      h1 = csub(psi[3 + c], cscale(s, psi[9 + c]));
    } else {
      if (S < 0) {
        h0 = cscale((R)2, psi[6 + c]);
        h1 = cscale((R)2, psi[9 + c]);
      } else {
        h0 = cscale((R)2, psi[0 + c]);
        h1 = cscale((R)2, psi[3 + c]);
      }
    }
    h[c] = cscale(coef, h0);
    h[3 + c] = cscale(coef, h1);
  }
}

template <int MU, int S, class R>
__device__ inline void reconstruct_acc(cplx<R>* acc, const cplx<R>* w) {
  const R s = (R)S;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const cplx<R> w0 = w[c], w1 = w[3 + c];
    if (MU == 3) {
      if (S < 0) {
        acc[6 + c] = cadd(acc[6 + c], w0);
        acc[9 + c] = cadd(acc[9 + c], w1);
      } else {
        acc[0 + c] = cadd(acc[0 + c], w0);
        acc[3 + c] = cadd(acc[3 + c], w1);
      }
      continue;
    }
    acc[0 + c] = cadd(acc[0 + c], w0);
    acc[3 + c] = cadd(acc[3 + c], w1);
    if (MU == 0) {
      acc[6 + c] = cadd(acc[6 + c], cscale(s, w1));
      acc[9 + c] = cadd(acc[9 + c], cscale(s, w0));
    } else if (MU == 1) {
      acc[6 + c] = csub(acc[6 + c], cscale(s, ctimesi(w1)));
      acc[9 + c] = cadd(acc[9 + c], cscale(s, ctimesi(w0)));
    } else {
      acc[6 + c] = cadd(acc[6 + c], cscale(s, w0));
      acc[9 + c] = csub(acc[9 + c], cscale(s, w1));
    }
  }
}

template <int SP, int LP, int RECON, int NRHS, int MU, bool FWD, class R>
__device__ inline void hop(const HopArgs& a, int s, const int* x, cplx<R> (*acc)[12]) {
  using SIO = SpinorIO<SP>;
  using LIO = LinkIO<LP, RECON>;
  int y[4] = {x[0], x[1], x[2], x[3]};
  R sgn = (R)1;
  if (FWD) {
    y[MU] += 1;
    if (y[MU] == a.g.n[MU]) {
      y[MU] = 0;
      sgn = (R)a.g.bc[MU];
    }
  } else {
    y[MU] -= 1;
    if (y[MU] < 0) {
      y[MU] = a.g.n[MU] - 1;
      sgn = (R)a.g.bc[MU];
    }
  }
  if (sgn == (R)0) return;
  const int sy = site_index(a.g, y);
  const R cm = sgn * (R)(FWD ? a.c.fm[MU] : a.c.bm[MU]);
  const R cp = sgn * (R)(FWD ? a.c.fp[MU] : a.c.bp[MU]);
  Su3<R> u;
  if (FWD)
    LIO::load(a.gauge, a.g.vh, a.pout, MU, s, u);
  else
    LIO::load(a.gauge, a.g.vh, 1 - a.pout, MU, sy, u);
#pragma unroll
  for (int r = 0; r < NRHS; ++r) {
    cplx<R> psi[12];
    SIO::load(a.in[r], a.in_norm[r], a.g.vh, sy, psi);
    cplx<R> h[6], w[6];
    if (cm != (R)0) {
      project<MU, -1>(psi, cm, h);
      if (FWD) {
        matvec(u, h, w);
        matvec(u, h + 3, w + 3);
      } else {
        matvec_dag(u, h, w);
        matvec_dag(u, h + 3, w + 3);
      }
      reconstruct_acc<MU, -1>(acc[r], w);
    }
    if (cp != (R)0) {
      project<MU, +1>(psi, cp, h);
      if (FWD) {
        matvec(u, h, w);
        matvec(u, h + 3, w + 3);
      } else {
        matvec_dag(u, h, w);
        matvec_dag(u, h + 3, w + 3);
      }
      reconstruct_acc<MU, +1>(acc[r], w);
    }
  }
}

template <int SP, int LP, int RECON, int NRHS, int EPI>
__global__ void __launch_bounds__(128) hop_kernel(HopArgs a) {
  using SIO = SpinorIO<SP>;
  using R = typename SIO::R;
  static_assert(sizeof(typename LinkIO<LP, RECON>::R) == sizeof(R), "link/spinor precision");
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.g.vh) return;
  int x[4];
  site_coords(a.g, a.pout, s, x);
  cplx<R> acc[NRHS][12];
#pragma unroll
  for (int r = 0; r < NRHS; ++r)
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[r][c] = {(R)0, (R)0};

  hop<SP, LP, RECON, NRHS, 0, true>(a, s, x, acc);
  hop<SP, LP, RECON, NRHS, 0, false>(a, s, x, acc);
  hop<SP, LP, RECON, NRHS, 1, true>(a, s, x, acc);
  hop<SP, LP, RECON, NRHS, 1, false>(a, s, x, acc);
  hop<SP, LP, RECON, NRHS, 2, true>(a, s, x, acc);
  hop<SP, LP, RECON, NRHS, 2, false>(a, s, x, acc);
  hop<SP, LP, RECON, NRHS, 3, true>(a, s, x, acc);
  hop<SP, LP, RECON, NRHS, 3, false>(a, s, x, acc);

#pragma unroll
  for (int r = 0; r < NRHS; ++r) {
    cplx<R> o[12];
    if (EPI == EPI_STORE) {
#pragma unroll
      for (int c = 0; c < 12; ++c) o[c] = acc[r][c];
    } else if (EPI == EPI_TWIST) {
      const R t = (R)a.a;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        o[0 + c] = csub(acc[r][0 + c], cscale(t, acc[r][6 + c]));
        o[3 + c] = csub(acc[r][3 + c], cscale(t, acc[r][9 + c]));
        o[6 + c] = cadd(acc[r][6 + c], cscale(t, acc[r][0 + c]));
        o[9 + c] = cadd(acc[r][9 + c], cscale(t, acc[r][3 + c]));
      }
    } else {
      cplx<R> gg[12];
      SIO::load(a.aux[r], a.aux_norm[r], a.g.vh, s, gg);
      const R f1 = (R)a.f1, f2 = (R)a.f2, f3 = (R)a.f3;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        o[0 + c] = csub(cadd(cscale(f1, gg[0 + c]), cscale(f2, gg[6 + c])), cscale(f3, acc[r][0 + c]));
        o[3 + c] = csub(cadd(cscale(f1, gg[3 + c]), cscale(f2, gg[9 + c])), cscale(f3, acc[r][3 + c]));
        o[6 + c] = csub(csub(cscale(f1, gg[6 + c]), cscale(f2, gg[0 + c])), cscale(f3, acc[r][6 + c]));
        o[9 + c] = csub(csub(cscale(f1, gg[9 + c]), cscale(f2, gg[3 + c])), cscale(f3, acc[r][9 + c]));
      }
    }
    SIO::store(a.out[r], a.out_norm[r], a.g.vh, s, o);
  }
}

// Host-side helper: the hop coefficients of Hsingle for action coefficients
// c1[mu] = coact(3,1,mu), c2[mu] = coact(3,2,mu) and dagger flag idag.
inline HopCoef make_hopcoef(const double* c1, const double* c2, int idag) {
  HopCoef h;
  for (int mu = 0; mu < 4; ++mu) {
    const double a = 0.5 * (c1[mu] + c2[mu]), b = 0.5 * (c1[mu] - c2[mu]);
    // forward hop: (c1 - c2 gamma) for idag=0, (c1 + c2 gamma) for idag=1
    h.fm[mu] = idag ? b : a;
    h.fp[mu] = idag ? a : b;
    // backward hop: (c1 + c2 gamma) for idag=0, (c1 - c2 gamma) for idag=1
    h.bm[mu] = idag ? a : b;
    h.bp[mu] = idag ? b : a;
  }
  return h;
}

}  // namespace qq
