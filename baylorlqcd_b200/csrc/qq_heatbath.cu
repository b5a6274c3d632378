// Quenched SU(3) gauge configurations on the GPU (input producer for the solvers).
//
// The reference generates configurations with a pseudo-heatbath (G/heatbath.f90
// phbup :33-76, su2up :239-323, sprd1 :327-467; staples G/gaugetools.f90:39-345)
// driven by a sequential lagged-Fibonacci stream whose consumption depends on the
// accept/reject history, so its configurations cannot be reproduced in parallel.
// This file is a statistically equivalent parallel version: Wilson plaquette action
// at coupling beta, Cabibbo-Marinari updates of the three SU(2) subgroups with the
// Kennedy-Pendleton sampler (Phys. Lett. B156 (1985) 393), all links of one
// direction and one checkerboard parity updated at once (they share no staple), and
// a counter-based Philox-4x32-10 generator (Salmon et al., SC11, 2011) keyed by
// (seed, link, sweep, subgroup, attempt).  Links are re-unitarised every 8 sweeps.
//
// Device layout here is lexicographic: link (mu, x) at [(mu * V + lex(x)) * 9]
// complex numbers, row-major 3x3.
#include <cmath>
#include <cstring>

#include "qq_ctx.h"

namespace qq {

namespace {

struct C3 {
  double re[3][3], im[3][3];
};

__device__ inline void mm3(const C3& a, const C3& b, C3& c) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double r = 0.0, s = 0.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        r += a.re[i][k] * b.re[k][j] - a.im[i][k] * b.im[k][j];
        s += a.re[i][k] * b.im[k][j] + a.im[i][k] * b.re[k][j];
      }
      c.re[i][j] = r;
      c.im[i][j] = s;
    }
}
__device__ inline void dag3(const C3& a, C3& c) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      c.re[i][j] = a.re[j][i];
      c.im[i][j] = -a.im[j][i];
    }
}
__device__ inline void load3(const double2* L, size_t idx, C3& u) {
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const double2 t = L[idx * 9 + q];
    u.re[q / 3][q % 3] = t.x;
    u.im[q / 3][q % 3] = t.y;
  }
}
__device__ inline void store3(double2* L, size_t idx, const C3& u) {
#pragma unroll
  for (int q = 0; q < 9; ++q) L[idx * 9 + q] = make_double2(u.re[q / 3][q % 3], u.im[q / 3][q % 3]);
}

struct Lat {
  int n[4];
  long long V;
  __device__ void coords(long long lex, int* x) const {
    x[0] = (int)(lex % n[0]);
    lex /= n[0];
    x[1] = (int)(lex % n[1]);
    lex /= n[1];
    x[2] = (int)(lex % n[2]);
    x[3] = (int)(lex / n[2]);
  }
  __device__ long long lex(const int* x) const {
    return x[0] + (long long)n[0] * (x[1] + (long long)n[1] * (x[2] + (long long)n[2] * x[3]));
  }
  __device__ long long shift(const int* x, int mu, int d) const {
    int y[4] = {x[0], x[1], x[2], x[3]};
    y[mu] = (y[mu] + d + n[mu]) % n[mu];
    return lex(y);
  }
};

// Philox-4x32-10
__device__ inline uint4 philox(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const unsigned hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}
__device__ inline double unif(unsigned u) { return ((double)u + 0.5) * 2.3283064365386963e-10; }

// Sum of the six staples around link (mu, x): A such that the local action is
// -(beta/3) Re Tr(U_mu(x) A).
__device__ void staple(const double2* L, const Lat& g, const int* x, int mu, C3& A) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A.re[i][j] = A.im[i][j] = 0.0;
  const long long xl = g.lex(x);
  const long long xpmu = g.shift(x, mu, 1);
  for (int nu = 0; nu < 4; ++nu) {
    if (nu == mu) continue;
    C3 a, b, c, t, t2, d;
    // forward: U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
    load3(L, (size_t)nu * g.V + xpmu, a);
    load3(L, (size_t)mu * g.V + g.shift(x, nu, 1), b);
    load3(L, (size_t)nu * g.V + xl, c);
    dag3(b, d);
    mm3(a, d, t);
    dag3(c, d);
    mm3(t, d, t2);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        A.re[i][j] += t2.re[i][j];
        A.im[i][j] += t2.im[i][j];
      }
    // backward: U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
    int xm[4] = {x[0], x[1], x[2], x[3]};
    xm[nu] = (xm[nu] - 1 + g.n[nu]) % g.n[nu];
    const long long xmnu = g.lex(xm);
    load3(L, (size_t)nu * g.V + g.shift(xm, mu, 1), a);
    load3(L, (size_t)mu * g.V + xmnu, b);
    load3(L, (size_t)nu * g.V + xmnu, c);
    dag3(a, d);
    C3 db;
    dag3(b, db);
    mm3(d, db, t);
    mm3(t, c, t2);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        A.re[i][j] += t2.re[i][j];
        A.im[i][j] += t2.im[i][j];
      }
  }
}

__global__ void heatbath_kernel(double2* L, Lat g, int mu, int parity, double beta, uint2 key,
                                unsigned sweep) {
  const long long half = g.V / 2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < half;
       t += (long long)gridDim.x * blockDim.x) {
    // t-th site of the given parity in lexicographic order
    const long long lex0 = 2 * t;
    int x[4];
    g.coords(lex0, x);
    if (((x[0] + x[1] + x[2] + x[3]) & 1) != parity) x[0] += 1;  // n[0] even
    const long long xl = g.lex(x);
    C3 A, U, W;
    staple(L, g, x, mu, A);
    load3(L, (size_t)mu * g.V + xl, U);
    for (int sg = 0; sg < 3; ++sg) {
      const int i = sg == 2 ? 1 : 0;
      const int j = sg == 0 ? 1 : 2;
      mm3(U, A, W);
      // SU(2) part of the (i,j) block of W: v = a0 + i a.sigma
      double a0 = 0.5 * (W.re[i][i] + W.re[j][j]);
      double a3 = 0.5 * (W.im[i][i] - W.im[j][j]);
      double a1 = 0.5 * (W.im[i][j] + W.im[j][i]);
      double a2 = 0.5 * (W.re[i][j] - W.re[j][i]);
      const double k = sqrt(a0 * a0 + a1 * a1 + a2 * a2 + a3 * a3);
      if (!(k > 1e-300)) continue;
      a0 /= k; a1 /= k; a2 /= k; a3 /= k;
      const double alpha = 2.0 * beta * k / 3.0;
      // Kennedy-Pendleton: x0 with density sqrt(1 - x0^2) exp(alpha x0)
      double x0 = 1.0;
      double r0 = 0, r1 = 0, r2 = 0;
      for (unsigned att = 0; att < 64; ++att) {
        const uint4 rb = philox(make_uint4((unsigned)xl, (unsigned)(mu | (sg << 2)) | ((unsigned)(xl >> 32) << 8),
                                           sweep, att),
                                key);
        const double u1 = unif(rb.x), u2 = unif(rb.y), u3 = unif(rb.z), u4 = unif(rb.w);
        const double c = cos(6.283185307179586 * u2);
        const double d = -(log(u1) + c * c * log(u3)) / alpha;
        if (u4 * u4 <= 1.0 - 0.5 * d) {
          x0 = 1.0 - d;
          break;
        }
      }
      {
        const uint4 rb = philox(make_uint4((unsigned)xl, (unsigned)(mu | (sg << 2) | 64) | ((unsigned)(xl >> 32) << 8),
                                           sweep, 999u),
                                key);
        r0 = 2.0 * unif(rb.x) - 1.0;      // cos(theta)
        r1 = 6.283185307179586 * unif(rb.y);  // phi
        (void)r2;
      }
      const double rad = sqrt(fmax(0.0, 1.0 - x0 * x0));
      const double st = sqrt(fmax(0.0, 1.0 - r0 * r0));
      const double x1 = rad * st * cos(r1), x2 = rad * st * sin(r1), x3 = rad * r0;
      // R = X V^dagger in quaternion form: X = x0 + i x.sigma, V = a0 + i a.sigma
      // (q1 q2)_0 = p0 q0 - p.q ; vec = p0 q + q0 p - p x q,  with q = conj(V) = (a0, -a)
      const double q0 = a0, q1 = -a1, q2 = -a2, q3 = -a3;
      const double R0 = x0 * q0 - (x1 * q1 + x2 * q2 + x3 * q3);
      const double R1 = x0 * q1 + q0 * x1 - (x2 * q3 - x3 * q2);
      const double R2 = x0 * q2 + q0 * x2 - (x3 * q1 - x1 * q3);
      const double R3 = x0 * q3 + q0 * x3 - (x1 * q2 - x2 * q1);
      // SU(2) matrix [[R0 + i R3, R2 + i R1], [-R2 + i R1, R0 - i R3]] embedded in (i, j)
      const double m_re[2][2] = {{R0, R2}, {-R2, R0}};
      const double m_im[2][2] = {{R3, R1}, {R1, -R3}};
      C3 N = U;
      const int idx[2] = {i, j};
      for (int a = 0; a < 2; ++a)
        for (int col = 0; col < 3; ++col) {
          double re = 0.0, im = 0.0;
          for (int b = 0; b < 2; ++b) {
            const int rb = idx[b];
            re += m_re[a][b] * U.re[rb][col] - m_im[a][b] * U.im[rb][col];
            im += m_re[a][b] * U.im[rb][col] + m_im[a][b] * U.re[rb][col];
          }
          N.re[idx[a]][col] = re;
          N.im[idx[a]][col] = im;
        }
      U = N;
    }
    store3(L, (size_t)mu * g.V + xl, U);
  }
}

__global__ void reunitarise_kernel(double2* L, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    C3 u;
    load3(L, t, u);
    double nr = 0.0;
    for (int c = 0; c < 3; ++c) nr += u.re[0][c] * u.re[0][c] + u.im[0][c] * u.im[0][c];
    nr = 1.0 / sqrt(nr);
    for (int c = 0; c < 3; ++c) {
      u.re[0][c] *= nr;
      u.im[0][c] *= nr;
    }
    double pr = 0.0, pi = 0.0;  // <row0, row1>
    for (int c = 0; c < 3; ++c) {
      pr += u.re[0][c] * u.re[1][c] + u.im[0][c] * u.im[1][c];
      pi += u.re[0][c] * u.im[1][c] - u.im[0][c] * u.re[1][c];
    }
    for (int c = 0; c < 3; ++c) {
      u.re[1][c] -= pr * u.re[0][c] - pi * u.im[0][c];
      u.im[1][c] -= pr * u.im[0][c] + pi * u.re[0][c];
    }
    nr = 0.0;
    for (int c = 0; c < 3; ++c) nr += u.re[1][c] * u.re[1][c] + u.im[1][c] * u.im[1][c];
    nr = 1.0 / sqrt(nr);
    for (int c = 0; c < 3; ++c) {
      u.re[1][c] *= nr;
      u.im[1][c] *= nr;
    }
    // row2 = conj(row0 x row1)
    for (int c = 0; c < 3; ++c) {
      const int a = (c + 1) % 3, b = (c + 2) % 3;
      const double re = u.re[0][a] * u.re[1][b] - u.im[0][a] * u.im[1][b] - (u.re[0][b] * u.re[1][a] - u.im[0][b] * u.im[1][a]);
      const double im = u.re[0][a] * u.im[1][b] + u.im[0][a] * u.re[1][b] - (u.re[0][b] * u.im[1][a] + u.im[0][b] * u.re[1][a]);
      u.re[2][c] = re;
      u.im[2][c] = -im;
    }
    store3(L, t, u);
  }
}

__global__ void coldstart_kernel(double2* L, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    for (int q = 0; q < 9; ++q) L[t * 9 + q] = make_double2(q % 4 == 0 ? 1.0 : 0.0, 0.0);
}

__global__ void plaquette_kernel(const double2* L, Lat g, double* partial) {
  double s = 0.0;
  for (long long xl = blockIdx.x * (long long)blockDim.x + threadIdx.x; xl < g.V;
       xl += (long long)gridDim.x * blockDim.x) {
    int x[4];
    g.coords(xl, x);
    for (int mu = 0; mu < 4; ++mu)
      for (int nu = mu + 1; nu < 4; ++nu) {
        C3 a, b, c, d, t, t2, e;
        load3(L, (size_t)mu * g.V + xl, a);
        load3(L, (size_t)nu * g.V + g.shift(x, mu, 1), b);
        load3(L, (size_t)mu * g.V + g.shift(x, nu, 1), c);
        load3(L, (size_t)nu * g.V + xl, d);
        mm3(a, b, t);
        dag3(c, e);
        mm3(t, e, t2);
        dag3(d, e);
        mm3(t2, e, t);
        s += (t.re[0][0] + t.re[1][1] + t.re[2][2]) / 3.0;
      }
  }
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// lexicographic links -> reference u(18, ntotal, 4, 2, 16)
__global__ void lex_to_ref_kernel(const double2* L, Lat g, RefDims d, Geom gg, double* ref) {
  for (long long xl = blockIdx.x * (long long)blockDim.x + threadIdx.x; xl < g.V;
       xl += (long long)gridDim.x * blockDim.x) {
    int x[4];
    g.coords(xl, x);
    int isite, ieo, ibleo;
    ref_site(gg, x, &isite, &ieo, &ibleo);
    const int ibl = 1 + (x[0] & 1) + 2 * (x[1] & 1) + 4 * (x[2] & 1) + 8 * (x[3] & 1);
    for (int mu = 0; mu < 4; ++mu) {
      double* u = ref + ref_ui(d, 1, isite, mu + 1, ieo, ibl);
      for (int q = 0; q < 9; ++q) {
        const double2 t = L[((size_t)mu * g.V + xl) * 9 + q];
        u[2 * q] = t.x;
        u[2 * q + 1] = t.y;
      }
    }
  }
}

}  // namespace

int heatbath_generate(qq_ctx* c, double beta, int nsweeps, unsigned long long seed, double* u_ref,
                      double* plaq) {
  Lat g;
  for (int mu = 0; mu < 4; ++mu) g.n[mu] = c->g.n[mu];
  g.V = (long long)g.n[0] * g.n[1] * g.n[2] * g.n[3];
  DevBuf L;
  QQ_CK(L.alloc(sizeof(double2) * 9 * 4 * (size_t)g.V));
  double2* Lp = L.as<double2>();
  coldstart_kernel<<<592, 256, 0, c->st>>>(Lp, 4 * g.V);
  QQ_CK(cudaGetLastError());
  const uint2 key = make_uint2((unsigned)seed, (unsigned)(seed >> 32));
  count_launch(1 + 8LL * nsweeps + (nsweeps + 7) / 8 + 2);
  for (int sw = 0; sw < nsweeps; ++sw) {
    for (int mu = 0; mu < 4; ++mu)
      for (int p = 0; p < 2; ++p) {
        heatbath_kernel<<<592, 128, 0, c->st>>>(Lp, g, mu, p, beta, key, (unsigned)sw);
        QQ_CK(cudaGetLastError());
      }
    if (sw % 8 == 7 || sw == nsweeps - 1) {
      reunitarise_kernel<<<592, 256, 0, c->st>>>(Lp, 4 * g.V);
      QQ_CK(cudaGetLastError());
    }
  }
  if (plaq) {
    plaquette_kernel<<<kRedBlocks, 256, 0, c->st>>>(Lp, g, c->partial.as<double>());
    QQ_CK(cudaGetLastError());
    std::vector<double> part(kRedBlocks);
    QQ_CK(cudaMemcpyAsync(part.data(), c->partial.p, sizeof(double) * kRedBlocks, cudaMemcpyDeviceToHost, c->st));
    QQ_CK(cudaStreamSynchronize(c->st));
    double s = 0.0;
    for (double v : part) s += v;
    *plaq = s / (6.0 * (double)g.V);
  }
  const size_t nu = (size_t)18 * c->rd.ntotal * 4 * 2 * 16;
  double* dref = nullptr;
  QQ_TRY(stage_out_begin(c, 0, u_ref, nu, &dref));
  QQ_CK(cudaMemsetAsync(dref, 0, nu * sizeof(double), c->st));
  lex_to_ref_kernel<<<592, 256, 0, c->st>>>(Lp, g, c->rd, c->g, dref);
  QQ_CK(cudaGetLastError());
  QQ_TRY(stage_out_end(c, 0, u_ref, nu, dref));
  QQ_CK(cudaStreamSynchronize(c->st));
  return QQ_OK;
}

}  // namespace qq
