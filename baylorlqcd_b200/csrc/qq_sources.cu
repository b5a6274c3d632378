// Sources for propagators and disconnected loops.
//
// The noise sources must reproduce the reference's random stream exactly, so the
// generator is the reference's lagged-Fibonacci generator (G/lagfib.f90: lags
// p = 521, q = 32, XOR; 31-bit words; seeded by bit extraction from the LCG
// x <- 69069 x and moved ahead by `myid + iseed` steps with a polynomial skip).  It
// is sequential by construction and produces O(V) numbers per source, so it runs on
// the host; the sources are written straight into the reference layout.
#include <cstdint>
#include <cstring>
#include <vector>

#include "qq_ctx.h"

namespace qq {

namespace {

class LagFib {
 public:
  static constexpr int kP = 521, kQ = 32;

  void seed(int ndelay) {
    // initial words: bit k of word j is the top bit of the (32 j + k)-th step of the
    // lagged XOR recursion started from LCG top bits (initbirep, lagfib.f90:96-146)
    std::vector<uint32_t> bits(kP);
    uint32_t lcg = 1;
    for (int i = 0; i < kP; ++i) {
      lcg *= 69069u;
      bits[i] = lcg >> 31;
    }
    int j = 0, k = kP - kQ;
    for (int w = 0; w < kP; ++w) {
      uint32_t word = 0;
      for (int b = 0; b < 32; ++b) {
        word = (word << 1) + bits[j];
        bits[j] ^= bits[k];
        j = (j + 1) % kP;
        k = (k + 1) % kP;
      }
      state_[w] = word >> 1;
    }
    skip(ndelay);
    jr_ = 0;
    kr_ = kP - kQ;
    seeded_ = true;
  }
  bool seeded() const { return seeded_; }

  double next() {
    const double fnorm = (double)0.465661e-9f;  // single-precision literal, lagfib.f90:225
    double r;
    do {
      state_[jr_] ^= state_[kr_];
      r = (double)(int32_t)state_[jr_] * fnorm;
    } while (r == 0.0);
    jr_ = jr_ + 1 == kP ? 0 : jr_ + 1;
    kr_ = kr_ + 1 == kP ? 0 : kr_ + 1;
    return r;
  }

 private:
  // Advance the register by `n` steps of the recursion using x^n mod the
  // characteristic polynomial x^p + x^(p-q) + 1 over GF(2) (bigdelay, :150-215).
  void skip(int n) {
    const int low_bits = 40;
    std::vector<uint32_t> ext(2 * kP - 1);
    for (int i = 0; i < kP; ++i) ext[i] = state_[i];
    for (int i = kP; i < 2 * kP - 1; ++i) ext[i] = ext[i - kP] ^ ext[i - kQ];
    // binary digits of n beyond the first p-1 steps, most significant last
    std::vector<int> digit(kP + 32, 0);
    int top = low_bits - 1;
    int m = n;
    while (m > kP - 1) {
      digit[++top] = m & 1;
      m >>= 1;
    }
    std::vector<uint32_t> poly(2 * kP, 0);
    poly[m] = 1;
    for (int d = top; d >= 0; --d) {
      for (int i = kP - 1; i >= 0; --i) {  // square (and shift by the digit)
        poly[2 * i + digit[d]] = poly[i];
        poly[2 * i + 1 - digit[d]] = 0;
      }
      for (int i = 2 * kP - 1; i >= kP; --i) {  // reduce
        poly[i - kP] ^= poly[i];
        poly[i - kQ] ^= poly[i];
      }
    }
    uint32_t out[kP];
    for (int w = 0; w < kP; ++w) {
      uint32_t acc = 0;
      for (int i = 0; i < kP; ++i)
        if (poly[i]) acc ^= ext[w + i];
      out[w] = acc;
    }
    std::memcpy(state_, out, sizeof(out));
  }

  uint32_t state_[kP] = {};
  int jr_ = 0, kr_ = kP - kQ;
  bool seeded_ = false;
};

LagFib g_rng;  // the reference's generator state is module-global too (lagfib.f90:60-66)

// One noise half-vector in the reference's loop order (disconloops.f90:4518-4570):
// colour outer, then site, spin, ieo, ibleo innermost.
void noise_half(const RefDims& d, double* b, bool z4) {
  std::memset(b, 0, sizeof(double) * (size_t)6 * d.ntotal * 64);
  for (int ic = 1; ic <= 3; ++ic)
    for (int isite = 1; isite <= d.nvhalf; ++isite)
      for (int id = 1; id <= 4; ++id)
        for (int ieo = 1; ieo <= 2; ++ieo)
          for (int ibl = 1; ibl <= 8; ++ibl) {
            const double r = g_rng.next();
            const size_t re = ref_gi(d, 2 * ic - 1, isite, id, ieo, ibl);
            if (!z4) {
              b[re] = r > 0.5 ? 1.0 : -1.0;
            } else if (r > 0.75) {
              b[re] = 1.0;
            } else if (0.5 < r && r < 0.75) {
              b[re] = -1.0;
            } else if (0.25 < r && r < 0.5) {
              b[re + 1] = 1.0;
            } else {
              b[re + 1] = -1.0;  // includes the exact ties 0.25, 0.5, 0.75
            }
          }
}

int write_out(qq_ctx* c, double* dst, const std::vector<double>& src) {
  if (is_device_ptr(dst)) {
    QQ_CK(cudaMemcpy(dst, src.data(), sizeof(double) * src.size(), cudaMemcpyHostToDevice));
  } else {
    std::memcpy(dst, src.data(), sizeof(double) * src.size());
  }
  (void)c;
  return QQ_OK;
}

}  // namespace

int lagfib_init(int myid, int iseed) {
  // The delay indexes the skip polynomial, so it must be >= 0 ("ndelay must be a
  // positive integer", lagfib.f90:89); the reference does not check and overruns.
  const long long ndelay = (long long)myid + iseed;
  if (ndelay < 0 || ndelay > 0x7fffffffLL)
    return set_error(QQ_BAD_ARG, "qq_initlagfib: myid + iseed must be in [0, 2^31)");
  g_rng.seed((int)ndelay);
  return QQ_OK;
}

int lagfib_rnds(int m, double* rn) {
  if (!g_rng.seeded()) return set_error(QQ_BAD_ARG, "qq_initlagfib has not been called");
  for (int i = 0; i < m; ++i) rn[i] = g_rng.next();
  return QQ_OK;
}

int sources_z(qq_ctx* c, double* be, double* bo, bool z4) {
  if (!g_rng.seeded()) return set_error(QQ_BAD_ARG, "qq_initlagfib has not been called");
  std::vector<double> e(c->ref_doubles()), o(c->ref_doubles());
  noise_half(c->rd, e.data(), z4);
  noise_half(c->rd, o.data(), z4);
  QQ_TRY(write_out(c, be, e));
  return write_out(c, bo, o);
}

// Q/quark.f90:46-108: unit entry at global site src (1-based), colour icsrc, spin idsrc.
int sources_point(qq_ctx* c, double* be, double* bo, const int src[4], int icsrc, int idsrc) {
  std::vector<double> e(c->ref_doubles(), 0.0), o(c->ref_doubles(), 0.0);
  int x[4];
  for (int mu = 0; mu < 4; ++mu) {
    x[mu] = src[mu] - 1;
    if (x[mu] < 0 || x[mu] >= c->g.n[mu]) return set_error(QQ_BAD_ARG, "source outside the lattice");
  }
  int isite, ieo, ibleo;
  ref_site(c->g, x, &isite, &ieo, &ibleo);
  const int parity = (x[0] + x[1] + x[2] + x[3]) & 1;
  (parity == 0 ? e : o)[ref_gi(c->rd, 2 * icsrc - 1, isite, idsrc, ieo, ibleo)] = 1.0;
  QQ_TRY(write_out(c, be, e));
  return write_out(c, bo, o);
}

}  // namespace qq
