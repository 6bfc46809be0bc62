// Shared definitions for the SPME reciprocal-space kernels (sm_100a).
//
// Grid conventions follow the reference (sfac.hpp:160-192):
//   real grid      [K0][K1][K2]      (x-major, z contiguous; unpadded here)
//   complex grid   [K0][K1][ldim]    ldim = K2/2 + 1 (half-complex last axis)
// Fractional coordinates s = iL^T x (Cell::scale, sfac.hpp:56-62) with the
// lower-triangular inverse box iL of Cell (sfac.hpp:37-52).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace spme {

constexpr int kMaxOrder = 8;  // MAX_SPL_ORDER (sfac.hpp:7); enforced here

// Box constants: iL lower triangle (Cell::iL) and 1/V, FP64, computed on the
// host with the reference's expressions (sfac.hpp:45-51).  Kernels read them
// from device memory, so a box change is a small copy, not new kernel
// arguments (a captured CUDA graph stays valid).
struct CellConst {
  double iL00, iL10, iL11, iL20, iL21, iL22, iV, pad;
};

// Grid constants passed by value to every kernel, plus the device address of
// the box constants.
struct Geom {
  int K0, K1, K2, ldim, order;
  const CellConst *cell;
};

// order x order polynomial table of the cardinal B-spline M_n: row j holds
// the Horner coefficients of M_n(t + j), t in [0,1) (BSpline, sfac.hpp:81-109).
struct Spline {
  float c[kMaxOrder * kMaxOrder];
};

__host__ __device__ inline int imod(int a, int b) { return ((a % b) + b) % b; }

// Index-checking build (-DSPME_CHECK).  SPME_IN(i, n, site) is true when
// 0 <= i < n.  Otherwise the module's error word records the first failure
// (site << 40 | the index's low 40 bits) and the caller skips the access:
// no trap, the context stays usable, and the host reads the word with
// sfac_check_take.  The product build compiles every check to `true`.
enum CheckSite : unsigned {
  CK_SORT_BUCKET = 0x101, CK_SORT_SCATTER, CK_SORT_FIXUP, CK_SORT_MERGE,
  CK_SPREAD_BUCKET = 0x201, CK_SPREAD_RANGE, CK_SPREAD_ATOM, CK_SPREAD_CASE, CK_SPREAD_ROW,
  CK_SPREAD_GRID,
  CK_GATHER_ATOM = 0x301, CK_GATHER_KEY, CK_GATHER_GRID,
  CK_FFT_LINE = 0x401, CK_FFT_CONV,
  CK_SERVE_ATOM = 0x501, CK_SERVE_OUT,
  CK_SELFTEST = 0xf01,
};
#ifdef SPME_CHECK
static __device__ unsigned long long spme_check_word;
__device__ __noinline__ static bool spme_check_fail(long long i, unsigned site) {
  const unsigned long long w = ((unsigned long long)site << 40) | ((unsigned long long)i & ((1ull << 40) - 1));
  atomicCAS(&spme_check_word, 0ull, w);
  return false;
}
#define SPME_IN(i, n, site)                                                                       \
  ((unsigned long long)(long long)(i) < (unsigned long long)(long long)(n) ? true                  \
                                                                            : spme::spme_check_fail( \
                                                                                  (long long)(i), (site)))
// Host: reads and clears this module's word (after the device is idle).
#define SPME_CHECK_READER(name)                                          \
  unsigned long long check_take_##name() {                               \
    unsigned long long v = 0, z = 0;                                     \
    if (cudaMemcpyFromSymbol(&v, spme_check_word, sizeof v) != cudaSuccess) return 0; \
    if (v) cudaMemcpyToSymbol(spme_check_word, &z, sizeof z);           \
    return v;                                                            \
  }
#else
#define SPME_IN(i, n, site) true
#define SPME_CHECK_READER(name) \
  unsigned long long check_take_##name() { return 0; }
#endif

// Division by a runtime-invariant positive integer d with a multiply-high and
// a shift (the round-up multiplier method of Granlund and Montgomery): for
// 0 <= x < 2^31, q = umulhi(x, m) >> s equals x / d exactly.
struct FastDiv {
  uint32_t d, m, s;
  __host__ __device__ FastDiv() : d(1), m(0), s(0) {}
  __host__ explicit FastDiv(uint32_t d_) : d(d_), m(0), s(0) {
    if (d <= 1) return;
    uint32_t l = 0;
    while ((1ull << l) < d) l++;  // ceil(log2 d)
    const uint64_t p = 31 + l;
    m = (uint32_t)(((1ull << p) + d - 1) / d);
    s = (uint32_t)(p - 32);
  }
  __device__ __forceinline__ uint32_t div(uint32_t x) const { return d <= 1 ? x : (__umulhi(x, m) >> s); }
  __device__ __forceinline__ void divmod(uint32_t x, uint32_t &q, uint32_t &r) const {
    q = div(x);
    r = x - q * d;
  }
};

// M_n(t + j) by Horner (BSpline::bspl_coef, sfac.hpp:124-131), FP32.
__device__ __forceinline__ float bspl_eval(const Spline &S, int n, float t, int j) {
  const float *r = S.c + j * n;
  float b = r[0];
#pragma unroll 8
  for (int i = 1; i < kMaxOrder; i++)
    if (i < n) b = fmaf(b, t, r[i]);
  return b;
}

// Value and derivative (BSpline::dbspl_coef, sfac.hpp:146-157), FP32.
__device__ __forceinline__ void dbspl_eval(const Spline &S, int n, float t, int j,
                                           float &b, float &db) {
  const float *r = S.c + j * n;
  float d = r[0];
  float v = fmaf(r[0], t, r[1]);
#pragma unroll 8
  for (int i = 2; i < kMaxOrder; i++)
    if (i < n) {
      d = fmaf(d, t, v);
      v = fmaf(v, t, r[i]);
    }
  b = v;
  db = d;
}

// Fractional coordinate component, rounded exactly as Cell::scale computes
// it on the host: ((x0*a + x1*b) + x2*c), no FMA contraction, then wrap.
__device__ __forceinline__ double wrap01_rn(double v) { return __dsub_rn(v, floor(v)); }

__device__ __forceinline__ void frac_coords(const CellConst &g, double x0, double x1, double x2,
                                            double &s0, double &s1, double &s2) {
  s0 = wrap01_rn(__dadd_rn(__dadd_rn(__dmul_rn(x0, g.iL00), __dmul_rn(x1, g.iL10)),
                           __dmul_rn(x2, g.iL20)));
  s1 = wrap01_rn(__dadd_rn(__dmul_rn(x1, g.iL11), __dmul_rn(x2, g.iL21)));
  s2 = wrap01_rn(__dmul_rn(x2, g.iL22));
}

// Host: box constants from L = [ax, by, cz, bx, cx, cy] (Cell, sfac.hpp:37-52),
// same expressions and operation order, so device keys round like the host's.
inline CellConst make_cell(const double L[6]) {
  CellConst c{};
  c.iV = 1. / (L[0] * L[1] * L[2]);
  c.iL00 = 1. / L[0];
  c.iL11 = 1. / L[1];
  c.iL22 = 1. / L[2];
  c.iL10 = -L[3] * L[2] * c.iV;
  c.iL20 = (L[3] * L[5] - L[1] * L[4]) * c.iV;
  c.iL21 = -L[0] * L[5] * c.iV;
  return c;
}

}  // namespace spme
