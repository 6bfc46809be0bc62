// Real-space Ewald term and the self / net-charge corrections: the parts of
// the Ewald energy beside the reciprocal sum (notes.tex:68-79).
//
// With the reference's influence function f(z) = exp(-z pi^2/eta^2)/(pi z)
// (ewald.py:124-132), the reciprocal energy (1/2V) sum f(m^2)|S(m)|^2 is the
// long-range part of the Coulomb energy (CGS) split by erfc(eta r)/r:
//   E_real = 1/2 sum_{i != j, |r_ij| < rcut} q_i q_j erfc(eta r_ij) / r_ij
//            (minimum image: rcut <= half the smallest box width),
//   E_self = -eta/sqrt(pi) sum q^2            (notes.tex:73-77),
//   E_net  = -pi (sum q)^2 / (2 V eta^2)      (neutralising background;
//                                              "further corrections are
//                                              needed if sum q != 0").
// E_recip + E_real + E_self + E_net does not depend on eta.
//
// Layout: the points are cell-sorted on a coarse grid whose cells are at
// least rcut/kRealSub wide (the same counting sort as the charge grid's, with
// coarse dimensions).  One warp takes 32 consecutive sorted points; the
// points of one coarse row (x, y cell) share their neighbourhood, so the warp
// walks, once for all its lanes, the union of their neighbour cells: the
// (2 kRealSub + 1)^2 neighbour rows (every row of an axis with fewer cells),
// each a contiguous z run [zlo - kRealSub, zhi + kRealSub] of the sorted
// order (zlo, zhi: the lanes' own z cells; the whole row when that run would
// wrap onto itself).  A warp whose points span several rows takes the rows
// one at a time with the other lanes masked.
//
// The candidates are concatenated into one stream and staged 64 at a time in
// shared memory (x, y in cell units relative to the warp's row, the z
// fraction and charge as a float4; the z cell relative to the warp's lowest z
// cell as a separate exact integer; the Cartesian position relative to the
// warp's first cell), read by broadcast: a reject pass over the 64 computes
// every lane's distance (Cartesian, against a cutoff widened by 1e-4 of rc^2
// to cover its rounding, when no image reduction is needed) and builds its
// bit masks of candidates inside, then each lane evaluates its accepted pairs
// one per round (erfc, exp), so the costly part runs on full lanes instead of
// on the few lanes a candidate happens to be near.  Every pair is visited
// from both sides, so each point's gradient has one writer and no atomics are
// needed.  Warps take their 32-point groups from a counter (groups differ in
// work: one or more rows, longer or shorter z runs), and every group writes
// its own energy / virial partials, summed in group order afterwards, so the
// result does not depend on which warp took which group.
//
// erfc(x) = exp(-x^2) erfcx(x): the exponential is the one the gradient needs
// anyway, and erfcx (smooth, between 1 and about 1/(x sqrt(pi))) is a
// cubic-Hermite table of kRealTab intervals on [0, min(eta rcut, 10)] built
// in FP64 per call and read from shared memory.
//
// Pair terms are FP32; each pair's energy is added in FP64 (the energy is a
// sum of terms of both signs that cancels to a small fraction of their
// magnitudes); gradient and virial terms are summed per staged batch in FP32
// and added to FP64 accumulators after each batch; energy and virial are
// reduced per group in FP64, then over groups in a fixed order
// (deterministic).  Separations are integer cell offsets plus the FP32
// in-cell fractions of the sort (about 1e-7 cells).  Pairs at zero separation
// (a point with itself, or two points at the same position) are skipped.
#include <algorithm>
#include <cmath>

#include "reduce.cuh"
#include "spme_kernels.hpp"

namespace spme {

constexpr int kRealWords = 16;  // per-group partials: e, W[6], q^2, q, pad
constexpr int kRealWarps = 4;   // warps per block of the pair kernel
constexpr int kRealBlocksPerSM = 6;
constexpr int kRealStage = 64;  // candidates staged per round of the walk

// Cubic-Hermite table of erfcx(x) = exp(x^2) erfc(x) on [0, xmax]: interval
// k holds f(k h + t h) = c.x + t (c.y + t (c.z + t c.w)), t in [0, 1].
__global__ void real_table_kernel(int ntab, double xmax, float4 *__restrict__ tab) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ntab) return;
  const double h = xmax / ntab, x0 = k * h, x1 = x0 + h;
  const double two_rsqrtpi = 1.1283791670955126;  // 2 / sqrt(pi)
  const double f0 = erfc(x0) * exp(x0 * x0), f1 = erfc(x1) * exp(x1 * x1);
  const double d0 = (2.0 * x0 * f0 - two_rsqrtpi) * h, d1 = (2.0 * x1 * f1 - two_rsqrtpi) * h;  // f' h
  tab[k] = make_float4((float)f0, (float)d0, (float)(3.0 * (f1 - f0) - 2.0 * d0 - d1),
                       (float)(2.0 * (f0 - f1) + d0 + d1));
}


// Coarse cell of every sorted point, packed c0 | c1 << 10 | c2 << 20; zeroes
// the pair kernel's group counter.
__global__ void __launch_bounds__(256) real_prep_kernel(int n, const uint32_t *__restrict__ keys, int nb1, int nb2,
                                                        int *__restrict__ cellc, int *__restrict__ next) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *next = 0;
  if (i >= n) return;
  const uint32_t key = keys[i];
  const int c2 = (int)(key % (uint32_t)nb2), r = (int)(key / (uint32_t)nb2);
  cellc[i] = (r / nb1) | ((r % nb1) << 10) | (c2 << 20);
}

struct RealArgs {
  int n, nb0, nb1, nb2;
  float inv0, inv1, inv2;        // 1 / nb
  float ax, by, cz, bx, cx, cy;  // lattice vectors per cell: a/nb0 = (ax,0,0), b/nb1 = (bx,by,0), c/nb2 = (cx,cy,cz)
  float eta, rc2;
  float rc2l;                    // rc2 widened past the rounding of the Cartesian reject test
  float tab_scale;               // erfcx table intervals per unit x
  int ngroups;                   // 32-point groups
  int *next;                     // group counter (zeroed by real_prep_kernel)
  const float4 *tab;             // erfcx table (kRealTab intervals)
  const float4 *rec;             // in-cell fractions (cells), charge; sorted
  const int *cellc;              // packed coarse cell; sorted
  const uint32_t *perm;
  const double *w;               // FP64 charges, input order (self and background sums)
  const int *cs;
  double *dx;                    // dE/dx in input order (n x 3), may be null
  double *partials;              // kRealWords per group
};

__device__ __forceinline__ int wrapc(int c, int nb) { return c < 0 ? c + nb : (c >= nb ? c - nb : c); }

// Per-lane state of the pair walk.
struct RealLane {
  float fx, fy, fz;  // own in-cell fractions
  float oz;          // own z cell relative to the warp's lowest z cell (exact small integer)
  float px, py, pz;  // own Cartesian position relative to the warp's row and lowest z cell
  float q;
  float g0, g1, g2, w[6];          // FP32 partial sums of the current chunk
  double E, G0, G1, G2, W[6];      // FP64 totals (E: every pair, in FP64)
};

// Minimum-image separation (cell units) of a staged candidate from lane L;
// WRAP reduces every axis modulo its cell count (axes with fewer than
// 2 kRealSub + 1 cells, or a z run that covers the whole row).
template <bool WRAP>
__device__ __forceinline__ float pair_r2(const RealArgs &A, const RealLane &L, float4 c, float cz, float &dxv,
                                         float &dyv, float &dzv) {
  // integer cell offset plus the difference of two in-cell fractions: exact
  // to the fractions' rounding for close pairs
  float t0 = c.x - L.fx, t1 = c.y - L.fy, t2 = (cz - L.oz) + (c.z - L.fz);
  if (WRAP) {
    t0 -= (float)A.nb0 * rintf(t0 * A.inv0);
    t1 -= (float)A.nb1 * rintf(t1 * A.inv1);
    t2 -= (float)A.nb2 * rintf(t2 * A.inv2);
  }
  dxv = t0 * A.ax + t1 * A.bx + t2 * A.cx;
  dyv = t1 * A.by + t2 * A.cy;
  dzv = t2 * A.cz;
  return dxv * dxv + dyv * dyv + dzv * dzv;
}

// Reject pass over 32 staged candidates: the bit mask of those inside the
// cutoff (zero separations are dropped later).
template <bool WRAP>
__device__ __forceinline__ unsigned real_reject(const RealArgs &A, const RealLane &L, const float4 *__restrict__ cand,
                                                const float *__restrict__ candz, const float4 *__restrict__ cart) {
  unsigned mask = 0;
  if (WRAP) {
#pragma unroll 8
    for (int k = 0; k < 32; k++) {
      float dxv, dyv, dzv;
      const float r2 = pair_r2<WRAP>(A, L, cand[k], candz[k], dxv, dyv, dzv);
      mask |= (r2 < A.rc2) ? (1u << k) : 0u;
    }
  } else {
    // no image reduction: a plain Cartesian distance against the widened
    // cutoff; the accepted pairs are tested again from the exact separation.
    // Eight candidates per byte of the mask, each with a constant bit.
#pragma unroll 1
    for (int k0 = 0; k0 < 32; k0 += 8) {
      unsigned byte = 0;
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const float4 p = cart[k0 + c];
        const float ddx = p.x - L.px, ddy = p.y - L.py, ddz = p.z - L.pz;
        const float r2 = ddx * ddx + ddy * ddy + ddz * ddz;
        byte |= (r2 < A.rc2l) ? (1u << c) : 0u;
      }
      mask |= byte << k0;
    }
  }
  return mask;
}

// One staged batch of kRealStage candidates: the reject passes, then the
// accepted pairs one per round (rounds: the most any lane accepted in the
// batch).  live0 / live1: the candidates of each half this lane takes (none
// for a lane outside the current row, none past the stream's end); two: the
// second half holds candidates (warp-uniform).
template <bool WRAP>
__device__ __forceinline__ void real_chunk(const RealArgs &A, RealLane &L, const float4 *__restrict__ cand,
                                           const float *__restrict__ candz, const float4 *__restrict__ cart,
                                           const float4 *__restrict__ tab, unsigned live0, unsigned live1,
                                           bool two) {
  unsigned m0 = real_reject<WRAP>(A, L, cand, candz, cart) & live0;
  unsigned m1 = two ? real_reject<WRAP>(A, L, cand + 32, candz + 32, cart + 32) & live1 : 0u;
  const float two_eta_sqrtpi = 1.1283791670955126f * A.eta;  // 2 eta / sqrt(pi)
  const float eta2 = A.eta * A.eta;
  while (m0 | m1) {
    int k;
    if (m0) {
      k = __ffs(m0) - 1;
      m0 &= m0 - 1;
    } else {
      k = 31 + __ffs(m1);
      m1 &= m1 - 1;
    }
    const float4 c = cand[k];
    float dxv, dyv, dzv;
    const float r2 = pair_r2<WRAP>(A, L, c, candz[k], dxv, dyv, dzv);
    if (!(r2 < A.rc2) || r2 == 0.f) continue;  // outside the cutoff; the point itself (or a coincident one)
    const float ir = rsqrtf(r2);
    const float ex = __expf(-eta2 * r2);  // exp(-x^2), x = eta r (error grows with x^2, where the term is small)
    const float u = A.eta * (r2 * ir) * A.tab_scale;
    const int ti = min((int)u, kRealTab - 1);
    const float tt = fminf(u - (float)ti, 1.f);
    const float4 cf = tab[ti];
    const float erfcx = fmaf(tt, fmaf(tt, fmaf(tt, cf.w, cf.z), cf.y), cf.x);
    const float phi = ex * erfcx * ir;  // erfc(eta r) / r
    const float qq = L.q * c.w;
    const float t = -qq * (two_eta_sqrtpi * ex + phi) * ir * ir;  // q q phi'(r) / r
    L.E += (double)(qq * phi);
    const float tx = t * dxv, ty = t * dyv, tz = t * dzv;
    L.g0 -= tx;
    L.g1 -= ty;
    L.g2 -= tz;
    L.w[0] = fmaf(tx, dxv, L.w[0]);
    L.w[1] = fmaf(ty, dyv, L.w[1]);
    L.w[2] = fmaf(tz, dzv, L.w[2]);
    L.w[3] = fmaf(ty, dxv, L.w[3]);
    L.w[4] = fmaf(tz, dxv, L.w[4]);
    L.w[5] = fmaf(tz, dyv, L.w[5]);
  }
  // chunk partials into the FP64 totals (each pair is visited from both
  // sides: half of the virial; the energy is halved at the end)
  L.G0 += (double)L.g0;
  L.G1 += (double)L.g1;
  L.G2 += (double)L.g2;
#pragma unroll
  for (int k = 0; k < 6; k++) L.W[k] += 0.5 * (double)L.w[k];
  L.g0 = L.g1 = L.g2 = 0.f;
#pragma unroll
  for (int k = 0; k < 6; k++) L.w[k] = 0.f;
}

// One 32-point group of sorted points per warp at a time, taken from the
// group counter; writes the group's partials.
__device__ __forceinline__ void real_group(const RealArgs &A, int grp, float4 *cand, float *candz, float4 *cart,
                                           const float4 *tab) {
  const int lane = threadIdx.x & 31;
  const int i = grp * 32 + lane;
  const bool valid = i < A.n;
  float4 ri = make_float4(0.f, 0.f, 0.f, 0.f);
  int c0 = 0, c1 = 0, c2 = 0, rowi = -1;
  if (valid) {
    ri = A.rec[i];
    const int pi = A.cellc[i];
    c0 = pi & 1023;
    c1 = (pi >> 10) & 1023;
    c2 = pi >> 20;
    rowi = (c0 << 10) | c1;
  }
  RealLane L;
  L.fx = ri.x;
  L.fy = ri.y;
  L.q = ri.w;
  L.g0 = L.g1 = L.g2 = 0.f;
  L.E = L.G0 = L.G1 = L.G2 = 0.0;
#pragma unroll
  for (int k = 0; k < 6; k++) {
    L.w[k] = 0.f;
    L.W[k] = 0.0;
  }
  const bool rel0 = A.nb0 >= 2 * kRealSub + 1, rel1 = A.nb1 >= 2 * kRealSub + 1;
  const int n0r = rel0 ? 2 * kRealSub + 1 : A.nb0, n1r = rel1 ? 2 * kRealSub + 1 : A.nb1;
  const int nrows = n0r * n1r;  // <= 25: one lane per neighbour row
  unsigned todo = __ballot_sync(0xffffffffu, valid);
  while (todo) {
    const int row = __shfl_sync(0xffffffffu, rowi, __ffs(todo) - 1);
    const bool act = rowi == row;
    todo &= ~__ballot_sync(0xffffffffu, act);
    const int rc0 = row >> 10, rc1 = row & 1023;
    const int zlo = __reduce_min_sync(0xffffffffu, act ? c2 : 0x7fffffff);
    const int zhi = __reduce_max_sync(0xffffffffu, act ? c2 : -1);
    const bool wholez = zhi - zlo + 2 * kRealSub + 1 >= A.nb2;
    const bool wrap = !rel0 || !rel1 || wholez;
    L.fz = ri.z;
    L.oz = (float)(c2 - zlo);
    {
      const float zc = L.oz + L.fz;
      L.px = L.fx * A.ax + L.fy * A.bx + zc * A.cx;
      L.py = L.fy * A.by + zc * A.cy;
      L.pz = zc * A.cz;
    }
    // this lane's neighbour row: offsets, pieces [s1, s1 + l1) and [s2, s2 + l2)
    // of the sorted order, with the z cell shifts that unwrap them
    int s1 = 0, l1 = 0, sh1 = 0, s2 = 0, l2 = 0, sh2 = 0;
    float o0 = 0.f, o1 = 0.f;
    if (lane < nrows) {
      const int r0 = lane / n1r, r1 = lane - r0 * n1r;
      const int nn0 = rel0 ? wrapc(rc0 + r0 - kRealSub, A.nb0) : r0;
      const int nn1 = rel1 ? wrapc(rc1 + r1 - kRealSub, A.nb1) : r1;
      o0 = (float)(rel0 ? r0 - kRealSub : r0 - rc0);
      o1 = (float)(rel1 ? r1 - kRealSub : r1 - rc1);
      const long rb = ((long)nn0 * A.nb1 + nn1) * A.nb2;
      if (wholez) {
        s1 = A.cs[rb];
        l1 = A.cs[rb + A.nb2] - s1;
      } else {
        const int za = zlo - kRealSub, zb = zhi + kRealSub;
        if (za < 0) {
          s1 = A.cs[rb + za + A.nb2];
          l1 = A.cs[rb + A.nb2] - s1;
          sh1 = -A.nb2;
          s2 = A.cs[rb];
          l2 = A.cs[rb + zb + 1] - s2;
        } else if (zb >= A.nb2) {
          s1 = A.cs[rb + za];
          l1 = A.cs[rb + A.nb2] - s1;
          s2 = A.cs[rb];
          l2 = A.cs[rb + zb + 1 - A.nb2] - s2;
          sh2 = A.nb2;
        } else {
          s1 = A.cs[rb + za];
          l1 = A.cs[rb + zb + 1] - s1;
        }
      }
    }
    // exclusive prefix of the rows' candidate counts
    int pre = l1 + l2;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, pre, o);
      if (lane >= o) pre += v;
    }
    const int total = __shfl_sync(0xffffffffu, pre, 31);
    pre -= l1 + l2;
    for (int v0 = 0; v0 < total; v0 += kRealStage) {
#pragma unroll
     for (int b = 0; b < kRealStage / 32; b++) {
      const int v = v0 + 32 * b + lane;
      float4 cv = make_float4(0.f, 0.f, 0.f, 0.f);  // past the end: masked out below
      float cvz = 0.f;
      float4 cvp = make_float4(0.f, 0.f, 0.f, 0.f);
      // row of stream position v: the last row whose prefix is <= v
      int r = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int pr = __shfl_sync(0xffffffffu, pre, r + step < nrows ? r + step : r);
        if (r + step < nrows && pr <= v) r += step;
      }
      const int rs1 = __shfl_sync(0xffffffffu, s1, r), rl1 = __shfl_sync(0xffffffffu, l1, r);
      const int rs2 = __shfl_sync(0xffffffffu, s2, r), rsh1 = __shfl_sync(0xffffffffu, sh1, r);
      const int rsh2 = __shfl_sync(0xffffffffu, sh2, r), rpre = __shfl_sync(0xffffffffu, pre, r);
      const float ro0 = __shfl_sync(0xffffffffu, o0, r), ro1 = __shfl_sync(0xffffffffu, o1, r);
      if (v < total) {
        const int loc = v - rpre;
        const int j = loc < rl1 ? rs1 + loc : rs2 + (loc - rl1);
        const int sh = loc < rl1 ? rsh1 : rsh2;
        const float4 rj = A.rec[j];
        const int cz = A.cellc[j] >> 20;
        cv = make_float4(ro0 + rj.x, ro1 + rj.y, rj.z, rj.w);
        cvz = (float)(cz + sh - zlo);
        const float zc = cvz + rj.z;
        cvp = make_float4(cv.x * A.ax + cv.y * A.bx + zc * A.cx, cv.y * A.by + zc * A.cy, zc * A.cz, 0.f);
      }
      cand[32 * b + lane] = cv;
      candz[32 * b + lane] = cvz;
      cart[32 * b + lane] = cvp;
     }
      __syncwarp();
      const int cnt = total - v0;  // candidates left in the stream, > 0
      const unsigned live0 = act ? (cnt >= 32 ? 0xffffffffu : (1u << cnt) - 1u) : 0u;
      const unsigned live1 = (act && cnt > 32) ? (cnt >= 64 ? 0xffffffffu : (1u << (cnt - 32)) - 1u) : 0u;
      if (wrap)
        real_chunk<true>(A, L, cand, candz, cart, tab, live0, live1, cnt > 32);
      else
        real_chunk<false>(A, L, cand, candz, cart, tab, live0, live1, cnt > 32);
      __syncwarp();  // every lane has read the batch before the next one is staged
    }
  }
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = 0.0;
  if (valid) {
    const int a = (int)A.perm[i];
    if (A.dx) {
      A.dx[3 * a] = L.G0;
      A.dx[3 * a + 1] = L.G1;
      A.dx[3 * a + 2] = L.G2;
    }
    acc[0] = 0.5 * L.E;
#pragma unroll
    for (int k = 0; k < 6; k++) acc[1 + k] = L.W[k];
    const double q = A.w[a];
    acc[7] = q * q;
    acc[8] = q;
  }
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const double v = warp_sum(acc[k]);
    if (lane == k) A.partials[(long)grp * kRealWords + k] = v;
  }
}

__global__ void __launch_bounds__(kRealWarps * 32, kRealBlocksPerSM) real_pair_kernel(RealArgs A) {
  __shared__ float4 cand_all[kRealWarps][kRealStage];
  __shared__ float candz_all[kRealWarps][kRealStage];
  __shared__ float4 cart_all[kRealWarps][kRealStage];
  __shared__ float4 tab[kRealTab];
  for (int k = threadIdx.x; k < kRealTab; k += blockDim.x) tab[k] = A.tab[k];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    int grp = 0;
    if (lane == 0) grp = atomicAdd(A.next, 1);
    grp = __shfl_sync(0xffffffffu, grp, 0);
    if (grp >= A.ngroups) break;
    real_group(A, grp, cand_all[warp], candz_all[warp], cart_all[warp], tab);
  }
}

// out = [E_real, E_self, E_net, vir_real (xx, yy, zz, yx, zx, zy), vir_net
// (added to each diagonal component)], in de1's virial convention
// (vir = -W / V with W = sum_pairs q q phi'(r)/r r r^T).
__global__ void real_finish_kernel(const double *__restrict__ partials, int nblocks, const CellConst *__restrict__ cell,
                                   double eta, double *__restrict__ out) {
  __shared__ double tot[9];
  sum_partials<9>(partials, nblocks, kRealWords, tot);
  if (threadIdx.x != 0) return;
  const double iV = cell->iV;
  const double pi = 3.14159265358979323846;
  out[0] = tot[0];
  out[1] = -eta / sqrt(pi) * tot[7];
  out[2] = -pi * tot[8] * tot[8] * iV / (2.0 * eta * eta);
  for (int k = 0; k < 6; k++) out[3 + k] = -tot[1 + k] * iV;
  out[9] = -pi * tot[8] * tot[8] * iV * iV / (2.0 * eta * eta);
}

size_t real_partial_words(int cap) { return (size_t)((cap + 31) / 32 + 1) * kRealWords; }

int launch_real_space(const Geom &coarse, const double L[6], int n, const double *x, const double *w, float eta,
                      float rcut, SortBuffers &sb, double4 *rec, float4 *tab, double *dx, double *partials,
                      double eta_d, double *out, cudaStream_t st) {
  int k = launch_cell_sort(coarse, n, x, w, sb, st, 0);  // one bucket per coarse cell
  const int ngroups = (n + 31) / 32;
  if (n > 0) {
    int *cellc = reinterpret_cast<int *>(rec);  // rec holds n ints here
    int *next = reinterpret_cast<int *>(partials + (size_t)ngroups * kRealWords);  // past the group records
    real_prep_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, sb.keys[sb.cur], coarse.K1, coarse.K2, cellc, next);
    const double xmax = fmin(eta_d * (double)rcut, 10.0);  // exp(-x^2) is 0 in FP32 beyond x = 10
    real_table_kernel<<<(kRealTab + 127) / 128, 128, 0, st>>>(kRealTab, xmax, tab);
    RealArgs A{};
    A.n = n;
    A.nb0 = coarse.K0;
    A.nb1 = coarse.K1;
    A.nb2 = coarse.K2;
    A.inv0 = 1.f / (float)coarse.K0;
    A.inv1 = 1.f / (float)coarse.K1;
    A.inv2 = 1.f / (float)coarse.K2;
    A.ax = (float)(L[0] / coarse.K0);
    A.by = (float)(L[1] / coarse.K1);
    A.cz = (float)(L[2] / coarse.K2);
    A.bx = (float)(L[3] / coarse.K1);
    A.cx = (float)(L[4] / coarse.K2);
    A.cy = (float)(L[5] / coarse.K2);
    A.eta = eta;
    A.rc2 = rcut * rcut;
    A.rc2l = A.rc2 * 1.0001f;
    A.tab_scale = (float)(kRealTab / xmax);
    A.ngroups = ngroups;
    A.next = next;
    A.tab = tab;
    A.rec = sb.rec_sorted;
    A.cellc = cellc;
    A.perm = sb.vals[sb.cur];
    A.w = w;
    A.cs = sb.cell_start;
    A.dx = dx;
    A.partials = partials;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = std::min((ngroups + kRealWarps - 1) / kRealWarps, nsm * kRealBlocksPerSM);
    real_pair_kernel<<<blocks, kRealWarps * 32, 0, st>>>(A);
    k += 3;
  }
  real_finish_kernel<<<1, 9 * 32, 0, st>>>(partials, ngroups, coarse.cell, eta_d, out);
  return k + 1;
}

}  // namespace spme
