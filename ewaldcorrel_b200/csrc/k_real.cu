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
// coarse dimensions), then one thread per sorted point visits the points of
// the (2 kRealSub + 1)^3 neighbouring coarse cells (every cell of an axis
// with fewer): for each (x, y) neighbour row the z cells are one contiguous
// run of the sorted order.  Every pair is visited from both sides, so each
// point's gradient has one writer and no atomics are needed; energy and
// virial are reduced per block in FP64, then in a fixed order
// (deterministic).  Separations come from the integer cell offsets plus the
// FP32 in-cell fractions of the sort (about 1e-7 nm for pairs within the
// cutoff); pair terms are FP32 (erfc, exp); all sums are FP64.
#include <cmath>

#include "reduce.cuh"
#include "spme_kernels.hpp"

namespace spme {

constexpr int kRealWords = 16;  // per-block partials: e, W[6], q^2, q, pad


// Coarse cell of every sorted point, packed c0 | c1 << 10 | c2 << 20.
__global__ void __launch_bounds__(256) real_prep_kernel(int n, const uint32_t *__restrict__ keys, int nb1, int nb2,
                                                        int *__restrict__ cellc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t key = keys[i];
  const int c2 = (int)(key % (uint32_t)nb2), r = (int)(key / (uint32_t)nb2);
  cellc[i] = (r / nb1) | ((r % nb1) << 10) | (c2 << 20);
}

struct RealArgs {
  int n, nb0, nb1, nb2;
  float inv0, inv1, inv2;         // 1 / nb
  float ax, by, cz, bx, cx, cy;   // lattice vectors a = (ax,0,0), b = (bx,by,0), c = (cx,cy,cz)
  float eta, rc2;
  const float4 *rec;              // in-cell fractions (cells), charge; sorted
  const int *cellc;               // packed coarse cell; sorted
  const uint32_t *perm;
  const double *w;                // FP64 charges, input order (self and background sums)
  const int *cs;
  double *dx;                     // dE/dx in input order (n x 3), may be null
  double *partials;               // kRealWords per block
};

__device__ __forceinline__ int wrapc(int c, int nb) { return c < 0 ? c + nb : (c >= nb ? c - nb : c); }

// Cells of one axis to visit around cell c: [c - kRealSub, c + kRealSub] when
// the axis has at least 2 kRealSub + 1 cells (all distinct), else every cell.
struct AxisRange {
  int lo, hi;  // inclusive offsets (relative when `rel`, absolute cells otherwise)
  bool rel;
};
__device__ __forceinline__ AxisRange axis_range(int nb) {
  return nb >= 2 * kRealSub + 1 ? AxisRange{-kRealSub, kRealSub, true} : AxisRange{0, nb - 1, false};
}

__global__ void __launch_bounds__(256) real_pair_kernel(RealArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = 0.0;
  if (i < A.n) {
    const float4 ri = A.rec[i];
    const int pi = A.cellc[i];
    const int c0 = pi & 1023, c1 = (pi >> 10) & 1023, c2 = pi >> 20;
    const AxisRange R0 = axis_range(A.nb0), R1 = axis_range(A.nb1), R2 = axis_range(A.nb2);
    const float two_eta_sqrtpi = 1.1283791670955126f * A.eta;  // 2 eta / sqrt(pi)
    const float eta2 = A.eta * A.eta;
    double e = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, W[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    // one contiguous run of sorted points
    auto run = [&](int j0, int j1) {
      for (int j = j0; j < j1; j++) {
        if (j == i) continue;
        const float4 rj = A.rec[j];
        const int pj = A.cellc[j];
        // minimum-image separation in cells: integer cell difference plus the
        // in-cell fractions, reduced modulo the axis (exact for the small
        // differences of pairs within the cutoff)
        float t0 = (float)((pj & 1023) - c0) + (rj.x - ri.x);
        float t1 = (float)(((pj >> 10) & 1023) - c1) + (rj.y - ri.y);
        float t2 = (float)((pj >> 20) - c2) + (rj.z - ri.z);
        t0 -= (float)A.nb0 * rintf(t0 * A.inv0);
        t1 -= (float)A.nb1 * rintf(t1 * A.inv1);
        t2 -= (float)A.nb2 * rintf(t2 * A.inv2);
        const float s0 = t0 * A.inv0, s1 = t1 * A.inv1, s2 = t2 * A.inv2;
        const float dxv = s0 * A.ax + s1 * A.bx + s2 * A.cx;
        const float dyv = s1 * A.by + s2 * A.cy;
        const float dzv = s2 * A.cz;
        const float r2 = dxv * dxv + dyv * dyv + dzv * dzv;
        if (r2 >= A.rc2) continue;
        const float r = sqrtf(r2), ir = 1.f / r;
        const float ec = erfcf(A.eta * r);
        const float phi = ec * ir;                                           // erfc(eta r) / r
        const float dphi = -(two_eta_sqrtpi * expf(-eta2 * r2) + phi) * ir;  // d phi / dr
        const float qq = ri.w * rj.w;
        e += 0.5 * (double)(qq * phi);
        const float t = qq * dphi * ir;  // q q phi'(r) / r
        g0 -= (double)(t * dxv);
        g1 -= (double)(t * dyv);
        g2 -= (double)(t * dzv);
        const float h = 0.5f * t;  // each pair is visited from both sides
        W[0] += (double)(h * dxv * dxv);
        W[1] += (double)(h * dyv * dyv);
        W[2] += (double)(h * dzv * dzv);
        W[3] += (double)(h * dyv * dxv);
        W[4] += (double)(h * dzv * dxv);
        W[5] += (double)(h * dzv * dyv);
      }
    };
    for (int d0 = R0.lo; d0 <= R0.hi; d0++) {
      const int n0 = R0.rel ? wrapc(c0 + d0, A.nb0) : d0;
      for (int d1 = R1.lo; d1 <= R1.hi; d1++) {
        const int n1 = R1.rel ? wrapc(c1 + d1, A.nb1) : d1;
        const long row = ((long)n0 * A.nb1 + n1) * A.nb2;
        if (!R2.rel) {
          run(A.cs[row], A.cs[row + A.nb2]);  // the whole row
        } else {
          // z cells c2 - Sub .. c2 + Sub: contiguous in the sorted order, in at
          // most two pieces when they wrap
          const int za = c2 - kRealSub, zb = c2 + kRealSub;
          if (za < 0) {
            run(A.cs[row + za + A.nb2], A.cs[row + A.nb2]);
            run(A.cs[row], A.cs[row + zb + 1]);
          } else if (zb >= A.nb2) {
            run(A.cs[row + za], A.cs[row + A.nb2]);
            run(A.cs[row], A.cs[row + zb + 1 - A.nb2]);
          } else {
            run(A.cs[row + za], A.cs[row + zb + 1]);
          }
        }
      }
    }
    const int a = (int)A.perm[i];
    if (A.dx) {
      A.dx[3 * a] = g0;
      A.dx[3 * a + 1] = g1;
      A.dx[3 * a + 2] = g2;
    }
    acc[0] = e;
#pragma unroll
    for (int k = 0; k < 6; k++) acc[1 + k] = W[k];
    const double q = A.w[a];
    acc[7] = q * q;
    acc[8] = q;
  }
  __shared__ double red[8][9];
  block_reduce_n<9>(acc, red, A.partials + (long)blockIdx.x * kRealWords);
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

size_t real_partial_words(int cap) { return (size_t)((cap + 255) / 256 + 1) * kRealWords; }

int launch_real_space(const Geom &coarse, const double L[6], int n, const double *x, const double *w, float eta,
                      float rcut, SortBuffers &sb, double4 *rec, double *dx, double *partials, double eta_d,
                      double *out, cudaStream_t st) {
  int k = launch_cell_sort(coarse, n, x, w, sb, st);
  const int blocks = (n + 255) / 256;
  if (n > 0) {
    int *cellc = reinterpret_cast<int *>(rec);  // rec holds n ints here
    real_prep_kernel<<<blocks, 256, 0, st>>>(n, sb.keys[sb.cur], coarse.K1, coarse.K2, cellc);
    RealArgs A{};
    A.n = n;
    A.nb0 = coarse.K0;
    A.nb1 = coarse.K1;
    A.nb2 = coarse.K2;
    A.inv0 = 1.f / (float)coarse.K0;
    A.inv1 = 1.f / (float)coarse.K1;
    A.inv2 = 1.f / (float)coarse.K2;
    A.ax = (float)L[0];
    A.by = (float)L[1];
    A.cz = (float)L[2];
    A.bx = (float)L[3];
    A.cx = (float)L[4];
    A.cy = (float)L[5];
    A.eta = eta;
    A.rc2 = rcut * rcut;
    A.rec = sb.rec_sorted;
    A.cellc = cellc;
    A.perm = sb.vals[sb.cur];
    A.w = w;
    A.cs = sb.cell_start;
    A.dx = dx;
    A.partials = partials;
    real_pair_kernel<<<blocks, 256, 0, st>>>(A);
    k += 2;
  }
  real_finish_kernel<<<1, 9 * 32, 0, st>>>(partials, blocks, coarse.cell, eta_d, out);
  return k + 1;
}

}  // namespace spme
