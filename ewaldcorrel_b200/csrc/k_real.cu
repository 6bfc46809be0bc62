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
// least rcut wide (the same counting sort as the charge grid's, with coarse
// dimensions), then one thread per sorted point visits the points of the 27
// (or fewer, for grids under 3 cells wide) neighbouring coarse cells.  Every
// pair is visited from both sides, so each point's gradient has one writer
// and no atomics are needed; energy and virial are reduced per block in
// FP64, then in a fixed order (deterministic).  Pair terms are FP32 (erfc,
// exp) on FP64 minimum-image displacements; all sums are FP64.
#include <cmath>

#include "reduce.cuh"
#include "spme_kernels.hpp"

namespace spme {

constexpr int kRealWords = 16;  // per-block partials: e, W[6], q^2, q, pad

// Sorted records: FP64 wrapped fractional coordinates and charge.
__global__ void __launch_bounds__(256) real_prep_kernel(int n, const CellConst *__restrict__ cell,
                                                        const double *__restrict__ x, const double *__restrict__ w,
                                                        const uint32_t *__restrict__ perm, double4 *__restrict__ rec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const CellConst c = *cell;
  const int a = (int)perm[i];
  double s0, s1, s2;
  frac_coords(c, x[3 * a], x[3 * a + 1], x[3 * a + 2], s0, s1, s2);
  rec[i] = make_double4(s0, s1, s2, w[a]);
}

struct RealArgs {
  int n, nb0, nb1, nb2;
  double ax, by, cz, bx, cx, cy;  // lattice vectors a = (ax,0,0), b = (bx,by,0), c = (cx,cy,cz)
  float eta, rc2;
  const double4 *rec;
  const uint32_t *keys, *perm;
  const int *cs;
  double *dx;        // dE/dx in input order (n x 3), may be null
  double *partials;  // kRealWords per block
};

__device__ __forceinline__ int wrapc(int c, int nb) { return c < 0 ? c + nb : (c >= nb ? c - nb : c); }

__global__ void __launch_bounds__(256) real_pair_kernel(RealArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = 0.0;
  if (i < A.n) {
    const double4 ri = A.rec[i];
    const uint32_t key = A.keys[i];
    const int c2 = (int)(key % (uint32_t)A.nb2), r01 = (int)(key / (uint32_t)A.nb2);
    const int c1 = r01 % A.nb1, c0 = r01 / A.nb1;
    const int lo0 = A.nb0 >= 3 ? -1 : 0, hi0 = A.nb0 >= 3 ? 1 : A.nb0 - 1;
    const int lo1 = A.nb1 >= 3 ? -1 : 0, hi1 = A.nb1 >= 3 ? 1 : A.nb1 - 1;
    const int lo2 = A.nb2 >= 3 ? -1 : 0, hi2 = A.nb2 >= 3 ? 1 : A.nb2 - 1;
    const float two_eta_sqrtpi = 1.1283791670955126f * A.eta;  // 2 eta / sqrt(pi)
    const float eta2 = A.eta * A.eta;
    double e = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, W[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int d0 = lo0; d0 <= hi0; d0++) {
      const int n0 = (A.nb0 >= 3) ? wrapc(c0 + d0, A.nb0) : d0;
      for (int d1 = lo1; d1 <= hi1; d1++) {
        const int n1 = (A.nb1 >= 3) ? wrapc(c1 + d1, A.nb1) : d1;
        const long row = ((long)n0 * A.nb1 + n1) * A.nb2;
        for (int d2 = lo2; d2 <= hi2; d2++) {
          const int n2 = (A.nb2 >= 3) ? wrapc(c2 + d2, A.nb2) : d2;
          const int j0 = A.cs[row + n2], j1 = A.cs[row + n2 + 1];
          for (int j = j0; j < j1; j++) {
            if (j == i) continue;
            const double4 rj = A.rec[j];
            double s0 = rj.x - ri.x, s1 = rj.y - ri.y, s2 = rj.z - ri.z;
            s0 -= rint(s0);
            s1 -= rint(s1);
            s2 -= rint(s2);
            const double dxv = s0 * A.ax + s1 * A.bx + s2 * A.cx;
            const double dyv = s1 * A.by + s2 * A.cy;
            const double dzv = s2 * A.cz;
            const float r2 = (float)(dxv * dxv + dyv * dyv + dzv * dzv);
            if (r2 >= A.rc2) continue;
            const float r = sqrtf(r2), ir = 1.f / r;
            const float ec = erfcf(A.eta * r);
            const float phi = ec * ir;                                           // erfc(eta r) / r
            const float dphi = -(two_eta_sqrtpi * expf(-eta2 * r2) + phi) * ir;  // d phi / dr
            const double qq = ri.w * rj.w;
            e += 0.5 * qq * (double)phi;
            const double t = qq * (double)(dphi * ir);  // q q phi'(r) / r
            g0 -= t * dxv;
            g1 -= t * dyv;
            g2 -= t * dzv;
            const double h = 0.5 * t;  // each pair is visited from both sides
            W[0] += h * dxv * dxv;
            W[1] += h * dyv * dyv;
            W[2] += h * dzv * dzv;
            W[3] += h * dyv * dxv;
            W[4] += h * dzv * dxv;
            W[5] += h * dzv * dyv;
          }
        }
      }
    }
    if (A.dx) {
      const int a = (int)A.perm[i];
      A.dx[3 * a] = g0;
      A.dx[3 * a + 1] = g1;
      A.dx[3 * a + 2] = g2;
    }
    acc[0] = e;
#pragma unroll
    for (int k = 0; k < 6; k++) acc[1 + k] = W[k];
    acc[7] = ri.w * ri.w;
    acc[8] = ri.w;
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
    real_prep_kernel<<<blocks, 256, 0, st>>>(n, coarse.cell, x, w, sb.vals[sb.cur], rec);
    RealArgs A{};
    A.n = n;
    A.nb0 = coarse.K0;
    A.nb1 = coarse.K1;
    A.nb2 = coarse.K2;
    A.ax = L[0];
    A.by = L[1];
    A.cz = L[2];
    A.bx = L[3];
    A.cx = L[4];
    A.cy = L[5];
    A.eta = eta;
    A.rc2 = rcut * rcut;
    A.rec = rec;
    A.keys = sb.keys[sb.cur];
    A.perm = sb.vals[sb.cur];
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
