// K6: force and potential gather (de2, sfac.cpp:409-483; potl,
// sfac.cpp:497-545).
//
// One thread per point, so every output has exactly one writer and the sum
// order is fixed.  The stencil origin is computed in FP64 exactly as the
// reference does (u = scale(x)*K, k1 = ceil(u), k0 = (k1 - order/2) mod K);
// the B-spline weights and the order^3 sum are FP32, factorised as
// sum_i wx_i sum_j wy_j sum_k wz_k Q  (one pass gives phi and all three
// derivatives).  The chain rule through iL and the scaling are FP64.
#include "reduce.cuh"
#include "spme_kernels.hpp"

namespace spme {

SPME_CHECK_READER(gather)

constexpr int kCellWords = 16;  // 9 used: sum_a s_a,i (dE/dr_a)_j

// idx[i] = (o + i) mod K for 0 <= o < K, without a division when K >= P.
template <int P>
__device__ __forceinline__ void wrap_run(int o, int K, int (&idx)[P]) {
  if (K >= P) {
#pragma unroll
    for (int i = 0; i < P; i++) {
      const int v = o + i;
      idx[i] = v >= K ? v - K : v;
    }
  } else {
#pragma unroll
    for (int i = 0; i < P; i++) idx[i] = (o + i) % K;
  }
}

// Order-P stencil sum of the grid around one point, factorised per axis:
// pot = sum_i wx_i sum_j wy_j sum_k wz_k Q, and the three derivatives.
// WRAP false: the z indices are z0 .. z0 + P - 1; true: iz[k] (z0 = 0).
template <int P, bool WRAP>
__device__ __forceinline__ void stencil_sum(const float *__restrict__ grid, const Geom &g, int o0,
                                            const int (&iy)[P], int z0, const int (&iz)[P], const float (&wx)[P],
                                            const float (&dwx)[P], const float (&wy)[P], const float (&dwy)[P],
                                            const float (&wz)[P], const float (&dwz)[P], float &pot, float &gx,
                                            float &gy, float &gz) {
  const long plane = (long)g.K1 * g.K2;
  int xi = o0;  // (o0 + i) mod K0
#pragma unroll 1
  for (int i = 0; i < P; i++, xi = (xi + 1 == g.K0) ? 0 : xi + 1) {
    const float *pl = grid + xi * plane + z0;
    float sy = 0.f, dy = 0.f, dz = 0.f;
#pragma unroll
    for (int j = 0; j < P; j++) {
      const float *col = pl + (long)iy[j] * g.K2;
      float sz = 0.f, dzz = 0.f;
#pragma unroll
      for (int k = 0; k < P; k++) {
        const float q = SPME_IN(col + (WRAP ? iz[k] : k) - grid, g.K0 * plane, CK_GATHER_GRID)
                            ? __ldg(col + (WRAP ? iz[k] : k))
                            : 0.f;
        sz = fmaf(wz[k], q, sz);
        dzz = fmaf(dwz[k], q, dzz);
      }
      sy = fmaf(wy[j], sz, sy);
      dy = fmaf(dwy[j], sz, dy);
      dz = fmaf(wy[j], dzz, dz);
    }
    pot = fmaf(wx[i], sy, pot);
    gx = fmaf(dwx[i], sy, gx);
    gy = fmaf(wx[i], dy, gy);
    gz = fmaf(wx[i], dz, gz);
  }
}


// Vector width of the row loads: each z run of P values is read as W / kVW
// aligned float2 loads from zb = o2 rounded down to even (W = P + 2 values,
// the weights shifted by o2 - zb with zeros around the run).  4 loads instead
// of 6 per row at order 6 (fewer L1 requests); the extra terms are exact
// zeros, so the sums are bit-identical to the scalar ones.  float4 windows
// (3 loads of 12 values) measured no faster.
constexpr int kVW = 2;  // float2
template <int P> struct VecWin { static constexpr int W = (P + kVW - 1 + kVW - 1) / kVW * kVW; };

// Row sums from aligned vector loads: the window [zb, zb + W) holds the run,
// the weights are pre-shifted (zeros outside the run).
template <int P>
__device__ __forceinline__ void stencil_sum_vec(const float *__restrict__ grid, const Geom &g, int o0,
                                                const int (&iy)[P], int zb, const float (&wz)[VecWin<P>::W],
                                                const float (&dwz)[VecWin<P>::W], const float (&wx)[P],
                                                const float (&dwx)[P], const float (&wy)[P], const float (&dwy)[P],
                                                float &pot, float &gx, float &gy, float &gz) {
  constexpr int W = VecWin<P>::W;
  const long plane = (long)g.K1 * g.K2;
  int xi = o0;
#pragma unroll 1
  for (int i = 0; i < P; i++, xi = (xi + 1 == g.K0) ? 0 : xi + 1) {
    const float *pl = grid + xi * plane + zb;
    float sy = 0.f, dy = 0.f, dz = 0.f;
#pragma unroll
    for (int j = 0; j < P; j++) {
      const float *col = pl + (long)iy[j] * g.K2;
      float sz = 0.f, dzz = 0.f;
#pragma unroll
      for (int v = 0; v < W / kVW; v++) {
        const float2 q = SPME_IN(col + 2 * v + 1 - grid, g.K0 * plane, CK_GATHER_GRID)
                             ? __ldg(reinterpret_cast<const float2 *>(col) + v)
                             : make_float2(0.f, 0.f);
        sz = fmaf(wz[2 * v], q.x, sz); dzz = fmaf(dwz[2 * v], q.x, dzz);
        sz = fmaf(wz[2 * v + 1], q.y, sz); dzz = fmaf(dwz[2 * v + 1], q.y, dzz);
      }
      sy = fmaf(wy[j], sz, sy);
      dy = fmaf(dwy[j], sz, dy);
      dz = fmaf(wy[j], dzz, dz);
    }
    pot = fmaf(wx[i], sy, pot);
    gx = fmaf(dwx[i], sy, gx);
    gy = fmaf(wx[i], dy, gy);
    gz = fmaf(wx[i], dz, gz);
  }
}

// Cell-sorted view of the points (from the cell sort of the same solve):
// sorted rank r is point perm[r], in cell key[r] with in-cell fractions
// rec[r].xyz.  Consecutive threads then read neighbouring grid points.
struct SortedView {
  const uint32_t *perm, *key;
  const float4 *rec;
  FastDiv K2d, K12d;  // division by K2 and by K1*K2
};

// CELL: also the per-block sums of s_i (dE/dr)_j over the block's points
// (s = iL^T x, unwrapped), written to cellp[block][9] in a fixed order.
// SORTED: thread r handles point perm[r], with the stencil origin from its
// cell (k1 = n + 1, argument 1 - f; for f = 0 this is the reference's
// origin shifted by one cell, whose extra weight M(0) = 0 -- the same sum);
// otherwise the origin comes from x in FP64 exactly as de2/potl compute it.
template <int P, bool GRAD, bool POT, bool CELL, bool SORTED>
__global__ void __launch_bounds__(256, CELL ? 2 : 3) gather_kernel(Geom g, Spline S, int n, const double *__restrict__ x,
                                                     const double *__restrict__ w,
                                                     const float *__restrict__ grid, double *__restrict__ dx,
                                                     double *__restrict__ phi, double *__restrict__ cellp,
                                                     SortedView sv) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double cacc[9];
  if (CELL) {
#pragma unroll
    for (int c = 0; c < 9; c++) cacc[c] = 0.0;
  }
  if (r < n) {
    const CellConst cc = *g.cell;
    int a, o0, o1, o2;
    float t0, t1, t2;
    if (SORTED) {
      a = (int)sv.perm[r];
      uint32_t key = sv.key[r];
      // a failed check substitutes atom 0 / key 0 (the run is flagged already)
      if (!SPME_IN(a, n, CK_GATHER_ATOM)) a = 0;
      if (!SPME_IN(key, (long)g.K0 * g.K1 * g.K2, CK_GATHER_KEY)) key = 0;
      const float4 u = sv.rec[r];
      const uint32_t n0 = sv.K12d.div(key), rem = key - n0 * (uint32_t)(g.K1 * g.K2);
      const uint32_t n1 = sv.K2d.div(rem), n2 = rem - n1 * (uint32_t)g.K2;
      o0 = imod((int)n0 + 1 - P / 2, g.K0);
      o1 = imod((int)n1 + 1 - P / 2, g.K1);
      o2 = imod((int)n2 + 1 - P / 2, g.K2);
      t0 = 1.f - u.x;
      t1 = 1.f - u.y;
      t2 = 1.f - u.z;
    } else {
      a = r;
      double s0, s1, s2;
      frac_coords(cc, x[3 * a + 0], x[3 * a + 1], x[3 * a + 2], s0, s1, s2);
      const double u0 = __dmul_rn(s0, (double)g.K0), u1 = __dmul_rn(s1, (double)g.K1),
                   u2 = __dmul_rn(s2, (double)g.K2);
      const int c0 = (int)ceil(u0), c1 = (int)ceil(u1), c2 = (int)ceil(u2);
      t0 = (float)((double)c0 - u0);
      t1 = (float)((double)c1 - u1);
      t2 = (float)((double)c2 - u2);
      o0 = imod(c0 - P / 2, g.K0);
      o1 = imod(c1 - P / 2, g.K1);
      o2 = imod(c2 - P / 2, g.K2);
    }
    float wx[P], dwx[P], wy[P], dwy[P], wz[P], dwz[P];
#pragma unroll
    for (int i = 0; i < P; i++) {
      dbspl_eval(S, P, t0, i, wx[i], dwx[i]);
      dbspl_eval(S, P, t1, i, wy[i], dwy[i]);
      dbspl_eval(S, P, t2, i, wz[i], dwz[i]);
    }
    int iy[P];
    wrap_run<P>(o1, g.K1, iy);
    float pot = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    int iz[P];
    // Warp-uniform choice (no divergent second copy of the stencil): when no
    // active lane's z run wraps, constant offsets from one address per row.
    const int sh = o2 & (kVW - 1), zb = o2 - sh;
    if ((g.K2 % kVW) == 0 && __all_sync(__activemask(), zb + VecWin<P>::W <= g.K2)) {
      constexpr int W = VecWin<P>::W;
      float wzv[W], dwzv[W];
#pragma unroll
      for (int k = 0; k < W; k++) {
        float v = 0.f, d = 0.f;
#pragma unroll
        for (int t = 0; t < kVW; t++)
          if (k - t >= 0 && k - t < P) {
            v = (sh == t) ? wz[k - t] : v;
            d = (sh == t) ? dwz[k - t] : d;
          }
        wzv[k] = v;
        dwzv[k] = d;
      }
      stencil_sum_vec<P>(grid, g, o0, iy, zb, wzv, dwzv, wx, dwx, wy, dwy, pot, gx, gy, gz);
    } else if (__all_sync(__activemask(), o2 + P <= g.K2)) {
      stencil_sum<P, false>(grid, g, o0, iy, o2, iz, wx, dwx, wy, dwy, wz, dwz, pot, gx, gy, gz);
    } else {
      wrap_run<P>(o2, g.K2, iz);
      stencil_sum<P, true>(grid, g, o0, iy, 0, iz, wx, dwx, wy, dwy, wz, dwz, pot, gx, gy, gz);
    }
    if (GRAD) {
      const double f = -w[a] * cc.iV;
      const double G0 = (double)gx * f * g.K0, G1 = (double)gy * f * g.K1, G2 = (double)gz * f * g.K2;
      const double d0 = cc.iL00 * G0;
      const double d1 = cc.iL10 * G0 + cc.iL11 * G1;
      const double d2 = cc.iL20 * G0 + cc.iL21 * G1 + cc.iL22 * G2;
      dx[3 * a + 0] = d0;
      dx[3 * a + 1] = d1;
      dx[3 * a + 2] = d2;
      if (CELL) {
        const double x0 = x[3 * a + 0], x1 = x[3 * a + 1], x2 = x[3 * a + 2];
        const double v0 = x0 * cc.iL00 + x1 * cc.iL10 + x2 * cc.iL20;  // unwrapped s
        const double v1 = x1 * cc.iL11 + x2 * cc.iL21;
        const double v2 = x2 * cc.iL22;
        cacc[0] = v0 * d0; cacc[1] = v0 * d1; cacc[2] = v0 * d2;
        cacc[3] = v1 * d0; cacc[4] = v1 * d1; cacc[5] = v1 * d2;
        cacc[6] = v2 * d0; cacc[7] = v2 * d1; cacc[8] = v2 * d2;
      }
    }
    if (POT) phi[a] = (double)pot * cc.iV;
  }
  if (CELL) {
    __shared__ double red[8][9];
    block_reduce_n<9>(cacc, red, cellp + (long)blockIdx.x * kCellWords);
  }
}

// dE/dL (6: [ax, by, cz, bx, cx, cy]) at fixed Cartesian positions:
//   D = -V iL^T Pi - sum_a s_a (dE/dr_a)^T,  dE/dL = lower triangle of D,
// Pi the virial (symmetric, from ev[1..6]); the first term is dE/dL at fixed
// fractional coordinates (notes.tex: V Pi = -(dE/dL)^T L).
__global__ void cell_grad_kernel(Geom g, const double *__restrict__ cellp, int nblocks,
                                 const double *__restrict__ ev, double *__restrict__ dEdL) {
  __shared__ double P9[9];
  sum_partials<9>(cellp, nblocks, kCellWords, P9);
  if (threadIdx.x != 0) return;
  const CellConst c = *g.cell;
  const double iL[3][3] = {{c.iL00, 0.0, 0.0}, {c.iL10, c.iL11, 0.0}, {c.iL20, c.iL21, c.iL22}};
  const double Pi[3][3] = {{ev[1], ev[4], ev[5]}, {ev[4], ev[2], ev[6]}, {ev[5], ev[6], ev[3]}};
  const double V = 1.0 / c.iV;
  double D[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double gs = 0.0;
      for (int k = 0; k < 3; k++) gs += iL[k][i] * Pi[k][j];
      D[i][j] = -V * gs - P9[3 * i + j];
    }
  dEdL[0] = D[0][0];
  dEdL[1] = D[1][1];
  dEdL[2] = D[2][2];
  dEdL[3] = D[1][0];
  dEdL[4] = D[2][0];
  dEdL[5] = D[2][1];
}

template <int P, bool SORTED>
static int gather_p(const Geom &g, const Spline &S, int n, const double *x, const double *w, const float *grid,
                    double *dx, double *phi, double *cellp, const SortedView &sv, cudaStream_t st) {
  const int blocks = (n + 255) / 256;
  if (cellp)
    gather_kernel<P, true, true, true, SORTED><<<blocks, 256, 0, st>>>(g, S, n, x, w, grid, dx, phi, cellp, sv);
  else if (dx && phi)
    gather_kernel<P, true, true, false, SORTED><<<blocks, 256, 0, st>>>(g, S, n, x, w, grid, dx, phi, nullptr, sv);
  else if (dx)
    gather_kernel<P, true, false, false, SORTED><<<blocks, 256, 0, st>>>(g, S, n, x, w, grid, dx, phi, nullptr, sv);
  else if (phi)
    gather_kernel<P, false, true, false, SORTED><<<blocks, 256, 0, st>>>(g, S, n, x, w, grid, dx, phi, nullptr, sv);
  else return 0;
  return 1;
}

template <bool SORTED>
static int gather_any(const Geom &g, const Spline &S, int n, const double *x, const double *w, const float *grid,
                      double *dx, double *phi, double *cellp, const SortedView &sv, cudaStream_t st) {
  switch (g.order) {
    case 2: return gather_p<2, SORTED>(g, S, n, x, w, grid, dx, phi, cellp, sv, st);
    case 4: return gather_p<4, SORTED>(g, S, n, x, w, grid, dx, phi, cellp, sv, st);
    case 6: return gather_p<6, SORTED>(g, S, n, x, w, grid, dx, phi, cellp, sv, st);
    case 8: return gather_p<8, SORTED>(g, S, n, x, w, grid, dx, phi, cellp, sv, st);
    default: return 0;
  }
}

static SortedView make_view(const Geom &g, const uint32_t *perm, const uint32_t *keys, const float4 *rec) {
  SortedView sv{perm, keys, rec, FastDiv((uint32_t)g.K2), FastDiv((uint32_t)g.K1 * (uint32_t)g.K2)};
  return sv;
}

int launch_gather(const Geom &g, const Spline &S, int n, const double *x, const double *w,
                  const float *grid, double *dx, double *phi, cudaStream_t st, const uint32_t *perm,
                  const uint32_t *keys, const float4 *rec) {
  if (n <= 0) return 0;
  if (perm) return gather_any<true>(g, S, n, x, w, grid, dx, phi, nullptr, make_view(g, perm, keys, rec), st);
  return gather_any<false>(g, S, n, x, w, grid, dx, phi, nullptr, SortedView{}, st);
}

// Gather of dE/dx and phi (phi may be null) plus dE/dL; ev must already hold
// the energy and virial of this solve.  cellp: ceil(n/256) x kCellWords.
int launch_gather_cell(const Geom &g, const Spline &S, int n, const double *x, const double *w,
                       const float *grid, double *dx, double *phi, double *cellp, const double *ev, double *dEdL,
                       cudaStream_t st, const uint32_t *perm, const uint32_t *keys, const float4 *rec) {
  int k = 0;
  if (n > 0) {
    if (perm) k = gather_any<true>(g, S, n, x, w, grid, dx, phi, cellp, make_view(g, perm, keys, rec), st);
    else k = gather_any<false>(g, S, n, x, w, grid, dx, phi, cellp, SortedView{}, st);
  }
  cell_grad_kernel<<<1, 9 * 32, 0, st>>>(g, cellp, (n + 255) / 256, ev, dEdL);
  return k + 1;
}

size_t gather_cell_words(int cap) { return (size_t)((cap + 255) / 256 + 1) * kCellWords; }

}  // namespace spme
