// K2: B-spline charge spreading (SFac::operator() + accum_spline,
// sfac.cpp:113-124,141-168).
//
// Owner-computes, like the reference: every grid point is written by exactly
// one thread, which sums the contributions of the atoms in the order^3
// neighbouring cells, cells in (i,j,k) order and atoms in sorted order.  No
// atomics anywhere, so the grid is bit-for-bit reproducible run to run.
#include "spme_kernels.hpp"

namespace spme {

// One thread per grid point (k1 fastest, so a warp reads 32 consecutive
// cell offsets per neighbour row: coalesced).
template <int P>
__global__ void __launch_bounds__(256) spread_owner_kernel(Geom g, Spline S,
                                                           const int *__restrict__ cell_start,
                                                           const float4 *__restrict__ rec,
                                                           float *__restrict__ grid) {
  const long npt = (long)g.K0 * g.K1 * g.K2;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= npt) return;
  const int k1 = (int)(gid % g.K2);
  const int j1 = (int)((gid / g.K2) % g.K1);
  const int i1 = (int)(gid / ((long)g.K2 * g.K1));
  const int h = P / 2;
  float ans = 0.f;
#pragma unroll 1
  for (int i = 0; i < P; i++) {
    const int xid = imod(i1 - h + i, g.K0) * g.K1;
#pragma unroll 1
    for (int j = 0; j < P; j++) {
      const long yid = (long)(xid + imod(j1 - h + j, g.K1)) * g.K2;
#pragma unroll
      for (int k = 0; k < P; k++) {
        const long cid = yid + imod(k1 - h + k, g.K2);
        const int r0 = __ldg(cell_start + cid), r1 = __ldg(cell_start + cid + 1);
        for (int r = r0; r < r1; r++) {
          const float4 u = __ldg(rec + r);
          ans += bspl_eval(S, P, u.x, i) * bspl_eval(S, P, u.y, j) * bspl_eval(S, P, u.z, k) * u.w;
        }
      }
    }
  }
  grid[gid] = ans;
}

int launch_spread(const Geom &g, const Spline &S, const int *cell_start, const float4 *rec_sorted,
                  float *grid, cudaStream_t st) {
  const long npt = (long)g.K0 * g.K1 * g.K2;
  const int blocks = (int)((npt + 255) / 256);
  switch (g.order) {
    case 2: spread_owner_kernel<2><<<blocks, 256, 0, st>>>(g, S, cell_start, rec_sorted, grid); break;
    case 4: spread_owner_kernel<4><<<blocks, 256, 0, st>>>(g, S, cell_start, rec_sorted, grid); break;
    case 6: spread_owner_kernel<6><<<blocks, 256, 0, st>>>(g, S, cell_start, rec_sorted, grid); break;
    case 8: spread_owner_kernel<8><<<blocks, 256, 0, st>>>(g, S, cell_start, rec_sorted, grid); break;
    default: return 0;
  }
  return 1;
}

}  // namespace spme
