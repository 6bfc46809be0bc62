// K6: force and potential gather (de2, sfac.cpp:409-483; potl,
// sfac.cpp:497-545).
//
// One thread per point, so every output has exactly one writer and the sum
// order is fixed.  The stencil origin is computed in FP64 exactly as the
// reference does (u = scale(x)*K, k1 = ceil(u), k0 = (k1 - order/2) mod K);
// the B-spline weights and the order^3 sum are FP32, factorised as
// sum_i wx_i sum_j wy_j sum_k wz_k Q  (one pass gives phi and all three
// derivatives).  The chain rule through iL and the scaling are FP64.
#include "spme_kernels.hpp"

namespace spme {

template <int P, bool GRAD, bool POT>
__global__ void __launch_bounds__(256) gather_kernel(Geom g, Spline S, int n, const double *__restrict__ x,
                                                     const double *__restrict__ w,
                                                     const float *__restrict__ grid, double *__restrict__ dx,
                                                     double *__restrict__ phi) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  double s0, s1, s2;
  frac_coords(g, x[3 * a + 0], x[3 * a + 1], x[3 * a + 2], s0, s1, s2);
  const double u0 = __dmul_rn(s0, (double)g.K0), u1 = __dmul_rn(s1, (double)g.K1),
               u2 = __dmul_rn(s2, (double)g.K2);
  const int c0 = (int)ceil(u0), c1 = (int)ceil(u1), c2 = (int)ceil(u2);
  const float t0 = (float)((double)c0 - u0), t1 = (float)((double)c1 - u1), t2 = (float)((double)c2 - u2);
  const int o0 = imod(c0 - P / 2, g.K0), o1 = imod(c1 - P / 2, g.K1), o2 = imod(c2 - P / 2, g.K2);
  float wx[P], dwx[P], wy[P], dwy[P], wz[P], dwz[P];
  int iz[P];
#pragma unroll
  for (int i = 0; i < P; i++) {
    dbspl_eval(S, P, t0, i, wx[i], dwx[i]);
    dbspl_eval(S, P, t1, i, wy[i], dwy[i]);
    dbspl_eval(S, P, t2, i, wz[i], dwz[i]);
    iz[i] = (o2 + i) % g.K2;
  }
  float pot = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll 1
  for (int i = 0; i < P; i++) {
    const long row_x = (long)((o0 + i) % g.K0) * g.K1;
    float sy = 0.f, dy = 0.f, dz = 0.f;
#pragma unroll
    for (int j = 0; j < P; j++) {
      const float *col = grid + (row_x + (o1 + j) % g.K1) * g.K2;
      float sz = 0.f, dzz = 0.f;
#pragma unroll
      for (int k = 0; k < P; k++) {
        const float q = __ldg(col + iz[k]);
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
  if (GRAD) {
    const double f = -w[a] * g.iV;
    const double G0 = (double)gx * f * g.K0, G1 = (double)gy * f * g.K1, G2 = (double)gz * f * g.K2;
    dx[3 * a + 0] = g.iL00 * G0;
    dx[3 * a + 1] = g.iL10 * G0 + g.iL11 * G1;
    dx[3 * a + 2] = g.iL20 * G0 + g.iL21 * G1 + g.iL22 * G2;
  }
  if (POT) phi[a] = (double)pot * g.iV;
}

template <int P>
static int gather_p(const Geom &g, const Spline &S, int n, const double *x, const double *w,
                     const float *grid, double *dx, double *phi, cudaStream_t st) {
  const int blocks = (n + 255) / 256;
  if (dx && phi) gather_kernel<P, true, true><<<blocks, 256, 0, st>>>(g, S, n, x, w, grid, dx, phi);
  else if (dx) gather_kernel<P, true, false><<<blocks, 256, 0, st>>>(g, S, n, x, w, grid, dx, phi);
  else if (phi) gather_kernel<P, false, true><<<blocks, 256, 0, st>>>(g, S, n, x, w, grid, dx, phi);
  else return 0;
  return 1;
}

int launch_gather(const Geom &g, const Spline &S, int n, const double *x, const double *w,
                  const float *grid, double *dx, double *phi, cudaStream_t st) {
  if (n <= 0) return 0;
  switch (g.order) {
    case 2: return gather_p<2>(g, S, n, x, w, grid, dx, phi, st);
    case 4: return gather_p<4>(g, S, n, x, w, grid, dx, phi, st);
    case 6: return gather_p<6>(g, S, n, x, w, grid, dx, phi, st);
    case 8: return gather_p<8>(g, S, n, x, w, grid, dx, phi, st);
    default: return 0;
  }
}

}  // namespace spme
