// K4 + K7: B-spline moduli, influence function and the fused reciprocal
// convolution (en, sfac.cpp:304-325; de1, sfac.cpp:339-396; set_A,
// sfac.cpp:213-292; bspl_dft, sfac.cpp:21-35).
//
// The moduli, the influence function and the energy/virial reductions are
// FP64; the structure factor itself is FP32.  Reductions are deterministic:
// a fixed grid of kConvBlocks blocks walks the modes with a fixed stride,
// each block reduces with a fixed shuffle tree, and one final block sums the
// block partials in index order.  No atomics.
#include "spme_kernels.hpp"

namespace spme {

// iB[i] = 1 / sum_{j=1}^{order-1} cos(-2 pi i (j - order/2) / n) M_order(j)
// (bspl_dft, sfac.cpp:21-35; real because the order is even).
__global__ void bspline_moduli_kernel(int n, int order, SplineNodes nodes, double *iB) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double om = -(2.0 * 3.14159265358979323846 * i) / n;
  double x = 0.0;
  for (int j = 1; j < order; j++) x += cos(om * (j - order / 2)) * nodes.Mj[j];
  iB[i] = 1.0 / x;
}

int launch_bspline_moduli(int n, int order, const SplineNodes &nodes, double *iB, cudaStream_t st) {
  bspline_moduli_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, order, nodes, iB);
  return 1;
}

// Ewald influence function f(m^2) = exp(-pi^2 m^2 / beta^2) / (pi m^2) and
// f'(m^2) = (-pi^2/beta^2 - 1/m^2) f  (ewald.py:124-132; f(0) = 0).
__device__ __forceinline__ double ewald_f(double r2, double fac, double &fp) {
  if (r2 < 1e-10) {
    fp = 0.0;
    return 0.0;
  }
  const double f = exp(r2 * fac) / (r2 * 3.14159265358979323846);
  fp = (fac - 1.0 / r2) * f;
  return f;
}

// Sum of f and f' m_a m_b over the reciprocal vectors m = iL (i,j,k) with
// |m| < max_m whose lattice index is congruent to the stored mode
// (kx, ky, kz) -- the images set_A visits and folds onto this mode
// (sfac.cpp:240-289, same sphere bounds, FP64 without contraction).  The
// conjugate images that set_A folds onto interior modes have the same f
// values, so the caller doubles those instead of revisiting them.
__device__ void ewald_images(const Influence &inf, int K0, int K1, int K2, int kx, int ky, int kz,
                             double &sf, double sd[6]) {
  const double R2 = __dmul_rn(inf.max_m, inf.max_m);
  const double fac = -__dmul_rn(3.14159265358979323846 / inf.beta, 3.14159265358979323846 / inf.beta);
  const int i0 = __double2int_rz(__ddiv_rn(inf.max_m, inf.iL00));
  sf = 0.0;
  for (int c = 0; c < 6; c++) sd[c] = 0.0;
  for (int i = -i0 + imod(kx + i0, K0); i <= i0; i += K0) {
    const double mx = __dmul_rn((double)i, inf.iL00);
    const double m20 = __dmul_rn(mx, mx);
    const double dy = sqrt(fmax(__dsub_rn(R2, m20), 0.0));
    const double my0 = __dmul_rn((double)i, inf.iL10);
    const int j0 = (int)ceil(__ddiv_rn(__dsub_rn(-dy, my0), inf.iL11));
    const int j1 = (int)floor(__ddiv_rn(__dsub_rn(dy, my0), inf.iL11));
    for (int j = j0 + imod(ky - j0, K1); j <= j1; j += K1) {
      const double my = __dadd_rn(my0, __dmul_rn((double)j, inf.iL11));
      const double m21 = __dadd_rn(m20, __dmul_rn(my, my));
      const double dz = sqrt(fmax(__dsub_rn(R2, m21), 0.0));
      const double mz0 = __dadd_rn(__dmul_rn((double)i, inf.iL20), __dmul_rn((double)j, inf.iL21));
      const int k0 = (int)ceil(__ddiv_rn(__dsub_rn(-dz, mz0), inf.iL22));
      const int k1 = (int)floor(__ddiv_rn(__dsub_rn(dz, mz0), inf.iL22));
      for (int k = k0 + imod(kz - k0, K2); k <= k1; k += K2) {
        const double mz = __dadd_rn(mz0, __dmul_rn((double)k, inf.iL22));
        const double m2 = __dadd_rn(m21, __dmul_rn(mz, mz));
        double fp;
        sf += ewald_f(m2, fac, fp);
        sd[0] += fp * mx * mx;
        sd[1] += fp * my * my;
        sd[2] += fp * mz * mz;
        sd[3] += fp * my * mx;
        sd[4] += fp * mz * mx;
        sd[5] += fp * mz * my;
      }
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int MODE, bool SCALE>
__global__ void __launch_bounds__(256) conv_kernel(Geom g, Influence inf, const double *__restrict__ iB0,
                                                   const double *__restrict__ iB1,
                                                   const double *__restrict__ iB2, float2 *__restrict__ S,
                                                   double *__restrict__ partials) {
  const int ldim = g.ldim, K1 = g.K1;
  const long nm = (long)g.K0 * K1 * ldim;
  const bool even = (g.K2 % 2) == 0;
  double acc[7];
#pragma unroll
  for (int c = 0; c < 7; c++) acc[c] = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nm; i += (long)gridDim.x * blockDim.x) {
    const int kz = (int)(i % ldim);
    const int ky = (int)((i / ldim) % K1);
    const int kx = (int)(i / ((long)ldim * K1));
    const float2 q = S[i];
    const double s = (double)q.x * q.x + (double)q.y * q.y;
    const bool plane = (kz == 0) || (even && kz == ldim - 1);
    double A, dA[6];
    if (MODE == 1) {
      A = inf.A[i];
#pragma unroll
      for (int c = 0; c < 6; c++) dA[c] = inf.dA[6 * i + c];
    } else {
      double sf, sd[6];
      ewald_images(inf, g.K0, K1, g.K2, kx, ky, kz, sf, sd);
      // set_A adds f/2 from each image and from each conjugate image
      // (interior modes), and f' m m in full from both.
      const double wA = plane ? 0.5 : 1.0;
      A = wA * sf;
#pragma unroll
      for (int c = 0; c < 6; c++) dA[c] = 2.0 * wA * sd[c];
    }
    acc[0] += s * A;
#pragma unroll
    for (int c = 0; c < 6; c++) acc[1 + c] += s * dA[c];
    if (SCALE) {
      double t = A * iB0[kx] * iB1[ky] * iB2[kz];
      if (plane) t *= 2.0;
      S[i] = make_float2(q.x * (float)t, q.y * (float)t);
    }
  }
  __shared__ double red[8][7];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 7; c++) {
    const double v = warp_sum(acc[c]);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w][threadIdx.x];
    partials[(long)blockIdx.x * kRedWords + threadIdx.x] = v;
  }
}

__global__ void conv_finish_kernel(const double *__restrict__ partials, int nblocks, double *__restrict__ out) {
  const int c = threadIdx.x;
  if (c >= 7) return;
  double v = 0.0;
  for (int b = 0; b < nblocks; b++) v += partials[(long)b * kRedWords + c];
  out[c] = v;
}

int launch_conv(const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                 const double *iB2, float2 *S, int want_scale, double *partials, double *out,
                 cudaStream_t st) {
  const long nm = (long)g.K0 * g.K1 * g.ldim;
  int blocks = (int)((nm + 255) / 256);
  if (blocks > kConvBlocks) blocks = kConvBlocks;
  if (inf.mode == 1) {
    if (want_scale) conv_kernel<1, true><<<blocks, 256, 0, st>>>(g, inf, iB0, iB1, iB2, S, partials);
    else conv_kernel<1, false><<<blocks, 256, 0, st>>>(g, inf, iB0, iB1, iB2, S, partials);
  } else {
    if (want_scale) conv_kernel<2, true><<<blocks, 256, 0, st>>>(g, inf, iB0, iB1, iB2, S, partials);
    else conv_kernel<2, false><<<blocks, 256, 0, st>>>(g, inf, iB0, iB1, iB2, S, partials);
  }
  conv_finish_kernel<<<1, 32, 0, st>>>(partials, blocks, out);
  return 2;
}

}  // namespace spme
