// K4 + K7: B-spline moduli, influence function and the fused reciprocal
// convolution (en, sfac.cpp:304-325; de1, sfac.cpp:339-396; set_A,
// sfac.cpp:213-292; bspl_dft, sfac.cpp:21-35).
//
// The moduli, the influence function and the energy/virial reductions are
// FP64; the structure factor itself is FP32.  Reductions are deterministic:
// a fixed grid of kConvBlocks blocks walks the modes with a fixed stride,
// each block reduces with a fixed shuffle tree, and one final block sums the
// block partials in index order.  No atomics.
#include "influence.cuh"

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

template <bool SCALE>
__global__ void __launch_bounds__(256) conv_kernel(Geom g, Influence inf, const double *__restrict__ iB0,
                                                   const double *__restrict__ iB1,
                                                   const double *__restrict__ iB2, float2 *__restrict__ S,
                                                   double *__restrict__ partials) {
  const int ldim = g.ldim, K1 = g.K1;
  const long nm = (long)g.K0 * K1 * ldim;
  const bool even = (g.K2 % 2) == 0;
  const InfConst ic = load_ic(inf);
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
    mode_influence(inf, ic, g, i, kx, ky, kz, plane, A, dA);
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
  block_reduce7(acc, red, partials + (long)blockIdx.x * kRedWords);
}

__global__ void conv_finish_kernel(const double *__restrict__ partials, int nblocks,
                                   const CellConst *__restrict__ cell, double *__restrict__ raw,
                                   double *__restrict__ ev) {
  finish_partials(partials, nblocks, cell, raw, ev);
}

int launch_conv(const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                const double *iB2, float2 *S, int want_scale, double *partials, double *out, double *ev,
                cudaStream_t st) {
  const long nm = (long)g.K0 * g.K1 * g.ldim;
  int blocks = (int)((nm + 255) / 256);
  if (blocks > kConvBlocks) blocks = kConvBlocks;
  if (want_scale) conv_kernel<true><<<blocks, 256, 0, st>>>(g, inf, iB0, iB1, iB2, S, partials);
  else conv_kernel<false><<<blocks, 256, 0, st>>>(g, inf, iB0, iB1, iB2, S, partials);
  conv_finish_kernel<<<1, 8 * 32, 0, st>>>(partials, blocks, g.cell, out, ev);
  return 2;
}

__global__ void ewald_rows_kernel(Geom g, Influence inf, RowImg *rows) {
  const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= (long)g.K0 * g.K1) return;
  const InfConst ic = *inf.ic;
  RowImg row;
  row.count = ewald_row(ic, g.K0, g.K1, (int)(r / g.K1), (int)(r % g.K1), row);
  row.pad = 0;
  rows[r] = row;
}

int launch_ewald_rows(const Geom &g, const Influence &inf, RowImg *rows, cudaStream_t st) {
  const long n = (long)g.K0 * g.K1;
  ewald_rows_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g, inf, rows);
  return 1;
}

// Tabulates the device Ewald influence function (inf.mode 2) per stored
// mode in the layout of set_A's tables: A[i] and dA[6 i + c] (FP64), so the
// solves read them instead of evaluating the images of every mode again.
__global__ void __launch_bounds__(256) ewald_table_kernel(Geom g, Influence inf, double *__restrict__ A,
                                                          double *__restrict__ dA) {
  const long nmodes = (long)g.K0 * g.K1 * g.ldim;
  const InfConst ic = *inf.ic;
  const bool even = (g.K2 % 2) == 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nmodes; i += (long)gridDim.x * blockDim.x) {
    const int kz = (int)(i % g.ldim);
    const long r = i / g.ldim;
    const int ky = (int)(r % g.K1), kx = (int)(r / g.K1);
    const bool plane = (kz == 0) || (even && kz == g.ldim - 1);
    double a, d[6];
    mode_influence(inf, ic, g, i, kx, ky, kz, plane, a, d);
    A[i] = a;
#pragma unroll
    for (int c = 0; c < 6; c++) dA[6 * i + c] = d[c];
  }
}

int launch_ewald_table(const Geom &g, const Influence &inf, double *A, double *dA, cudaStream_t st) {
  ewald_table_kernel<<<4 * 148, 256, 0, st>>>(g, inf, A, dA);
  return 1;
}

// Compact table of the device Ewald function (mode 4), one double per mode:
// 0 when no image lies in the sphere; -1 when several do; otherwise A with
// its 6 lowest mantissa bits replaced by the single image's lattice shift
// (si+2) | (sj+2) << 2 | (sk+2) << 4 (a relative change below 2^-46).
__global__ void __launch_bounds__(256) ewald_compact_kernel(Geom g, Influence inf, double *__restrict__ A) {
  const long nmodes = (long)g.K0 * g.K1 * g.ldim;
  const InfConst ic = *inf.ic;
  const bool even = (g.K2 % 2) == 0;
  const int K0 = g.K0, K1 = g.K1, K2 = g.K2;
  for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < nmodes; m += (long)gridDim.x * blockDim.x) {
    const int kz = (int)(m % g.ldim);
    const long r = m / g.ldim;
    const int ky = (int)(r % K1), kx = (int)(r / K1);
    const bool plane = (kz == 0) || (even && kz == g.ldim - 1);
    // set_A's image set (radial_images' loops), counting the images
    const double R2 = __dmul_rn(ic.max_m, ic.max_m);
    const int i0 = __double2int_rz(__ddiv_rn(ic.max_m, ic.iL00));
    double sf = 0.0;
    int count = 0, li = 0, lj = 0, lk = 0;
    for (int i = -i0 + imod(kx + i0, K0); i <= i0; i += K0) {
      const double mx = __dmul_rn((double)i, ic.iL00);
      const double m20 = __dmul_rn(mx, mx);
      const double dy = sqrt(fmax(__dsub_rn(R2, m20), 0.0));
      const double my0 = __dmul_rn((double)i, ic.iL10);
      const int j0 = (int)ceil(__ddiv_rn(__dsub_rn(-dy, my0), ic.iL11));
      const int j1 = (int)floor(__ddiv_rn(__dsub_rn(dy, my0), ic.iL11));
      for (int j = j0 + imod(ky - j0, K1); j <= j1; j += K1) {
        const double my = __dadd_rn(my0, __dmul_rn((double)j, ic.iL11));
        const double m21 = __dadd_rn(m20, __dmul_rn(my, my));
        const double dz = sqrt(fmax(__dsub_rn(R2, m21), 0.0));
        const double mz0 = __dadd_rn(__dmul_rn((double)i, ic.iL20), __dmul_rn((double)j, ic.iL21));
        const int k0 = (int)ceil(__ddiv_rn(__dsub_rn(-dz, mz0), ic.iL22));
        const int k1 = (int)floor(__ddiv_rn(__dsub_rn(dz, mz0), ic.iL22));
        for (int k = k0 + imod(kz - k0, K2); k <= k1; k += K2) {
          const double mz = __dadd_rn(mz0, __dmul_rn((double)k, ic.iL22));
          const double m2 = __dadd_rn(m21, __dmul_rn(mz, mz));
          double fp;
          sf += ewald_f(m2, ic.fac, fp);
          count++;
          li = i;
          lj = j;
          lk = k;
        }
      }
    }
    const double a = (plane ? 0.5 : 1.0) * sf;
    double packed = -1.0;  // several images (or a shift out of range): row enumeration
    if (count == 0) {
      packed = 0.0;
    } else if (count == 1) {
      const int si = (li - kx) / K0, sj = (lj - ky) / K1, sk = (lk - kz) / K2;
      if (si >= -2 && si <= 1 && sj >= -2 && sj <= 1 && sk >= -2 && sk <= 1) {
        const unsigned long long c = (unsigned long long)((si + 2) | ((sj + 2) << 2) | ((sk + 2) << 4));
        packed = __longlong_as_double((long long)((__double_as_longlong(a) & ~0x3FULL) | c));
      }
    }
    A[m] = packed;
  }
}

int launch_ewald_compact(const Geom &g, const Influence &inf, double *A, cudaStream_t st) {
  ewald_compact_kernel<<<4 * 148, 256, 0, st>>>(g, inf, A);
  return 1;
}

// Tabulates a caller-sampled radial function (TableRadial) per stored mode,
// over the same image set as set_A (radial_images), into set_A's table
// layout: A = (1/2 on the kz = 0 / Nyquist planes) sum f, dA = 2 x that
// weight x sum f' m m.
__global__ void __launch_bounds__(256) radial_table_kernel(Geom g, InfConst ic, TableRadial fn, double *__restrict__ A,
                                                           double *__restrict__ dA) {
  const long nmodes = (long)g.K0 * g.K1 * g.ldim;
  const bool even = (g.K2 % 2) == 0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nmodes; i += (long)gridDim.x * blockDim.x) {
    const int kz = (int)(i % g.ldim);
    const long r = i / g.ldim;
    const int ky = (int)(r % g.K1), kx = (int)(r / g.K1);
    const bool plane = (kz == 0) || (even && kz == g.ldim - 1);
    double sf, sd[6];
    radial_images(ic, fn, g.K0, g.K1, g.K2, kx, ky, kz, sf, sd);
    const double wA = plane ? 0.5 : 1.0;
    A[i] = wA * sf;
#pragma unroll
    for (int c = 0; c < 6; c++) dA[6 * i + c] = 2.0 * wA * sd[c];
  }
}

int launch_radial_table(const Geom &g, const InfConst &ic, const double *f, const double *df, int nt, double dm2,
                        double *A, double *dA, cudaStream_t st) {
  TableRadial fn{f, df, nt, dm2, 1.0 / dm2};
  radial_table_kernel<<<4 * 148, 256, 0, st>>>(g, ic, fn, A, dA);
  return 1;
}

int launch_finish(const double *partials, int nblocks, const CellConst *cell, double *raw, double *ev,
                  cudaStream_t st) {
  conv_finish_kernel<<<1, 8 * 32, 0, st>>>(partials, nblocks, cell, raw, ev);
  return 1;
}

}  // namespace spme
