// Influence function of the reciprocal convolution, per stored mode
// (set_A, sfac.cpp:213-292; ewald.py:124-132), FP64, and FP64 reductions.
#pragma once

#include "reduce.cuh"
#include "spme_kernels.hpp"

namespace spme {

// Ewald influence function f(m^2) = exp(-pi^2 m^2 / beta^2) / (pi m^2) and
// f'(m^2) = (-pi^2/beta^2 - 1/m^2) f  (ewald.py:124-132; f(0) = 0), with
// fac = -pi^2/beta^2.  One correctly rounded reciprocal of m^2 serves both.
__device__ __forceinline__ double ewald_f(double r2, double fac, double &fp) {
  if (r2 < 1e-10) {
    fp = 0.0;
    return 0.0;
  }
  constexpr double kInvPi = 0.318309886183790671537767526745028724;
  const double ir2 = __drcp_rn(r2);
  const double f = exp(r2 * fac) * (ir2 * kInvPi);
  fp = (fac - ir2) * f;
  return f;
}

// Sum of f and f' m_a m_b over the reciprocal vectors m = iL (i,j,k) with
// |m| < max_m whose lattice index is congruent to the stored mode
// (kx, ky, kz) -- the images set_A visits and folds onto this mode
// (sfac.cpp:240-289, same sphere bounds, FP64 without contraction).  The
// conjugate images that set_A folds onto interior modes have the same f
// values, so the caller doubles those instead of revisiting them.
// F: f(m^2) returning f and storing f'(m^2) in fp.
template <class F>
__device__ __forceinline__ void radial_images(const InfConst &inf, const F &fn, int K0, int K1, int K2, int kx, int ky,
                                              int kz, double &sf, double sd[6]) {
  const double R2 = __dmul_rn(inf.max_m, inf.max_m);
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
        sf += fn(m2, fp);
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

struct EwaldRadial {
  double fac;
  __device__ __forceinline__ double operator()(double m2, double &fp) const { return ewald_f(m2, fac, fp); }
};

// A radial function sampled by the caller: f and f' at m^2 = k dm2,
// k = 0..nt-1, evaluated by cubic Hermite interpolation in m^2 (f to fourth
// order in dm2, f' as the interpolant's derivative to third order); 0 beyond
// the last sample.
struct TableRadial {
  const double *f, *df;
  int nt;
  double dm2, inv_dm2;
  __device__ __forceinline__ double operator()(double m2, double &fp) const {
    const double t = m2 * inv_dm2;
    if (!(t <= (double)(nt - 1))) {
      fp = 0.0;
      return 0.0;
    }
    int k = (int)t;
    if (k > nt - 2) k = nt - 2;
    const double u = t - (double)k, u2 = u * u, u3 = u2 * u;
    const double p0 = f[k], p1 = f[k + 1], m0 = df[k] * dm2, m1 = df[k + 1] * dm2;
    const double v = (2.0 * u3 - 3.0 * u2 + 1.0) * p0 + (u3 - 2.0 * u2 + u) * m0 + (3.0 * u2 - 2.0 * u3) * p1 +
                     (u3 - u2) * m1;
    fp = ((6.0 * u2 - 6.0 * u) * p0 + (3.0 * u2 - 4.0 * u + 1.0) * m0 + (6.0 * u - 6.0 * u2) * p1 +
          (3.0 * u2 - 2.0 * u) * m1) * inv_dm2;
    return v;
  }
};

__device__ __forceinline__ void ewald_images(const InfConst &inf, int K0, int K1, int K2, int kx, int ky, int kz,
                                             double &sf, double sd[6]) {
  radial_images(inf, EwaldRadial{inf.fac}, K0, K1, K2, kx, ky, kz, sf, sd);
}


// Image pairs (i, j) of row (kx, ky) and their z bounds, exactly as
// ewald_images enumerates them.  Returns the pair count, or -1 when the row
// has more than kRowPairs pairs.
__device__ __forceinline__ int ewald_row(const InfConst &inf, int K0, int K1, int kx, int ky, RowImg &r) {
  const double R2 = __dmul_rn(inf.max_m, inf.max_m);
  const int i0 = __double2int_rz(__ddiv_rn(inf.max_m, inf.iL00));
  int c = 0;
  for (int i = -i0 + imod(kx + i0, K0); i <= i0; i += K0) {
    const double mx = __dmul_rn((double)i, inf.iL00);
    const double m20 = __dmul_rn(mx, mx);
    const double dy = sqrt(fmax(__dsub_rn(R2, m20), 0.0));
    const double my0 = __dmul_rn((double)i, inf.iL10);
    const int j0 = (int)ceil(__ddiv_rn(__dsub_rn(-dy, my0), inf.iL11));
    const int j1 = (int)floor(__ddiv_rn(__dsub_rn(dy, my0), inf.iL11));
    for (int j = j0 + imod(ky - j0, K1); j <= j1; j += K1) {
      if (c >= kRowPairs) return -1;
      const double my = __dadd_rn(my0, __dmul_rn((double)j, inf.iL11));
      const double m21 = __dadd_rn(m20, __dmul_rn(my, my));
      const double dz = sqrt(fmax(__dsub_rn(R2, m21), 0.0));
      const double mz0 = __dadd_rn(__dmul_rn((double)i, inf.iL20), __dmul_rn((double)j, inf.iL21));
      r.k0[c] = (int)ceil(__ddiv_rn(__dsub_rn(-dz, mz0), inf.iL22));
      r.k1[c] = (int)floor(__ddiv_rn(__dsub_rn(dz, mz0), inf.iL22));
      r.mx[c] = mx;
      r.my[c] = my;
      r.m21[c] = m21;
      r.mz0[c] = mz0;
      c++;
    }
  }
  return c;
}

// Same sums as ewald_images from a row's precomputed pairs: per pair only
// the z images (k = kz mod K2 within [k0, k1]) and their exp are evaluated.
__device__ __forceinline__ void ewald_images_row(const InfConst &inf, const FastDiv &K2d, const RowImg &r, int K2,
                                                 int kz, double &sf, double sd[6]) {
  const double fac = inf.fac;
  sf = 0.0;
  for (int c = 0; c < 6; c++) sd[c] = 0.0;
  const int n = r.count;
  for (int c = 0; c < n; c++) {
    const int k0 = r.k0[c], k1 = r.k1[c];
    const double mx = r.mx[c], my = r.my[c], m21 = r.m21[c], mz0 = r.mz0[c];
    // first k >= k0 with k = kz (mod K2)
    const int d = kz - k0;
    int k = k0 + (d >= 0 ? d - (int)K2d.div((uint32_t)d) * K2
                         : (K2 - 1) - (int)((uint32_t)(-d - 1) - K2d.div((uint32_t)(-d - 1)) * K2));
    for (; k <= k1; k += K2) {
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

// A (with set_A's half weight on the kz = 0 and even-K2 Nyquist planes) and
// dA (6 components) of stored mode (kx, ky, kz), index i = (kx*K1 + ky)*ldim + kz.
// The device Ewald constants, or zeros when the influence comes from tables.
__device__ __forceinline__ InfConst load_ic(const Influence &inf) {
  InfConst c{};
  if (inf.mode >= 2) c = *inf.ic;
  return c;
}

// ic: the device Ewald constants (load_ic(inf)), loaded once by the caller.
__device__ __forceinline__ void mode_influence(const Influence &inf, const InfConst &ic, const Geom &g, long i, int kx,
                                               int ky, int kz, bool plane, double &A, double dA[6]) {
  if (inf.mode == 1) {
    A = inf.A[i];
#pragma unroll
    for (int c = 0; c < 6; c++) dA[c] = inf.dA[6 * i + c];
  } else {
    double sf, sd[6];
    const RowImg &r = inf.rows[(long)kx * g.K1 + ky];
    if (r.count >= 0) ewald_images_row(ic, inf.K2d, r, g.K2, kz, sf, sd);
    else ewald_images(ic, g.K0, g.K1, g.K2, kx, ky, kz, sf, sd);
    // set_A adds f/2 from each image and from each conjugate image
    // (interior modes), and f' m m in full from both.
    const double wA = plane ? 0.5 : 1.0;
    A = wA * sf;
#pragma unroll
    for (int c = 0; c < 6; c++) dA[c] = 2.0 * wA * sd[c];
  }
}

// Same A as mode_influence; instead of returning dA it adds sq * A to acc[0]
// and sq * dA[c] to acc[1 + c] image by image (fewer live registers).
__device__ __forceinline__ double mode_influence_acc(const Influence &inf, const InfConst &ic, const Geom &g, long i,
                                                     int kx, int ky, int kz, bool plane, double sq, double (&acc)[7]) {
  const double wA = plane ? 0.5 : 1.0;
  if (inf.mode == 1) {
    const double A = inf.A[i];
    acc[0] += sq * A;
#pragma unroll
    for (int c = 0; c < 6; c++) acc[1 + c] += sq * inf.dA[6 * i + c];
    return A;
  }
  const RowImg &r = inf.rows[(long)kx * g.K1 + ky];
  if (r.count < 0) {
    double sf, sd[6];
    ewald_images(ic, g.K0, g.K1, g.K2, kx, ky, kz, sf, sd);
    const double A = wA * sf;
    acc[0] += sq * A;
#pragma unroll
    for (int c = 0; c < 6; c++) acc[1 + c] += sq * (2.0 * wA * sd[c]);
    return A;
  }
  const double fac = ic.fac;
  const double w2 = 2.0 * wA * sq;
  double sf = 0.0;
  const int n = r.count;
  for (int c = 0; c < n; c++) {
    const int k0 = r.k0[c], k1 = r.k1[c];
    const int d = kz - k0;
    int k = k0 + (d >= 0 ? d - (int)inf.K2d.div((uint32_t)d) * g.K2
                         : (g.K2 - 1) - (int)((uint32_t)(-d - 1) - inf.K2d.div((uint32_t)(-d - 1)) * g.K2));
    if (k > k1) continue;
    const double mx = r.mx[c], my = r.my[c], m21 = r.m21[c], mz0 = r.mz0[c];
    for (; k <= k1; k += g.K2) {
      const double mz = __dadd_rn(mz0, __dmul_rn((double)k, ic.iL22));
      const double m2 = __dadd_rn(m21, __dmul_rn(mz, mz));
      double fp;
      sf += ewald_f(m2, fac, fp);
      const double t = w2 * fp;
      acc[1] += t * mx * mx;
      acc[2] += t * my * my;
      acc[3] += t * mz * mz;
      acc[4] += t * my * mx;
      acc[5] += t * mz * mx;
      acc[6] += t * mz * my;
    }
  }
  const double A = wA * sf;
  acc[0] += sq * A;
  return A;
}

// Mode 4, one stored mode: the packed compact-table entry; for a single image
// the lattice vector (kx + si K0, ky + sj K1, kz + sk K2) gives m and
// dA = 2 wA f'(m^2) m m = 2 (fac - 1/m^2) A m m (A = wA f); several images
// (a negative entry) take mode 2's row enumeration.  Adds sq A and sq dA to
// acc.
__device__ __forceinline__ double ewald_row_acc_multi(const Influence &inf, const InfConst &ic, const Geom &g, long i,
                                                   int kx, int ky, int kz, bool plane, double sq, double *acc) {
  double a7[7] = {0, 0, 0, 0, 0, 0, 0};
  Influence m2 = inf;
  m2.mode = 2;
  const double A = mode_influence_acc(m2, ic, g, i, kx, ky, kz, plane, sq, a7);
#pragma unroll
  for (int c = 0; c < 7; c++) acc[c] += a7[c];
  return A;
}

__device__ __forceinline__ double compact_acc(const Influence &inf, const InfConst &ic, const Geom &g, long i, int kx,
                                              int ky, int kz, bool plane, double sq, double packed,
                                              double (&acc)[7]) {
  if (packed < 0.0) return ewald_row_acc_multi(inf, ic, g, i, kx, ky, kz, plane, sq, acc);
  const unsigned long long bits = (unsigned long long)__double_as_longlong(packed);
  const double A = __longlong_as_double((long long)(bits & ~0x3FULL));
  if (A == 0.0) return 0.0;
  const int code = (int)(bits & 0x3F);
  const double ii = (double)(kx + ((code & 3) - 2) * g.K0);
  const double jj = (double)(ky + (((code >> 2) & 3) - 2) * g.K1);
  const double kk = (double)(kz + (((code >> 4) & 3) - 2) * g.K2);
  const double mx = ii * ic.iL00;
  const double my = ii * ic.iL10 + jj * ic.iL11;
  const double mz = ii * ic.iL20 + jj * ic.iL21 + kk * ic.iL22;
  const double m2 = mx * mx + my * my + mz * mz;
  const double t = 2.0 * (ic.fac - __drcp_rn(m2)) * A * sq;
  acc[0] += sq * A;
  acc[1] += t * mx * mx;
  acc[2] += t * my * my;
  acc[3] += t * mz * mz;
  acc[4] += t * my * mx;
  acc[5] += t * mz * mx;
  acc[6] += t * mz * my;
  return A;
}

// The influence source fixed at compile time (one kernel per source keeps
// each variant's registers to its own path): IM = 1 tables, 2 row tables
// (mode 2), 4 compact table (mode 4).
template <int IM>
__device__ __forceinline__ double influence_acc(const Influence &inf, const InfConst &ic, const Geom &g, long i, int kx,
                                                int ky, int kz, bool plane, double sq, double (&acc)[7]) {
  if constexpr (IM == 4) {
    return compact_acc(inf, ic, g, i, kx, ky, kz, plane, sq, inf.A[i], acc);
  } else {
    Influence f = inf;
    f.mode = IM;
    return mode_influence_acc(f, ic, g, i, kx, ky, kz, plane, sq, acc);
  }
}

__device__ __forceinline__ void block_reduce7(const double (&acc)[7], double (*red)[7], double *out_global) {
  block_reduce_n<7>(acc, red, out_global);
}

// Sum of the block partials (warp c sums component c: lanes take blocks in
// a fixed stride, then a fixed shuffle tree), and the final energy/virial
// ev = [E, vir_xx, vir_yy, vir_zz, vir_yx, vir_zx, vir_zy] as de1 forms them
// (sfac.cpp:384-395).  Needs >= 7 warps; raw receives the 7 sums.
__device__ __forceinline__ void finish_partials(const double *__restrict__ partials, int nblocks,
                                                const CellConst *__restrict__ cell, double *__restrict__ raw,
                                                double *__restrict__ ev) {
  __shared__ double tot[7];
  sum_partials<7>(partials, nblocks, kRedWords, tot);
  const double iV = cell->iV;
  if (raw && threadIdx.x < 7) raw[threadIdx.x] = tot[threadIdx.x];
  if (ev && threadIdx.x == 0) {
    const double fac = iV * iV;
    ev[0] = tot[0] * iV;
    ev[1] = (tot[1] + tot[0]) * fac;
    ev[2] = (tot[2] + tot[0]) * fac;
    ev[3] = (tot[3] + tot[0]) * fac;
    ev[4] = tot[4] * fac;
    ev[5] = tot[5] * fac;
    ev[6] = tot[6] * fac;
  }
}

}  // namespace spme
