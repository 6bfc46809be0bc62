// K3/K5: hand-written batched mixed-radix FFT passes (FP32) for the 3D
// r2c / c2r transforms of the SPME grid (sfac.cpp:78-81,125,392).
//
// Convention (FFTW's, which the reference uses): unnormalised, forward sign
// -1, inverse +1; the r2c output keeps ldim = K2/2+1 values of the last
// axis.  A 3D transform is three passes: z (real rows, two rows packed into
// one complex line), y and x (strided complex lines); the inverse runs in
// reverse.  Each CTA loads B lines into shared memory ([j][b] layout, pitch
// B+1 to spread banks), runs Stockham autosort stages with radix 4, 2, 3, 5,
// 7 butterflies written out and a direct-DFT butterfly for any other prime,
// and stores the lines back.  Twiddles come from an FP32 table built in FP64
// (fft_twiddle_kernel).
#include <type_traits>

#include "fft_engine.cuh"
#include "fft_reg.cuh"
#include "influence.cuh"

namespace spme {

SPME_CHECK_READER(fft)

// --- z pass, forward: real rows -> half-complex rows --------------------
// CTA handles 2B real rows (B complex lines); row pitch K2 (real) / ldim.
__global__ void __launch_bounds__(256) fft_z_r2c_kernel(FftLen L, int nrows, const float *__restrict__ rin,
                                                        float2 *__restrict__ cout, int ldim, int B,
                                                        int bufsz, FastDiv Bd) {
  extern __shared__ float2 sm[];
  const int n = L.n, P = B + 1;
  float2 *tw = sm, *b0 = sm + n, *b1 = b0 + bufsz;
  load_twiddles(tw, L);
  const long row0 = (long)blockIdx.x * 2 * B;
  for (int e = threadIdx.x; e < 2 * B * n; e += blockDim.x) {
    const int rl = e / n, z = e % n;
    const long row = row0 + rl;
    const float v = (row < nrows) ? rin[row * n + z] : 0.f;
    float *slot = reinterpret_cast<float *>(&b0[z * P + (rl >> 1)]);
    slot[rl & 1] = v;
  }
  __syncthreads();
  float2 *res = run_stages<-1>(L, b0, b1, tw, Bd, P);
  for (int e = threadIdx.x; e < 2 * B * ldim; e += blockDim.x) {
    const int rl = e / ldim, k = e % ldim;
    const long row = row0 + rl;
    if (row >= nrows) continue;
    const int b = rl >> 1;
    const float2 u = res[k * P + b], v = res[((n - k) % n) * P + b];
    float2 X;
    if ((rl & 1) == 0) X = make_float2(0.5f * (u.x + v.x), 0.5f * (u.y - v.y));
    else X = make_float2(0.5f * (u.y + v.y), -0.5f * (u.x - v.x));
    cout[row * ldim + k] = X;
  }
}

// --- z pass, inverse: half-complex rows -> real rows --------------------
// Self-conjugate bins (k = 0 and the even-n Nyquist bin) contribute their
// real part only, as a c2r transform does.
__global__ void __launch_bounds__(256) fft_z_c2r_kernel(FftLen L, int nrows, const float2 *__restrict__ cin,
                                                        float *__restrict__ rout, int ldim, int B,
                                                        int bufsz, FastDiv Bd) {
  extern __shared__ float2 sm[];
  const int n = L.n, P = B + 1;
  float2 *tw = sm, *b0 = sm + n, *b1 = b0 + bufsz;
  load_twiddles(tw, L);
  const long row0 = (long)blockIdx.x * 2 * B;
  // stage the 2B half rows in b1 as [row_local][k]
  for (int e = threadIdx.x; e < 2 * B * ldim; e += blockDim.x) {
    const int rl = e / ldim, k = e % ldim;
    const long row = row0 + rl;
    float2 X = (row < nrows) ? cin[row * ldim + k] : make_float2(0.f, 0.f);
    if (k == 0 || 2 * k == n) X.y = 0.f;
    b1[rl * ldim + k] = X;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < B * n; e += blockDim.x) {
    const int b = e % B, k = e / B;
    float2 z;
    if (k < ldim) {
      const float2 A = b1[(2 * b) * ldim + k], Bv = b1[(2 * b + 1) * ldim + k];
      z = make_float2(A.x - Bv.y, A.y + Bv.x);
    } else {
      const float2 A = b1[(2 * b) * ldim + (n - k)], Bv = b1[(2 * b + 1) * ldim + (n - k)];
      z = make_float2(A.x + Bv.y, Bv.x - A.y);
    }
    b0[k * P + b] = z;
  }
  __syncthreads();
  float2 *res = run_stages<+1>(L, b0, b1, tw, Bd, P);
  for (int e = threadIdx.x; e < 2 * B * n; e += blockDim.x) {
    const int rl = e / n, z = e % n;
    const long row = row0 + rl;
    if (row >= nrows) continue;
    const float2 v = res[z * P + (rl >> 1)];
    rout[row * n + z] = (rl & 1) ? v.y : v.x;
  }
}

// --- strided complex pass (y or x axis) ---------------------------------
// Line b (0 <= b < nlines) starts at (b / inner) * outer + (b % inner);
// element j at +j*stride.  With scale != 0 the forward x pass also divides
// by the B-spline moduli: S *= iB0[kx] iB1[ky] iB2[kz] (sfac.cpp:128-138),
// the factor formed in FP64.
template <int SIGN>
__global__ void __launch_bounds__(256) fft_strided_kernel(FftLen L, long nlines, long inner, long outer,
                                                          long stride, float2 *__restrict__ data, int B,
                                                          int bufsz, DeconvArgs dc, FastDiv Bd) {
  extern __shared__ float2 sm[];
  const int n = L.n, P = B + 1;
  float2 *tw = sm, *b0 = sm + n, *b1 = b0 + bufsz;
  load_twiddles(tw, L);
  const long line0 = (long)blockIdx.x * B;
  for (int e = threadIdx.x; e < B * n; e += blockDim.x) {
    const int b = e % B, j = e / B;
    const long line = line0 + b;
    float2 v = make_float2(0.f, 0.f);
    if (line < nlines) v = data[(line / inner) * outer + (line % inner) + j * stride];
    b0[j * P + b] = v;
  }
  __syncthreads();
  float2 *res = run_stages<SIGN>(L, b0, b1, tw, Bd, P);
  for (int e = threadIdx.x; e < B * n; e += blockDim.x) {
    const int b = e % B, j = e / B;
    const long line = line0 + b;
    if (line >= nlines) continue;
    float2 v = res[j * P + b];
    if (dc.iB0) {
      // x pass: line = ky*ldim + kz, j = kx
      const int ky = (int)(line / dc.ldim), kz = (int)(line % dc.ldim);
      const float t = (float)(dc.iB0[j] * dc.iB1[ky] * dc.iB2[kz]);
      v = cscale(v, t);
    }
    data[(line / inner) * outer + (line % inner) + j * stride] = v;
  }
}


// --- fused plane pass, forward: one CTA per x-plane -----------------------
// z r2c of the plane's K1 real rows (two rows per complex line), then the
// y transform of its ldim columns, both in shared memory; one read of the
// real plane, one write of the half-complex plane.  Loads, the r2c unpack
// and stores are CTA-wide (coalesced); each transform step is
// warp-synchronous over a warp's own columns (dz / dy: columns per warp).
__global__ void __launch_bounds__(512) fft_plane_fwd_kernel(FftLen Ly, FftLen Lz, const float *__restrict__ rin,
                                                            float2 *__restrict__ cout, int sz, FastDiv dz, FastDiv dy,
                                                            FastDiv dK2, FastDiv dldim) {
  extern __shared__ float2 sm[];
  const int K1 = Ly.n, K2 = Lz.n, ldim = K2 / 2 + 1;
  float2 *twy = sm, *twz = twy + K1, *A = twz + K2, *Bf = A + sz;
  load_twiddles(twy, Ly);
  load_twiddles(twz, Lz);
  const long x = blockIdx.x;
  const float *plane = rin + x * K1 * K2;
  float2 *out = cout + x * K1 * ldim;
  const int nb1 = (K1 + 1) / 2, P1 = nb1 + 1, P2 = ldim + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e = threadIdx.x; e < K1 * K2; e += blockDim.x) {
    uint32_t y, z;
    dK2.divmod((uint32_t)e, y, z);
    reinterpret_cast<float *>(&A[z * P1 + (y >> 1)])[y & 1] = plane[e];
  }
  if (K1 & 1)
    for (int z = threadIdx.x; z < K2; z += blockDim.x) A[z * P1 + nb1 - 1].y = 0.f;
  __syncthreads();
  {
    const int c0 = warp * (int)dz.d, nc = min((int)dz.d, nb1 - c0);
    if (nc > 0) run_stages_w<-1>(Lz, A, Bf, twz, dz, P1, c0, nc, lane);
  }
  float2 *R1 = (Lz.nst & 1) ? Bf : A;
  float2 *O = (R1 == A) ? Bf : A;
  __syncthreads();
  for (int e = threadIdx.x; e < K1 * ldim; e += blockDim.x) {
    uint32_t y, k;
    dldim.divmod((uint32_t)e, y, k);
    const int b = (int)y >> 1;
    const float2 u = R1[k * P1 + b], v = R1[((K2 - (int)k) % K2) * P1 + b];
    O[y * P2 + k] = (y & 1) ? make_float2(0.5f * (u.y + v.y), -0.5f * (u.x - v.x))
                            : make_float2(0.5f * (u.x + v.x), 0.5f * (u.y - v.y));
  }
  __syncthreads();
  {
    const int c0 = warp * (int)dy.d, nc = min((int)dy.d, ldim - c0);
    if (nc > 0) run_stages_w<-1>(Ly, O, R1, twy, dy, P2, c0, nc, lane);
  }
  float2 *R2 = (Ly.nst & 1) ? R1 : O;
  __syncthreads();
  for (int e = threadIdx.x; e < K1 * ldim; e += blockDim.x) {
    uint32_t y, k;
    dldim.divmod((uint32_t)e, y, k);
    out[e] = R2[y * P2 + k];
  }
}

// --- fused plane pass, inverse: y transform then z c2r per x-plane -------
// CTA 0 first reduces the energy/virial partials of the preceding x pass
// (when `partials` is given): the reduction needs no extra launch.
__global__ void __launch_bounds__(512) fft_plane_inv_kernel(FftLen Ly, FftLen Lz, const float2 *__restrict__ cin,
                                                            float *__restrict__ rout, int sz,
                                                            const double *__restrict__ partials, int nblocks,
                                                            const CellConst *__restrict__ cell,
                                                            double *__restrict__ raw, double *__restrict__ ev,
                                                            FastDiv dz, FastDiv dy, FastDiv dK2, FastDiv dldim,
                                                            FastDiv dnb1) {
  if (partials && blockIdx.x == 0) finish_partials(partials, nblocks, cell, raw, ev);
  extern __shared__ float2 sm[];
  const int K1 = Ly.n, K2 = Lz.n, ldim = K2 / 2 + 1;
  float2 *twy = sm, *twz = twy + K1, *A = twz + K2, *Bf = A + sz;
  load_twiddles(twy, Ly);
  load_twiddles(twz, Lz);
  const long x = blockIdx.x;
  const float2 *in = cin + x * K1 * ldim;
  float *plane = rout + x * K1 * K2;
  const int nb1 = (K1 + 1) / 2, P1 = nb1 + 1, P2 = ldim + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e = threadIdx.x; e < K1 * ldim; e += blockDim.x) {
    uint32_t y, k;
    dldim.divmod((uint32_t)e, y, k);
    A[y * P2 + k] = in[e];
  }
  __syncthreads();
  {
    const int c0 = warp * (int)dy.d, nc = min((int)dy.d, ldim - c0);
    if (nc > 0) run_stages_w<+1>(Ly, A, Bf, twy, dy, P2, c0, nc, lane);
  }
  float2 *R = (Ly.nst & 1) ? Bf : A;
  float2 *O = (R == A) ? Bf : A;
  __syncthreads();
  // complex lines z = X_{2b} + i X_{2b+1} over the full K2 (Hermitian
  // extension; self-conjugate bins contribute their real part only)
  for (int e = threadIdx.x; e < K2 * nb1; e += blockDim.x) {
    uint32_t k, b;
    dnb1.divmod((uint32_t)e, k, b);
    const int kk = ((int)k < ldim) ? (int)k : K2 - (int)k;
    const bool selfc = (kk == 0) || (2 * kk == K2);
    float2 a = R[(2 * b) * P2 + kk];
    float2 c = ((int)(2 * b + 1) < K1) ? R[(2 * b + 1) * P2 + kk] : make_float2(0.f, 0.f);
    if (selfc) {
      a.y = 0.f;
      c.y = 0.f;
    }
    O[k * P1 + b] = ((int)k < ldim) ? make_float2(a.x - c.y, a.y + c.x) : make_float2(a.x + c.y, c.x - a.y);
  }
  __syncthreads();
  {
    const int c0 = warp * (int)dz.d, nc = min((int)dz.d, nb1 - c0);
    if (nc > 0) run_stages_w<+1>(Lz, O, R, twz, dz, P1, c0, nc, lane);
  }
  float2 *R2 = (Lz.nst & 1) ? R : O;
  __syncthreads();
  for (int e = threadIdx.x; e < K1 * K2; e += blockDim.x) {
    uint32_t y, z;
    dK2.divmod((uint32_t)e, y, z);
    const float2 v = R2[z * P1 + (y >> 1)];
    plane[e] = (y & 1) ? v.y : v.x;
  }
}

// --- x pass with the pointwise reciprocal step ---------------------------
// Lines (ky, kz) of length K0 (stride K1*ldim), B per CTA, B/8 per warp.
//   XM_FWD_DECONV : forward, then S = F iB0 iB1 iB2          (sfac, sfac.cpp:125-138)
//   XM_CONV_INV   : S given; energy/virial sums of |S|^2, S *= A iB (x2 on the
//                   kz = 0 / even-K2 Nyquist planes), inverse (de1, sfac.cpp:357-392)
//   XM_FWD_CONV_INV: forward, then the same with S = F iB, inverse (fused solve)
//   XM_EN         : S given; the energy/virial sums only (en, sfac.cpp:304-325),
//                   with exactly XM_CONV_INV's blocks and per-thread order, so
//                   en() and de1() return the same energy bit for bit.
// Energy/virial sums are FP64, reduced per CTA in a fixed order (lane tree,
// then warps in order) into partials[blockIdx.x].
enum { XM_FWD_DECONV = 0, XM_CONV_INV = 1, XM_FWD_CONV_INV = 2, XM_EN = 3 };

template <int MODE>
__global__ void __launch_bounds__(256) fft_x_kernel(FftLen L, Geom g, Influence inf, const double *__restrict__ iB0,
                                                    const double *__restrict__ iB1, const double *__restrict__ iB2,
                                                    float2 *__restrict__ data, int B, int bufsz,
                                                    double *__restrict__ partials, FastDiv Bd, FastDiv Bwd) {
  extern __shared__ float2 sm[];
  __shared__ double red[8][7];
  const int n = L.n, P = B + 1, ldim = g.ldim, K1 = g.K1;
  const long nlines = (long)K1 * ldim;
  float2 *tw = sm, *b0 = sm + n, *b1 = b0 + bufsz;
  load_twiddles(tw, L);
  const long line0 = (long)blockIdx.x * B;
  for (int e = threadIdx.x; e < B * n; e += blockDim.x) {
    uint32_t j, b;
    Bd.divmod((uint32_t)e, j, b);
    const long line = line0 + b;
    b0[j * P + b] = (line < nlines) ? data[line + j * nlines] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bw = (int)Bwd.d, c0 = warp * bw;
  float2 *cur = b0, *oth = b1;
  if (MODE == XM_FWD_DECONV || MODE == XM_FWD_CONV_INV) {
    run_stages_w<-1>(L, b0, b1, tw, Bwd, P, c0, bw, lane);
    if (L.nst & 1) {
      cur = b1;
      oth = b0;
    }
  }
  if (MODE == XM_FWD_DECONV) {
    for (int e = lane; e < bw * n; e += 32) {
      uint32_t j, bl;
      Bwd.divmod((uint32_t)e, j, bl);
      const int b = c0 + (int)bl;
      const long line = line0 + b;
      if (line >= nlines) continue;
      const int ky = (int)(line / ldim), kz = (int)(line % ldim);
      cur[j * P + b] = cscale(cur[j * P + b], (float)(iB0[j] * iB1[ky] * iB2[kz]));
    }
  } else {
    const bool even = (g.K2 % 2) == 0;
    const InfConst ic = load_ic(inf);
    double acc[7];
#pragma unroll
    for (int c = 0; c < 7; c++) acc[c] = 0.0;
    for (int e = lane; e < bw * n; e += 32) {
      uint32_t j, bl;
      Bwd.divmod((uint32_t)e, j, bl);
      const int b = c0 + (int)bl;
      const long line = line0 + b;
      if (line >= nlines) continue;
      const int ky = (int)(line / ldim), kz = (int)(line % ldim), kx = (int)j;
      const long i = ((long)kx * K1 + ky) * ldim + kz;
      const bool plane = (kz == 0) || (even && kz == ldim - 1);
      const float2 q = cur[j * P + b];
      const double ib = iB0[kx] * iB1[ky] * iB2[kz];
      double s = (double)q.x * q.x + (double)q.y * q.y;
      if (MODE == XM_FWD_CONV_INV) s *= ib * ib;  // |F iB|^2
      double A, dA[6];
      mode_influence(inf, ic, g, i, kx, ky, kz, plane, A, dA);
      acc[0] += s * A;
#pragma unroll
      for (int c = 0; c < 6; c++) acc[1 + c] += s * dA[c];
      if (MODE != XM_EN) {
        double t = A * ib * (MODE == XM_FWD_CONV_INV ? ib : 1.0);
        if (plane) t *= 2.0;
        cur[j * P + b] = cscale(q, (float)t);
      }
    }
#pragma unroll
    for (int c = 0; c < 7; c++) {
      const double v = warp_sum(acc[c]);
      if (lane == 0) red[warp][c] = v;
    }
    if (MODE != XM_EN) {
      __syncwarp();
      run_stages_w<+1>(L, cur, oth, tw, Bwd, P, c0, bw, lane);
      if (L.nst & 1) cur = oth;
    }
  }
  __syncthreads();
  if (MODE != XM_FWD_DECONV && threadIdx.x < 7) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w][threadIdx.x];
    partials[(long)blockIdx.x * kRedWords + threadIdx.x] = v;
  }
  if (MODE == XM_EN) return;
  for (int e = threadIdx.x; e < B * n; e += blockDim.x) {
    uint32_t j, b;
    Bd.divmod((uint32_t)e, j, b);
    const long line = line0 + b;
    if (line < nlines) data[line + j * nlines] = cur[j * P + b];
  }
}

// --- x pass, two-level register transform ---------------------------------
// Same modes and results as fft_x_kernel, for K0 = n1 * n2 with n1, n2 <= 16.
// B lines per CTA (a power of two, lines b fastest in the thread index so
// that every global access is B consecutive complex values); thread t*B + b
// runs step-1 task j2 = t (t < n2) and step-2 task k1 = t (t < n1) of line b.
// The exchange buffer holds element (k1, j2) of line b at (k1*n2 + j2)*B + b.
// The reciprocal step happens on the step-2 registers (all kx = k1 + n1*k2
// of the line), so forward transform, convolution and inverse transform cost
// two exchanges in total.
template <int MODE, int IM>
__global__ void __launch_bounds__(512) fft_x2_kernel(int n, int n1, int n2, const float2 *__restrict__ twg, Geom g,
                                                     Influence inf, const double *__restrict__ iB0,
                                                     const double *__restrict__ iB1, const double *__restrict__ iB2,
                                                     float2 *__restrict__ data, int lgB,
                                                     double *__restrict__ partials) {
  extern __shared__ float2 sm[];
  __shared__ double red[16][7];
  const int B = 1 << lgB;
  float2 *tw = sm, *ex = sm + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = twg[i];
  const int ldim = g.ldim, K1 = g.K1;
  const long nlines = (long)K1 * ldim;
  const int b = threadIdx.x & (B - 1), t = threadIdx.x >> lgB;
  const long line = (long)blockIdx.x * B + b;
  const bool live = line < nlines;
  const int ky = live ? (int)(line / ldim) : 0, kz = live ? (int)(line - (long)ky * ldim) : 0;
  constexpr bool FWD = (MODE == XM_FWD_DECONV || MODE == XM_FWD_CONV_INV);
  // compact influence table: the CTA's n x B entries are copied to shared
  // memory (abuf[kx * B + b]) with cp.async now and used after the forward
  // steps, so their HBM latency overlaps the transform
  double *abuf = reinterpret_cast<double *>(ex + (size_t)B * n);
  constexpr bool PREFETCH = (IM == 4 && MODE != XM_FWD_DECONV);
  if (PREFETCH) {
    for (int e = threadIdx.x; e < B * n; e += blockDim.x) {
      const int bb = e & (B - 1), kx = e >> lgB;
      const long ln = (long)blockIdx.x * B + bb;
      if (ln < nlines) {
        const int y = (int)(ln / ldim), z = (int)(ln - (long)y * ldim);
        const unsigned dst = (unsigned)__cvta_generic_to_shared(abuf + e);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst),
                     "l"(inf.A + ((long)kx * K1 + y) * ldim + z)
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  __syncthreads();
  if (FWD && t < n2) {
    const int j2 = t;
    rdft::with_radix(n1, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 u[R];
#pragma unroll
      for (int j1 = 0; j1 < R; j1++)
        u[j1] = (live && SPME_IN(j2 + n2 * j1, n, CK_FFT_LINE)) ? data[line + (long)(j2 + n2 * j1) * nlines]
                                                                : make_float2(0.f, 0.f);
      rdft::dft<R, -1>(u);
#pragma unroll
      for (int k1 = 0; k1 < R; k1++) ex[(k1 * n2 + j2) * B + b] = cmul(u[k1], tw[j2 * k1]);
    });
  }
  if (PREFETCH) asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (FWD || PREFETCH) __syncthreads();
  double acc[7];
#pragma unroll
  for (int c = 0; c < 7; c++) acc[c] = 0.0;
  if (t < n1) {
    const int k1 = t;
    rdft::with_radix(n2, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 w[R];
      if (FWD) {
#pragma unroll
        for (int j2 = 0; j2 < R; j2++) w[j2] = ex[(k1 * n2 + j2) * B + b];
        rdft::dft<R, -1>(w);
      } else {
#pragma unroll
        for (int k2 = 0; k2 < R; k2++)
          w[k2] = (live && SPME_IN(k1 + n1 * k2, n, CK_FFT_LINE)) ? data[line + (long)(k1 + n1 * k2) * nlines]
                                                                  : make_float2(0.f, 0.f);
      }
      if (MODE == XM_FWD_DECONV) {
        if (live) {
          const double s12 = iB1[ky] * iB2[kz];
#pragma unroll
          for (int k2 = 0; k2 < R; k2++) {
            const int kx = k1 + n1 * k2;
            if (SPME_IN(kx, n, CK_FFT_LINE)) data[line + (long)kx * nlines] = cscale(w[k2], (float)(iB0[kx] * s12));
          }
        }
      } else if (IM == 1) {
        // tabulated influence function: the line's values stay in registers
        // and all R modes' table loads are in flight together
        if (live) {
          const bool even = (g.K2 % 2) == 0;
          const bool plane = (kz == 0) || (even && kz == ldim - 1);
          const double s12 = iB1[ky] * iB2[kz];
#pragma unroll
          for (int k2 = 0; k2 < R; k2++) {
            const int kx = k1 + n1 * k2;
            const long i = SPME_IN(((long)kx * K1 + ky) * ldim + kz, (long)n * K1 * ldim, CK_FFT_CONV)
                               ? ((long)kx * K1 + ky) * ldim + kz
                               : 0;
            const float2 q = w[k2];
            const double ib = iB0[kx] * s12;
            double sq = (double)q.x * q.x + (double)q.y * q.y;
            if (MODE == XM_FWD_CONV_INV) sq *= ib * ib;  // |F iB|^2
            const double A = inf.A[i];
            acc[0] += sq * A;
#pragma unroll
            for (int c = 0; c < 6; c++) acc[1 + c] += sq * inf.dA[6 * i + c];
            if (MODE != XM_EN) {
              double f = A * ib * (MODE == XM_FWD_CONV_INV ? ib : 1.0);
              if (plane) f *= 2.0;
              w[k2] = cscale(q, (float)f);
            }
          }
        }
        if (MODE != XM_EN) {
          rdft::dft<R, +1>(w);
#pragma unroll
          for (int j2 = 0; j2 < R; j2++) {
            float2 c = tw[j2 * k1];
            c.y = -c.y;
            ex[(k1 * n2 + j2) * B + b] = cmul(w[j2], c);
          }
        }
      } else {
        // the pointwise step walks the line's values through the thread's
        // own exchange slots (a run-time index into registers would spill)
        float2 *slot = ex + k1 * n2 * B + b;
#pragma unroll
        for (int k2 = 0; k2 < R; k2++) slot[k2 * B] = w[k2];
        if (live) {
          const bool even = (g.K2 % 2) == 0;
          const bool plane = (kz == 0) || (even && kz == ldim - 1);
          const InfConst ic = load_ic(inf);
          const double s12 = iB1[ky] * iB2[kz];
#pragma unroll 1
          for (int k2 = 0; k2 < R; k2++) {
            const int kx = k1 + n1 * k2;
            const long i = SPME_IN(((long)kx * K1 + ky) * ldim + kz, (long)n * K1 * ldim, CK_FFT_CONV)
                               ? ((long)kx * K1 + ky) * ldim + kz
                               : 0;
            const float2 q = slot[k2 * B];
            const double ib = iB0[kx] * s12;
            double sq = (double)q.x * q.x + (double)q.y * q.y;
            if (MODE == XM_FWD_CONV_INV) sq *= ib * ib;  // |F iB|^2
            double A;
            if constexpr (PREFETCH) A = compact_acc(inf, ic, g, i, kx, ky, kz, plane, sq, abuf[kx * B + b], acc);
            else A = influence_acc<IM>(inf, ic, g, i, kx, ky, kz, plane, sq, acc);
            if (MODE != XM_EN) {
              double f = A * ib * (MODE == XM_FWD_CONV_INV ? ib : 1.0);
              if (plane) f *= 2.0;
              slot[k2 * B] = cscale(q, (float)f);
            }
          }
        }
        if (MODE != XM_EN) {
#pragma unroll
          for (int k2 = 0; k2 < R; k2++) w[k2] = slot[k2 * B];
          rdft::dft<R, +1>(w);
#pragma unroll
          for (int j2 = 0; j2 < R; j2++) {
            float2 c = tw[j2 * k1];
            c.y = -c.y;
            ex[(k1 * n2 + j2) * B + b] = cmul(w[j2], c);
          }
        }
      }
    });
  }
  if (MODE != XM_FWD_DECONV) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 7; c++) {
      const double v = warp_sum(acc[c]);
      if (lane == 0) red[warp][c] = v;
    }
  }
  if (MODE == XM_FWD_DECONV) return;
  __syncthreads();
  if (threadIdx.x < 7) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w][threadIdx.x];
    partials[(long)blockIdx.x * kRedWords + threadIdx.x] = v;
  }
  if (MODE == XM_EN) return;
  if (t < n2 && live) {
    const int j2 = t;
    rdft::with_radix(n1, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 u[R];
#pragma unroll
      for (int k1 = 0; k1 < R; k1++) u[k1] = ex[(k1 * n2 + j2) * B + b];
      rdft::dft<R, +1>(u);
#pragma unroll
      for (int j1 = 0; j1 < R; j1++)
        if (SPME_IN(j2 + n2 * j1, n, CK_FFT_LINE)) data[line + (long)(j2 + n2 * j1) * nlines] = u[j1];
    });
  }
}

// --- per-axis passes, two-level register transform -------------------------
// Thread t*B + b works on line b of the CTA's B (= 2^lgB) lines: step-1 task
// j2 = t (t < n2), step-2 task k1 = t (t < n1); exchange slot of element
// (k1, j2) of line b: (k1*n2 + j2)*B + b.  tw: exp(-2 pi i e / n), e < n.

// y pass: complex lines along y of every x-plane; line l = x*lpp + kz at
// data[x*pstride + kz + j*es].  With `partials`, CTA 0 first reduces the
// preceding x pass's energy/virial partials (needs >= 7 warps).
template <int SIGN>
__global__ void __launch_bounds__(512) fft_y2_kernel(int n, int n1, int n2, const float2 *__restrict__ twg,
                                                     float2 *__restrict__ data, long nlines, FastDiv lpp,
                                                     long pstride, int es, int lgB,
                                                     const double *__restrict__ partials, int nblocks,
                                                     const CellConst *__restrict__ cell, double *__restrict__ raw,
                                                     double *__restrict__ ev) {
  if (partials && blockIdx.x == 0) finish_partials(partials, nblocks, cell, raw, ev);
  extern __shared__ float2 sm[];
  const int B = 1 << lgB;
  float2 *tw = sm, *ex = sm + n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = twg[i];
  const int b = threadIdx.x & (B - 1), t = threadIdx.x >> lgB;
  const long l = (long)blockIdx.x * B + b;
  const bool live = l < nlines;
  uint32_t pl = 0, r = 0;
  if (live) lpp.divmod((uint32_t)l, pl, r);
  const long base = (long)pl * pstride + r;
  __syncthreads();
  if (t < n2) {
    const int j2 = t;
    rdft::with_radix(n1, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 u[R];
#pragma unroll
      for (int j1 = 0; j1 < R; j1++)
        u[j1] = (live && SPME_IN(j2 + n2 * j1, n, CK_FFT_LINE)) ? data[base + (long)(j2 + n2 * j1) * es]
                                                                : make_float2(0.f, 0.f);
      rdft::dft<R, SIGN>(u);
#pragma unroll
      for (int k1 = 0; k1 < R; k1++) ex[(k1 * n2 + j2) * B + b] = cmul(u[k1], twid<SIGN>(tw, j2 * k1));
    });
  }
  __syncthreads();
  if (t < n1 && live) {
    const int k1 = t;
    rdft::with_radix(n2, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 w[R];
#pragma unroll
      for (int j2 = 0; j2 < R; j2++) w[j2] = ex[(k1 * n2 + j2) * B + b];
      rdft::dft<R, SIGN>(w);
#pragma unroll
      for (int k2 = 0; k2 < R; k2++)
        if (SPME_IN(k1 + n1 * k2, n, CK_FFT_LINE)) data[base + (long)(k1 + n1 * k2) * es] = w[k2];
    });
  }
}

// Copies the contiguous block src[0 .. valid) (elements of T in rows of
// `width`) into sh[r * pitch + c] for the first `total` elements, zero past
// `valid`.  16-byte loads, four per thread issued before any of them is
// stored, so that a small CTA keeps many loads in flight (a row-by-row loop
// whose stores wait on each load leaves one in flight per thread); the row
// and column of each element are advanced incrementally.  src must be
// 16-byte aligned.
template <typename T>
__device__ __forceinline__ void stage_rows(const T *__restrict__ src, int valid, int total, int width, int pitch,
                                           T *sh) {
  constexpr int PER = 16 / sizeof(T);
  const int nv = (total + PER - 1) / PER;
  const int step = PER * blockDim.x;  // elements per pass of the CTA
  const int sr = step / width, sc = step - sr * width;
  int r = (PER * threadIdx.x) / width, c = PER * threadIdx.x - r * width;
  for (int i = threadIdx.x; i < nv; i += 4 * blockDim.x) {
    float4 v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int iu = i + u * blockDim.x, f = iu * PER;
      if (iu < nv && f + PER <= valid) {
        v[u] = __ldg(reinterpret_cast<const float4 *>(src) + iu);
      } else {
        T *e = reinterpret_cast<T *>(&v[u]);
#pragma unroll
        for (int k = 0; k < PER; k++) e[k] = (iu < nv && f + k < valid) ? src[f + k] : T{};
      }
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int iu = i + u * blockDim.x;
      if (iu < nv) {
        const T *e = reinterpret_cast<const T *>(&v[u]);
        int rr = r, cc = c;
#pragma unroll
        for (int k = 0; k < PER; k++) {
          if (iu * PER + k < total) sh[rr * pitch + cc] = e[k];
          if (++cc == width) {
            cc = 0;
            rr++;
          }
        }
      }
      r += sr;
      c += sc;
      if (c >= width) {
        c -= width;
        r++;
      }
    }
  }
}

// z pass, real to half-complex: 2B consecutive real rows of length n per
// CTA (row pair b forms the complex line row[2b] + i row[2b+1]); the rows
// are read and the ldim = n/2 + 1 outputs written as contiguous blocks.
// Shared: tw[n] | ex[B*n] | rows (2B x (n+1) floats), later Z (B x (n+1) complex).
__global__ void __launch_bounds__(512) fft_zr2c2_kernel(int n, int n1, int n2, const float2 *__restrict__ twg,
                                                        const float *__restrict__ rin, float2 *__restrict__ cout,
                                                        long nrows, int lgB) {
  extern __shared__ float2 sm[];
  const int B = 1 << lgB, ldim = n / 2 + 1, RP = n + 1, ZP = n + 1;
  float2 *tw = sm, *ex = sm + n, *Z = ex + B * n;
  float *rows = reinterpret_cast<float *>(Z);
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = twg[i];
  const long row0 = (long)blockIdx.x * 2 * B;
  const int nr = (int)min((long)(2 * B), nrows - row0);
  const float *src = rin + row0 * n;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    stage_rows<float>(src, nr * n, 2 * B * n, n, RP, rows);
  } else {
    for (int rr = threadIdx.x >> 5; rr < 2 * B; rr += nw)
      for (int j = lane; j < n; j += 32) rows[rr * RP + j] = (rr < nr) ? src[(long)rr * n + j] : 0.f;
  }
  __syncthreads();
  const int b = threadIdx.x & (B - 1), t = threadIdx.x >> lgB;
  if (t < n2) {
    const int j2 = t;
    const float *ra = rows + (2 * b) * RP, *rb = ra + RP;
    rdft::with_radix(n1, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 u[R];
#pragma unroll
      for (int j1 = 0; j1 < R; j1++) u[j1] = make_float2(ra[j2 + n2 * j1], rb[j2 + n2 * j1]);
      rdft::dft<R, -1>(u);
#pragma unroll
      for (int k1 = 0; k1 < R; k1++) ex[(k1 * n2 + j2) * B + b] = cmul(u[k1], tw[j2 * k1]);
    });
  }
  __syncthreads();
  if (t < n1) {
    const int k1 = t;
    rdft::with_radix(n2, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 w[R];
#pragma unroll
      for (int j2 = 0; j2 < R; j2++) w[j2] = ex[(k1 * n2 + j2) * B + b];
      rdft::dft<R, -1>(w);
#pragma unroll
      for (int k2 = 0; k2 < R; k2++)
        if (SPME_IN(k1 + n1 * k2, n, CK_FFT_LINE)) Z[b * ZP + k1 + n1 * k2] = w[k2];
    });
  }
  __syncthreads();
  float2 *dst = cout + row0 * ldim;
  for (int rr = threadIdx.x >> 5; rr < nr; rr += nw) {
    const float2 *zb = Z + (rr >> 1) * ZP;
    for (int k = lane; k < ldim; k += 32) {
      const float2 u = zb[k], v = zb[k == 0 ? 0 : n - k];
      dst[(long)rr * ldim + k] = (rr & 1) ? make_float2(0.5f * (u.y + v.y), -0.5f * (u.x - v.x))
                                          : make_float2(0.5f * (u.x + v.x), 0.5f * (u.y - v.y));
    }
  }
}

// z pass, half-complex to real: the inverse of fft_zr2c2_kernel.  The
// complex line of row pair b is X_2b + i X_2b+1 over the full length (the
// Hermitian extension; self-conjugate bins keep their real parts only, as a
// c2r transform ignores their imaginary parts).
// Shared: tw[n] | ex[B*n] | H (2B x (ldim+1) complex), later rows (2B x (n+1) floats).
__global__ void __launch_bounds__(512) fft_zc2r2_kernel(int n, int n1, int n2, const float2 *__restrict__ twg,
                                                        const float2 *__restrict__ cin, float *__restrict__ rout,
                                                        long nrows, int lgB) {
  extern __shared__ float2 sm[];
  const int B = 1 << lgB, ldim = n / 2 + 1, HP = ldim + 1, RP = n + 1;
  float2 *tw = sm, *ex = sm + n, *H = ex + B * n;
  float *rows = reinterpret_cast<float *>(H);
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = twg[i];
  const long row0 = (long)blockIdx.x * 2 * B;
  const int nr = (int)min((long)(2 * B), nrows - row0);
  const float2 *src = cin + row0 * ldim;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    stage_rows<float2>(src, nr * ldim, 2 * B * ldim, ldim, HP, H);
  } else {
    for (int rr = threadIdx.x >> 5; rr < 2 * B; rr += nw)
      for (int k = lane; k < ldim; k += 32)
        H[rr * HP + k] = (rr < nr) ? src[(long)rr * ldim + k] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const int b = threadIdx.x & (B - 1), t = threadIdx.x >> lgB;
  if (t < n2) {
    const int j2 = t;
    const float2 *ha = H + (2 * b) * HP, *hb = ha + HP;
    rdft::with_radix(n1, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 u[R];
#pragma unroll
      for (int j1 = 0; j1 < R; j1++) {
        const int k = j2 + n2 * j1;
        const bool lo = k < ldim;
        const int kk = lo ? k : n - k;
        float2 a = ha[kk], c = hb[kk];
        if (kk == 0 || 2 * kk == n) {
          a.y = 0.f;
          c.y = 0.f;
        }
        u[j1] = lo ? make_float2(a.x - c.y, a.y + c.x) : make_float2(a.x + c.y, c.x - a.y);
      }
      rdft::dft<R, +1>(u);
#pragma unroll
      for (int k1 = 0; k1 < R; k1++) ex[(k1 * n2 + j2) * B + b] = cmul(u[k1], twid<+1>(tw, j2 * k1));
    });
  }
  __syncthreads();
  if (t < n1) {
    const int k1 = t;
    float *ra = rows + (2 * b) * RP, *rb = ra + RP;
    rdft::with_radix(n2, [&](auto RI) {
      constexpr int R = decltype(RI)::value;
      float2 w[R];
#pragma unroll
      for (int j2 = 0; j2 < R; j2++) w[j2] = ex[(k1 * n2 + j2) * B + b];
      rdft::dft<R, +1>(w);
#pragma unroll
      for (int k2 = 0; k2 < R; k2++) {
        ra[k1 + n1 * k2] = w[k2].x;
        rb[k1 + n1 * k2] = w[k2].y;
      }
    });
  }
  __syncthreads();
  float *dst = rout + row0 * n;
  for (int rr = threadIdx.x >> 5; rr < nr; rr += nw)
    for (int j = lane; j < n; j += 32) dst[(long)rr * n + j] = rows[rr * RP + j];
}

// FP32 twiddles exp(-2 pi i k / n), evaluated in FP64.
__global__ void fft_twiddle_kernel(int n, float2 *tw) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double s, c;
  sincospi(-2.0 * (double)k / (double)n, &s, &c);
  tw[k] = make_float2((float)c, (float)s);
}

int fft_make_len(FftLen &L, int n, float2 *tw_dev, cudaStream_t st) {
  L.n = n;
  L.nst = 0;
  int m = n;
  while (m % 4 == 0) { L.rad[L.nst++] = 4; m /= 4; }
  while (m % 2 == 0) { L.rad[L.nst++] = 2; m /= 2; }
  for (int p = 3; m > 1; p += 2) {
    while (m % p == 0) { L.rad[L.nst++] = p; m /= p; }
    if ((long)p * p > m && m > 1) { L.rad[L.nst++] = m; m = 1; }
  }
  int Ns = 1;
  for (int s = 0; s < L.nst; s++) {
    L.ns[s] = FastDiv((uint32_t)Ns);
    Ns *= L.rad[s];
  }
  L.tw = tw_dev;
  fft_twiddle_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, tw_dev);
  return 1;
}

// Lines per CTA and shared-memory size for a pass over `nlines` lines of
// length n: as many lines as fit 96 KB, then fewer while the pass would have
// under four CTAs per SM (148 SMs), down to 4 lines (32-byte segments).
static void fft_shape(int n, long nlines, int &B, int &bufsz, size_t &smem) {
  B = 64;
  while (B > 1 && (size_t)(n + 2 * (size_t)n * (B + 1)) * sizeof(float2) > 96 * 1024) B >>= 1;
  while (B > 4 && (nlines + B - 1) / B < 4 * 148) B >>= 1;
  bufsz = n * (B + 1);
  const int need_c2r = 2 * B * (n / 2 + 1);
  if (need_c2r > bufsz) bufsz = need_c2r;
  smem = (size_t)(n + 2 * (size_t)bufsz) * sizeof(float2);
}

void fft_prepare_kernels() {
  const int lim = 200 * 1024;
  cudaFuncSetAttribute((const void *)fft_z_r2c_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_z_c2r_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_strided_kernel<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_strided_kernel<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_plane_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_plane_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_x_kernel<XM_FWD_DECONV>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_x_kernel<XM_CONV_INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_x_kernel<XM_FWD_CONV_INV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       lim);
  cudaFuncSetAttribute((const void *)fft_x_kernel<XM_EN>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  const void *x2[] = {(const void *)fft_x2_kernel<XM_FWD_DECONV, 1>, (const void *)fft_x2_kernel<XM_CONV_INV, 1>,
                      (const void *)fft_x2_kernel<XM_CONV_INV, 2>, (const void *)fft_x2_kernel<XM_CONV_INV, 4>,
                      (const void *)fft_x2_kernel<XM_FWD_CONV_INV, 1>, (const void *)fft_x2_kernel<XM_FWD_CONV_INV, 2>,
                      (const void *)fft_x2_kernel<XM_FWD_CONV_INV, 4>, (const void *)fft_x2_kernel<XM_EN, 1>,
                      (const void *)fft_x2_kernel<XM_EN, 2>, (const void *)fft_x2_kernel<XM_EN, 4>};
  for (const void *f : x2) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_y2_kernel<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_y2_kernel<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_zr2c2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute((const void *)fft_zc2r2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

// Shared memory of the plane kernels: twiddles + two buffers of `sz`.
static size_t plane_smem(int K1, int K2, int &sz) {
  const int ldim = K2 / 2 + 1, nb1 = (K1 + 1) / 2;
  sz = K2 * (nb1 + 1);
  if (K1 * (ldim + 1) > sz) sz = K1 * (ldim + 1);
  return (size_t)(K1 + K2 + 2 * (size_t)sz) * sizeof(float2);
}
constexpr size_t kPlaneSmemMax = 200 * 1024;

bool fft_plane_fits(int K1, int K2) {
  int sz;
  return plane_smem(K1, K2, sz) <= kPlaneSmemMax;
}

long fft_x_blocks_max(int K1, int K2) { return ((long)K1 * (K2 / 2 + 1) + 7) / 8; }

// Shape of a two-level per-axis pass over `nlines` lines of length n:
// B = 2^lgB lines per CTA (8..32), B*max(n1, n2) threads (at least
// min_threads, at most 512), B halved while fewer than two CTAs per SM
// (148 SMs) would run.  False when n has no n1 * n2 split.
static bool lines2_shape(int n, long nlines, int min_threads, int &n1, int &n2, int &lgB, int &threads) {
  if (!rdft::split_line(n, n1, n2)) return false;
  const int m = n1 > n2 ? n1 : n2;
  int B = 8;
  while (B < 32 && B * m < 128) B <<= 1;
  while (B > 8 && (nlines + B - 1) / B < 2 * 148) B >>= 1;
  while (B > 8 && B * m > 512) B >>= 1;
  if (B * m > 512) return false;
  lgB = 0;
  while ((1 << lgB) < B) lgB++;
  threads = (B * m + 31) / 32 * 32;
  if (threads < min_threads) threads = min_threads;
  return true;
}

// Which z/y implementation a plan uses: the fused plane kernels (an x-plane
// in shared memory), the two-level per-axis passes, or the Stockham
// per-axis passes (any length).
enum { ZY_PLANE = 1, ZY_TWO_LEVEL = 2, ZY_STOCKHAM = 3 };
static int zy_choice(const FftPlan3 &F) {
  const int K1 = F.len[1].n, K2 = F.len[2].n;
  int sz, a, b;
  const bool plane = plane_smem(K1, K2, sz) <= kPlaneSmemMax;
  const bool two = rdft::split_line(K1, a, b) && rdft::split_line(K2, a, b);
  if (F.zy_mode == ZY_PLANE && plane) return ZY_PLANE;
  if (F.zy_mode == ZY_STOCKHAM) return ZY_STOCKHAM;
  if (two) return ZY_TWO_LEVEL;
  return plane ? ZY_PLANE : ZY_STOCKHAM;
}

// Forward z (r2c) and y transforms.
int fwd_zy(const FftPlan3 &F, const float *real, float2 *cplx, cudaStream_t st) {
  const int K0 = F.len[0].n, K1 = F.len[1].n, K2 = F.len[2].n, ldim = K2 / 2 + 1;
  const int zy = zy_choice(F);
  if (zy == ZY_PLANE) {
    int sz;
    const size_t psm = plane_smem(K1, K2, sz);
    const int nb1 = (K1 + 1) / 2;
    fft_plane_fwd_kernel<<<K0, 512, psm, st>>>(F.len[1], F.len[2], real, cplx, sz, FastDiv((nb1 + 15) / 16),
                                               FastDiv((ldim + 15) / 16), FastDiv(K2), FastDiv(ldim));
    return 1;
  }
  const long nrows = (long)K0 * K1;
  const long nl = (long)K0 * ldim;
  if (zy == ZY_TWO_LEVEL) {
    int n1, n2, lgB, thr;
    lines2_shape(K2, (nrows + 1) / 2, 0, n1, n2, lgB, thr);
    int B = 1 << lgB;
    size_t smem = (size_t)(K2 + (size_t)B * K2 + (size_t)B * (K2 + 4)) * sizeof(float2);
    fft_zr2c2_kernel<<<(unsigned)((nrows + 2 * B - 1) / (2 * B)), thr, smem, st>>>(K2, n1, n2, F.len[2].tw, real,
                                                                                  cplx, nrows, lgB);
    lines2_shape(K1, nl, 0, n1, n2, lgB, thr);
    B = 1 << lgB;
    smem = (size_t)(K1 + (size_t)B * K1) * sizeof(float2);
    fft_y2_kernel<-1><<<(unsigned)((nl + B - 1) / B), thr, smem, st>>>(K1, n1, n2, F.len[1].tw, cplx, nl,
                                                                       FastDiv(ldim), (long)K1 * ldim, ldim, lgB,
                                                                       nullptr, 0, nullptr, nullptr, nullptr);
    return 2;
  }
  int B, bufsz;
  size_t smem;
  fft_shape(K2, (nrows + 1) / 2, B, bufsz, smem);
  fft_z_r2c_kernel<<<(unsigned)((nrows + 2 * B - 1) / (2 * B)), 256, smem, st>>>(F.len[2], (int)nrows, real, cplx,
                                                                                 ldim, B, bufsz, FastDiv(B));
  fft_shape(K1, nl, B, bufsz, smem);
  DeconvArgs none{};
  fft_strided_kernel<-1><<<(int)((nl + B - 1) / B), 256, smem, st>>>(F.len[1], nl, ldim, (long)K1 * ldim, ldim,
                                                                     cplx, B, bufsz, none, FastDiv(B));
  return 2;
}

// Inverse y and z (c2r) transforms; with `partials`, the energy/virial
// partials are reduced first (inside the first kernel when it can).
int inv_yz(const FftPlan3 &F, float2 *cplx, float *real, const double *partials, int nblocks,
           const CellConst *cell, double *raw, double *ev, cudaStream_t st) {
  const int K0 = F.len[0].n, K1 = F.len[1].n, K2 = F.len[2].n, ldim = K2 / 2 + 1;
  const int zy = zy_choice(F);
  if (zy == ZY_PLANE) {
    int sz;
    const size_t psm = plane_smem(K1, K2, sz);
    const int nb1 = (K1 + 1) / 2;
    fft_plane_inv_kernel<<<K0, 512, psm, st>>>(F.len[1], F.len[2], cplx, real, sz, partials, nblocks, cell, raw,
                                               ev, FastDiv((nb1 + 15) / 16), FastDiv((ldim + 15) / 16), FastDiv(K2),
                                               FastDiv(ldim), FastDiv(nb1));
    return 1;
  }
  const long nrows = (long)K0 * K1;
  const long nl = (long)K0 * ldim;
  if (zy == ZY_TWO_LEVEL) {
    int n1, n2, lgB, thr;
    lines2_shape(K1, nl, partials ? 256 : 0, n1, n2, lgB, thr);
    int B = 1 << lgB;
    size_t smem = (size_t)(K1 + (size_t)B * K1) * sizeof(float2);
    fft_y2_kernel<+1><<<(unsigned)((nl + B - 1) / B), thr, smem, st>>>(K1, n1, n2, F.len[1].tw, cplx, nl,
                                                                       FastDiv(ldim), (long)K1 * ldim, ldim, lgB,
                                                                       partials, nblocks, cell, raw, ev);
    lines2_shape(K2, (nrows + 1) / 2, 0, n1, n2, lgB, thr);
    B = 1 << lgB;
    smem = (size_t)(K2 + (size_t)B * K2 + (size_t)B * (K2 + 4)) * sizeof(float2);
    fft_zc2r2_kernel<<<(unsigned)((nrows + 2 * B - 1) / (2 * B)), thr, smem, st>>>(K2, n1, n2, F.len[2].tw, cplx,
                                                                                  real, nrows, lgB);
    return 2;
  }
  int k = 0;
  if (partials) k += launch_finish(partials, nblocks, cell, raw, ev, st);
  int B, bufsz;
  size_t smem;
  fft_shape(K1, nl, B, bufsz, smem);
  DeconvArgs none{};
  fft_strided_kernel<+1><<<(int)((nl + B - 1) / B), 256, smem, st>>>(F.len[1], nl, ldim, (long)K1 * ldim, ldim,
                                                                     cplx, B, bufsz, none, FastDiv(B));
  fft_shape(K2, (nrows + 1) / 2, B, bufsz, smem);
  fft_z_c2r_kernel<<<(unsigned)((nrows + 2 * B - 1) / (2 * B)), 256, smem, st>>>(F.len[2], (int)nrows, cplx, real,
                                                                                 ldim, B, bufsz, FastDiv(B));
  return k + 2;
}

// Lines per CTA of the x pass: 8 warps x bw lines; bw is the smallest power
// of two giving every lane a butterfly in the first stage, halved while the
// pass would have under two CTAs per SM (148 SMs); x_lines overrides it.
static int x_lines_per_cta(const FftPlan3 &F, int n, long nlines) {
  int B = (F.x_lines + 7) / 8 * 8;
  if (B <= 0) {
    const int m = F.len[0].nst > 0 ? n / F.len[0].rad[0] : n;
    int bw = 1;
    while (bw < 8 && m * bw < 32) bw <<= 1;
    while (bw > 1 && (nlines + 8 * bw - 1) / (8 * bw) < 2 * 148) bw >>= 1;
    B = 8 * bw;
  }
  if (B < 8) B = 8;
  return B;
}

// Two-level x pass: lines per CTA B = 2^lgB (8..32) with B*max(n1, n2)
// threads (<= 512): grown to CTAs of at least 8 warps (each CTA pays for its
// twiddles and setup once), halved only while the SMs would not all get one
// (up to 1/16 of them may idle: 147 CTAs of 32 lines beat 294 of 16 and 588
// of 8 for a 96^3 grid, 98 vs 100 vs 102 us per solve); x_lines overrides B.
// Returns false when K0 has no n1 * n2 split.
static bool x2_shape(const FftPlan3 &F, int n, long nlines, int &n1, int &n2, int &lgB, int &threads) {
  if (!rdft::split_line(n, n1, n2)) return false;
  const int m = n1 > n2 ? n1 : n2;
  int B;
  if (F.x_lines > 0) {
    B = 8;
    while (B < F.x_lines && B < 32) B <<= 1;
  } else {
    B = 8;
    while (B < 32 && B * m < 256) B <<= 1;
    while (B > 8 && (nlines + B - 1) / B < 148 - 148 / 16) B >>= 1;
  }
  while (B > 8 && B * m > 512) B >>= 1;
  if (B * m > 512) return false;
  lgB = 0;
  while ((1 << lgB) < B) lgB++;
  threads = (B * m + 31) / 32 * 32;
  return true;
}

template <int MODE>
static int x_pass(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                  const double *iB2, float2 *cplx, double *partials, int &nblocks, cudaStream_t st) {
  const long nl = (long)g.K1 * g.ldim;
  const int n = g.K0;
  int n1, n2, lgB, threads;
  if (x2_shape(F, n, nl, n1, n2, lgB, threads)) {
    const int B = 1 << lgB;
    const size_t smem = (size_t)(n + (size_t)B * n) * sizeof(float2);
    nblocks = (int)((nl + B - 1) / B);
    auto go = [&](auto IMC) {
      constexpr int IM = decltype(IMC)::value;
      const size_t sm = smem + (IM == 4 && MODE != XM_FWD_DECONV ? (size_t)B * n * sizeof(double) : 0);
      fft_x2_kernel<MODE, IM><<<nblocks, threads, sm, st>>>(n, n1, n2, F.len[0].tw, g, inf, iB0, iB1, iB2, cplx,
                                                            lgB, partials);
    };
    if (MODE == XM_FWD_DECONV || inf.mode == 1) go(std::integral_constant<int, 1>{});
    else if (inf.mode == 4) go(std::integral_constant<int, 4>{});
    else go(std::integral_constant<int, 2>{});
    return 1;
  }
  int B = x_lines_per_cta(F, n, nl);
  int bufsz = n * (B + 1);
  size_t smem = (size_t)(n + 2 * (size_t)bufsz) * sizeof(float2);
  while (smem > 200 * 1024 && B > 8) {
    B >>= 1;
    bufsz = n * (B + 1);
    smem = (size_t)(n + 2 * (size_t)bufsz) * sizeof(float2);
  }
  nblocks = (int)((nl + B - 1) / B);
  fft_x_kernel<MODE><<<nblocks, 256, smem, st>>>(F.len[0], g, inf, iB0, iB1, iB2, cplx, B, bufsz, partials,
                                                 FastDiv(B), FastDiv(B / 8));
  return 1;
}

int launch_fft_forward(const FftPlan3 &F, const Geom &g, const float *real, float2 *cplx, const DeconvArgs &dc,
                       cudaStream_t st) {
  int nb;
  Influence none{};
  return fwd_zy(F, real, cplx, st) + x_pass<XM_FWD_DECONV>(F, g, none, dc.iB0, dc.iB1, dc.iB2, cplx, nullptr, nb, st);
}

int launch_conv_inverse(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0,
                        const double *iB1, const double *iB2, float2 *cplx, float *real, double *partials,
                        double *raw, double *ev, cudaStream_t st) {
  int nb;
  int k = x_pass<XM_CONV_INV>(F, g, inf, iB0, iB1, iB2, cplx, partials, nb, st);
  return k + inv_yz(F, cplx, real, partials, nb, g.cell, raw, ev, st);
}

int launch_conv_energy(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                       const double *iB2, float2 *cplx, double *partials, double *raw, cudaStream_t st) {
  int nb;
  const int k = x_pass<XM_CONV_INV>(F, g, inf, iB0, iB1, iB2, cplx, partials, nb, st);
  return k + launch_finish(partials, nb, g.cell, raw, nullptr, st);
}

int launch_energy(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                  const double *iB2, float2 *cplx, double *partials, double *raw, cudaStream_t st) {
  int nb;
  x_pass<XM_EN>(F, g, inf, iB0, iB1, iB2, cplx, partials, nb, st);
  return 1 + launch_finish(partials, nb, g.cell, raw, nullptr, st);
}

int launch_x_conv(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                  const double *iB2, float2 *cplx, double *partials, int &nblocks, cudaStream_t st) {
  return x_pass<XM_FWD_CONV_INV>(F, g, inf, iB0, iB1, iB2, cplx, partials, nblocks, st);
}

int launch_fft_conv_solve(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0,
                          const double *iB1, const double *iB2, const float *real_in, float2 *cplx,
                          float *real_out, double *partials, double *raw, double *ev, cudaStream_t st) {
  int nb;
  int k = fwd_zy(F, real_in, cplx, st);
  k += x_pass<XM_FWD_CONV_INV>(F, g, inf, iB0, iB1, iB2, cplx, partials, nb, st);
  return k + inv_yz(F, cplx, real_out, partials, nb, g.cell, raw, ev, st);
}

}  // namespace spme
