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
#include "spme_kernels.hpp"

namespace spme {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// sign * i * a
template <int SIGN>
__device__ __forceinline__ float2 rot(float2 a) {
  return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}
template <int SIGN>
__device__ __forceinline__ float2 twid(const float2 *tw, int k) {
  float2 w = tw[k];
  if (SIGN > 0) w.y = -w.y;
  return w;
}

// In-register R-point DFTs, X[q] = sum_r v[r] exp(SIGN 2 pi i r q / R).
template <int R, int SIGN>
struct Bfly;

template <int SIGN>
struct Bfly<2, SIGN> {
  __device__ static void run(float2 *v, const float2 *, int) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <int SIGN>
struct Bfly<3, SIGN> {
  __device__ static void run(float2 *v, const float2 *, int) {
    const float c = -0.5f, s = 0.86602540378443864676f;
    float2 t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    float2 mid = make_float2(fmaf(c, t.x, v[0].x), fmaf(c, t.y, v[0].y));
    float2 r = rot<SIGN>(cscale(d, s));
    v[0] = cadd(v[0], t);
    v[1] = cadd(mid, r);
    v[2] = csub(mid, r);
  }
};
template <int SIGN>
struct Bfly<4, SIGN> {
  __device__ static void run(float2 *v, const float2 *, int) {
    float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    float2 t2 = cadd(v[1], v[3]), t3 = rot<SIGN>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};
template <int SIGN>
struct Bfly<5, SIGN> {
  __device__ static void run(float2 *v, const float2 *, int) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    float2 m1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    float2 m2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    float2 r1 = rot<SIGN>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    float2 r2 = rot<SIGN>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(m1, r1);
    v[4] = csub(m1, r1);
    v[2] = cadd(m2, r2);
    v[3] = csub(m2, r2);
  }
};
// Any other radix: direct DFT with roots from the length-n table
// (w_R = tw[n/R]).
template <int R, int SIGN>
struct Bfly {
  __device__ static void run(float2 *v, const float2 *tw, int n) {
    float2 out[R];
    const int step = n / R;
#pragma unroll
    for (int q = 0; q < R; q++) {
      float2 acc = v[0];
#pragma unroll
      for (int r = 1; r < R; r++) acc = cadd(acc, cmul(v[r], twid<SIGN>(tw, ((r * q) % R) * step)));
      out[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; q++) v[q] = out[q];
  }
};

// One Stockham stage over B lines: in/out are [j][b] with pitch P.
template <int R, int SIGN>
__device__ __forceinline__ void stage(const float2 *in, float2 *out, const float2 *tw, int n, int Ns,
                                      int B, int P) {
  const int m = n / R;
  const int twstep = n / (Ns * R);
  for (int item = threadIdx.x; item < m * B; item += blockDim.x) {
    const int b = item % B, j = item / B;
    const int k = j % Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      v[r] = in[(j + r * m) * P + b];
      if (r > 0) v[r] = cmul(v[r], twid<SIGN>(tw, r * k * twstep));
    }
    Bfly<R, SIGN>::run(v, tw, n);
    const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) out[(idxD + r * Ns) * P + b] = v[r];
  }
}

// Radices outside the compiled set: the same stage, reading the inputs
// straight from shared memory (O(R^2) per butterfly, any R).
template <int SIGN>
__device__ void stage_any(const float2 *in, float2 *out, const float2 *tw, int n, int R, int Ns, int B,
                          int P) {
  const int m = n / R;
  const int twstep = n / (Ns * R);
  const int step = n / R;
  for (int item = threadIdx.x; item < m * B * R; item += blockDim.x) {
    const int q = item % R;
    const int rest = item / R;
    const int b = rest % B, j = rest / B;
    const int k = j % Ns;
    float2 acc = make_float2(0.f, 0.f);
    for (int r = 0; r < R; r++) {
      float2 x = in[(j + r * m) * P + b];
      x = cmul(x, twid<SIGN>(tw, r * k * twstep));
      acc = cadd(acc, cmul(x, twid<SIGN>(tw, ((r * q) % R) * step)));
    }
    const int idxD = (j / Ns) * Ns * R + k;
    out[(idxD + q * Ns) * P + b] = acc;
  }
}

// Runs all stages; returns the buffer holding the result.
template <int SIGN>
__device__ float2 *run_stages(const FftLen &L, float2 *b0, float2 *b1, const float2 *tw, int B, int P) {
  int Ns = 1;
  for (int s = 0; s < L.nst; s++) {
    const int R = L.rad[s];
    switch (R) {
      case 2: stage<2, SIGN>(b0, b1, tw, L.n, Ns, B, P); break;
      case 3: stage<3, SIGN>(b0, b1, tw, L.n, Ns, B, P); break;
      case 4: stage<4, SIGN>(b0, b1, tw, L.n, Ns, B, P); break;
      case 5: stage<5, SIGN>(b0, b1, tw, L.n, Ns, B, P); break;
      case 7: stage<7, SIGN>(b0, b1, tw, L.n, Ns, B, P); break;
      default: stage_any<SIGN>(b0, b1, tw, L.n, R, Ns, B, P); break;
    }
    __syncthreads();
    float2 *t = b0;
    b0 = b1;
    b1 = t;
    Ns *= R;
  }
  return b0;
}

__device__ __forceinline__ void load_twiddles(float2 *tw_s, const FftLen &L) {
  for (int i = threadIdx.x; i < L.n; i += blockDim.x) tw_s[i] = L.tw[i];
}

// --- z pass, forward: real rows -> half-complex rows --------------------
// CTA handles 2B real rows (B complex lines); row pitch K2 (real) / ldim.
__global__ void __launch_bounds__(256) fft_z_r2c_kernel(FftLen L, int nrows, const float *__restrict__ rin,
                                                        float2 *__restrict__ cout, int ldim, int B,
                                                        int bufsz) {
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
  float2 *res = run_stages<-1>(L, b0, b1, tw, B, P);
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
                                                        int bufsz) {
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
  float2 *res = run_stages<+1>(L, b0, b1, tw, B, P);
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
                                                          int bufsz, DeconvArgs dc) {
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
  float2 *res = run_stages<SIGN>(L, b0, b1, tw, B, P);
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
  L.tw = tw_dev;
  fft_twiddle_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, tw_dev);
  return 1;
}

// Lines per CTA and shared-memory size for a pass over lines of length n.
static void fft_shape(int n, int &B, int &bufsz, size_t &smem) {
  B = 64;
  while (B > 1 && (size_t)(n + 2 * (size_t)n * (B + 1)) * sizeof(float2) > 96 * 1024) B >>= 1;
  bufsz = n * (B + 1);
  const int need_c2r = 2 * B * (n / 2 + 1);
  if (need_c2r > bufsz) bufsz = need_c2r;
  smem = (size_t)(n + 2 * (size_t)bufsz) * sizeof(float2);
}

static void set_smem(const void *fn, size_t smem) {
  if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

int launch_fft_forward(const FftPlan3 &F, const float *real, float2 *cplx, const DeconvArgs &dc,
                       cudaStream_t st) {
  const int K0 = F.len[0].n, K1 = F.len[1].n, K2 = F.len[2].n, ldim = K2 / 2 + 1;
  int B, bufsz;
  size_t smem;
  // z: real rows -> half-complex rows
  fft_shape(K2, B, bufsz, smem);
  const int nrows = K0 * K1;
  set_smem((const void *)fft_z_r2c_kernel, smem);
  fft_z_r2c_kernel<<<(nrows + 2 * B - 1) / (2 * B), 256, smem, st>>>(F.len[2], nrows, real, cplx, ldim, B,
                                                                      bufsz);
  DeconvArgs none{};
  // y: lines (x, kz), stride ldim
  fft_shape(K1, B, bufsz, smem);
  set_smem((const void *)fft_strided_kernel<-1>, smem);
  long nl = (long)K0 * ldim;
  fft_strided_kernel<-1><<<(int)((nl + B - 1) / B), 256, smem, st>>>(F.len[1], nl, ldim, (long)K1 * ldim,
                                                                     ldim, cplx, B, bufsz, none);
  // x: lines (y, kz), stride K1*ldim, with the moduli division
  fft_shape(K0, B, bufsz, smem);
  set_smem((const void *)fft_strided_kernel<-1>, smem);
  nl = (long)K1 * ldim;
  fft_strided_kernel<-1><<<(int)((nl + B - 1) / B), 256, smem, st>>>(F.len[0], nl, nl, 0, nl, cplx, B,
                                                                     bufsz, dc);
  return 3;
}

int launch_fft_inverse(const FftPlan3 &F, float2 *cplx, float *real, cudaStream_t st) {
  const int K0 = F.len[0].n, K1 = F.len[1].n, K2 = F.len[2].n, ldim = K2 / 2 + 1;
  int B, bufsz;
  size_t smem;
  DeconvArgs none{};
  fft_shape(K0, B, bufsz, smem);
  set_smem((const void *)fft_strided_kernel<+1>, smem);
  long nl = (long)K1 * ldim;
  fft_strided_kernel<+1><<<(int)((nl + B - 1) / B), 256, smem, st>>>(F.len[0], nl, nl, 0, nl, cplx, B,
                                                                     bufsz, none);
  fft_shape(K1, B, bufsz, smem);
  set_smem((const void *)fft_strided_kernel<+1>, smem);
  nl = (long)K0 * ldim;
  fft_strided_kernel<+1><<<(int)((nl + B - 1) / B), 256, smem, st>>>(F.len[1], nl, ldim, (long)K1 * ldim,
                                                                     ldim, cplx, B, bufsz, none);
  fft_shape(K2, B, bufsz, smem);
  const int nrows = K0 * K1;
  set_smem((const void *)fft_z_c2r_kernel, smem);
  fft_z_c2r_kernel<<<(nrows + 2 * B - 1) / (2 * B), 256, smem, st>>>(F.len[2], nrows, cplx, real, ldim, B,
                                                                      bufsz);
  return 3;
}

}  // namespace spme
