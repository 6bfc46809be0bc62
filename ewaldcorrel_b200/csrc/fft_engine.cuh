// Shared-memory Stockham FFT engine (FP32) used by the FFT pass kernels.
//
// Data of B lines of length n live in shared memory as [j][b] with pitch P
// (element j of line b at j*P + b).  Each stage of radix R reads R inputs at
// stride n/R, applies twiddles exp(SIGN 2 pi i r (j mod Ns) / (Ns R)), runs an
// R-point DFT and writes the outputs in autosort order (Stockham), so the
// result is in natural order without bit reversal.  Radix 2, 3, 4, 5 and 7
// butterflies are written out; any other prime uses a direct DFT.
#pragma once

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

// One Stockham stage over B lines: in/out are [j][b] with pitch P.  Bd and
// Nd divide by B and by Ns (the product of the earlier radices) without
// hardware integer division.
template <int R, int SIGN>
__device__ __forceinline__ void stage(const float2 *in, float2 *out, const float2 *tw, int n, const FastDiv &Nd,
                                      const FastDiv &Bd, int P) {
  const int m = n / R;
  const int Ns = (int)Nd.d;
  const int twstep = n / (Ns * R);
  const int items = m * (int)Bd.d;
  for (int item = threadIdx.x; item < items; item += blockDim.x) {
    uint32_t j, b, q, k;
    Bd.divmod((uint32_t)item, j, b);
    Nd.divmod(j, q, k);
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      v[r] = in[(j + r * m) * P + b];
      if (r > 0) v[r] = cmul(v[r], twid<SIGN>(tw, r * (int)k * twstep));
    }
    Bfly<R, SIGN>::run(v, tw, n);
    const int idxD = (int)(q * Ns * R + k);
#pragma unroll
    for (int r = 0; r < R; r++) out[(idxD + r * Ns) * P + b] = v[r];
  }
}

// Radices outside the compiled set: the same stage, reading the inputs
// straight from shared memory (O(R^2) per butterfly, any R).
template <int SIGN>
__device__ void stage_any(const float2 *in, float2 *out, const float2 *tw, int n, int R, const FastDiv &Nd,
                          const FastDiv &Bd, int P) {
  const int m = n / R;
  const int Ns = (int)Nd.d;
  const int B = (int)Bd.d;
  const int twstep = n / (Ns * R);
  const int step = n / R;
  for (int item = threadIdx.x; item < m * B * R; item += blockDim.x) {
    const int qo = item % R;
    const int rest = item / R;
    const int b = rest % B, j = rest / B;
    const int k = j % Ns;
    float2 acc = make_float2(0.f, 0.f);
    for (int r = 0; r < R; r++) {
      float2 x = in[(j + r * m) * P + b];
      x = cmul(x, twid<SIGN>(tw, r * k * twstep));
      acc = cadd(acc, cmul(x, twid<SIGN>(tw, ((r * qo) % R) * step)));
    }
    const int idxD = (j / Ns) * Ns * R + k;
    out[(idxD + qo * Ns) * P + b] = acc;
  }
}

// Runs all stages; returns the buffer holding the result.
template <int SIGN>
__device__ float2 *run_stages(const FftLen &L, float2 *b0, float2 *b1, const float2 *tw, const FastDiv &Bd, int P) {
  for (int s = 0; s < L.nst; s++) {
    const int R = L.rad[s];
    const FastDiv &Nd = L.ns[s];
    switch (R) {
      case 2: stage<2, SIGN>(b0, b1, tw, L.n, Nd, Bd, P); break;
      case 3: stage<3, SIGN>(b0, b1, tw, L.n, Nd, Bd, P); break;
      case 4: stage<4, SIGN>(b0, b1, tw, L.n, Nd, Bd, P); break;
      case 5: stage<5, SIGN>(b0, b1, tw, L.n, Nd, Bd, P); break;
      case 7: stage<7, SIGN>(b0, b1, tw, L.n, Nd, Bd, P); break;
      default: stage_any<SIGN>(b0, b1, tw, L.n, R, Nd, Bd, P); break;
    }
    __syncthreads();
    float2 *t = b0;
    b0 = b1;
    b1 = t;
  }
  return b0;
}

// ---- warp-synchronous variant --------------------------------------------
// One warp transforms the lines (columns) [c0, c0 + nc) of the shared
// [j][b] arrays on its own: items are spread over its lanes, stages are
// separated by __syncwarp only.  Bwd divides by the warp's column capacity
// (>= nc); warps own disjoint columns, so they never wait on one another.
template <int R, int SIGN>
__device__ __forceinline__ void stage_w(const float2 *in, float2 *out, const float2 *tw, int n, const FastDiv &Nd,
                                        const FastDiv &Bwd, int P, int c0, int nc, int lane) {
  const int m = n / R;
  const int Ns = (int)Nd.d;
  const int twstep = n / (Ns * R);
  const int items = m * (int)Bwd.d;
  for (int item = lane; item < items; item += 32) {
    uint32_t j, bl, q, k;
    Bwd.divmod((uint32_t)item, j, bl);
    if ((int)bl >= nc) continue;
    const int b = c0 + (int)bl;
    Nd.divmod(j, q, k);
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      v[r] = in[(j + r * m) * P + b];
      if (r > 0) v[r] = cmul(v[r], twid<SIGN>(tw, r * (int)k * twstep));
    }
    Bfly<R, SIGN>::run(v, tw, n);
    const int idxD = (int)(q * Ns * R + k);
#pragma unroll
    for (int r = 0; r < R; r++) out[(idxD + r * Ns) * P + b] = v[r];
  }
}

template <int SIGN>
__device__ void stage_any_w(const float2 *in, float2 *out, const float2 *tw, int n, int R, const FastDiv &Nd, int Bw,
                            int P, int c0, int nc, int lane) {
  const int m = n / R;
  const int Ns = (int)Nd.d;
  const int twstep = n / (Ns * R);
  const int step = n / R;
  for (int item = lane; item < m * Bw * R; item += 32) {
    const int qo = item % R;
    const int rest = item / R;
    const int bl = rest % Bw, j = rest / Bw;
    if (bl >= nc) continue;
    const int b = c0 + bl;
    const int k = j % Ns;
    float2 acc = make_float2(0.f, 0.f);
    for (int r = 0; r < R; r++) {
      float2 x = in[(j + r * m) * P + b];
      x = cmul(x, twid<SIGN>(tw, r * k * twstep));
      acc = cadd(acc, cmul(x, twid<SIGN>(tw, ((r * qo) % R) * step)));
    }
    const int idxD = (j / Ns) * Ns * R + k;
    out[(idxD + qo * Ns) * P + b] = acc;
  }
}

// All stages for one warp's columns; returns the buffer holding the result
// (the same for every warp: it depends only on the stage count).
template <int SIGN>
__device__ float2 *run_stages_w(const FftLen &L, float2 *b0, float2 *b1, const float2 *tw, const FastDiv &Bwd, int P,
                                int c0, int nc, int lane) {
  for (int s = 0; s < L.nst; s++) {
    const int R = L.rad[s];
    const FastDiv &Nd = L.ns[s];
    switch (R) {
      case 2: stage_w<2, SIGN>(b0, b1, tw, L.n, Nd, Bwd, P, c0, nc, lane); break;
      case 3: stage_w<3, SIGN>(b0, b1, tw, L.n, Nd, Bwd, P, c0, nc, lane); break;
      case 4: stage_w<4, SIGN>(b0, b1, tw, L.n, Nd, Bwd, P, c0, nc, lane); break;
      case 5: stage_w<5, SIGN>(b0, b1, tw, L.n, Nd, Bwd, P, c0, nc, lane); break;
      case 7: stage_w<7, SIGN>(b0, b1, tw, L.n, Nd, Bwd, P, c0, nc, lane); break;
      default: stage_any_w<SIGN>(b0, b1, tw, L.n, R, Nd, (int)Bwd.d, P, c0, nc, lane); break;
    }
    __syncwarp();
    float2 *t = b0;
    b0 = b1;
    b1 = t;
  }
  return b0;
}

__device__ __forceinline__ void load_twiddles(float2 *tw_s, const FftLen &L) {
  for (int i = threadIdx.x; i < L.n; i += blockDim.x) tw_s[i] = L.tw[i];
}

}  // namespace spme
