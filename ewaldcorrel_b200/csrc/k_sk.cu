// Structure-factor analysis: <|S(m)|^2> over frames and its radial binning,
// the reference's original use of the library (run.py:27-47 accumulates
// |get_S()|^2 over frames; plot.py:9-32 bins it by |k|).
//
// Accumulation is element-wise over the stored half-space modes (FP64, one
// writer per mode).  Radial binning is deterministic without floating-point
// atomics: each warp walks a fixed contiguous run of modes 32 at a time and
// its lane 0 adds the 32 (bin, value) pairs to the warp's own shared-memory
// histogram in lane order; the CTA sums its warps' histograms in warp order
// into per-block partials, which one last kernel sums over blocks in order.
#include "reduce.cuh"
#include "spme_kernels.hpp"

namespace spme {

constexpr int kSkWarps = 4;
constexpr int kSkBins = 1024;  // bins per binning pass (shared memory: warps x bins x (sum, count))
constexpr int kSkBlocks = 296;

__global__ void __launch_bounds__(256) sk_accumulate_kernel(long nmodes, const float2 *__restrict__ S,
                                                            double *__restrict__ acc) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nmodes; i += (long)gridDim.x * blockDim.x) {
    const float2 s = S[i];
    acc[i] += (double)s.x * s.x + (double)s.y * s.y;
  }
}

// Bin of stored mode i: |k| = 2 pi |m|, m the reciprocal-lattice vector of
// the signed frequency indices n (m . x = n . s: m_x = n0 iL00,
// m_y = n0 iL10 + n1 iL11, m_z = n0 iL20 + n1 iL21 + n2 iL22, as set_A forms
// it, sfac.cpp:240-262; x, y aliased to (-K/2, K/2], z the stored half-space
// index 0..ldim-1); bins [b0, b0 + nb) of width dk.  -1 when outside.
__device__ __forceinline__ int sk_bin(const Geom &g, const CellConst &c, long i, double dk, int b0, int nb) {
  const int kz = (int)(i % g.ldim);
  const long r = i / g.ldim;
  const int ky = (int)(r % g.K1), kx = (int)(r / g.K1);
  const double n0 = (kx > g.K0 / 2) ? kx - g.K0 : kx;
  const double n1 = (ky > g.K1 / 2) ? ky - g.K1 : ky;
  const double n2 = kz;
  const double m0 = n0 * c.iL00;
  const double m1 = n0 * c.iL10 + n1 * c.iL11;
  const double m2 = n0 * c.iL20 + n1 * c.iL21 + n2 * c.iL22;
  const double k = 2.0 * 3.14159265358979323846 * sqrt(m0 * m0 + m1 * m1 + m2 * m2);
  const double b = floor(k / dk) - b0;
  return (b >= 0.0 && b < (double)nb) ? (int)b : -1;
}

// partials[block][2 * nb]: sums then counts of bins [b0, b0 + nb).
__global__ void __launch_bounds__(kSkWarps * 32) sk_radial_kernel(Geom g, const double *__restrict__ acc, double dk,
                                                                  int b0, int nb, double *__restrict__ partials) {
  __shared__ double hs[kSkWarps][kSkBins];
  __shared__ float hc[kSkWarps][kSkBins];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int b = threadIdx.x; b < kSkWarps * kSkBins; b += blockDim.x) {
    (&hs[0][0])[b] = 0.0;
    (&hc[0][0])[b] = 0.f;
  }
  __syncthreads();
  const CellConst c = *g.cell;
  const long nmodes = (long)g.K0 * g.K1 * g.ldim;
  const long nw = (long)gridDim.x * kSkWarps, wid = (long)blockIdx.x * kSkWarps + warp;
  const long lo = nmodes * wid / nw, hi = nmodes * (wid + 1) / nw;  // this warp's contiguous run
  for (long base = lo; base < hi; base += 32) {
    const long i = base + lane;
    int bin = -1;
    double v = 0.0;
    if (i < hi) {
      bin = sk_bin(g, c, i, dk, b0, nb);
      v = acc[i];
    }
    for (int k = 0; k < 32; k++) {
      const int bk = __shfl_sync(0xffffffffu, bin, k);
      const double vk = __shfl_sync(0xffffffffu, v, k);
      if (lane == 0 && bk >= 0) {
        hs[warp][bk] += vk;
        hc[warp][bk] += 1.f;
      }
    }
  }
  __syncthreads();
  double *out = partials + (long)blockIdx.x * 2 * nb;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    double s = 0.0, n = 0.0;
#pragma unroll
    for (int w = 0; w < kSkWarps; w++) {
      s += hs[w][b];
      n += (double)hc[w][b];
    }
    out[b] = s;
    out[nb + b] = n;
  }
}

__global__ void sk_radial_finish_kernel(const double *__restrict__ partials, int nblocks, int nb,
                                        double *__restrict__ sums, double *__restrict__ counts) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  double s = 0.0, n = 0.0;
  for (int k = 0; k < nblocks; k++) {
    s += partials[(long)k * 2 * nb + b];
    n += partials[(long)k * 2 * nb + nb + b];
  }
  sums[b] = s;
  counts[b] = n;
}

int launch_sk_accumulate(long nmodes, const float2 *S, double *acc, cudaStream_t st) {
  sk_accumulate_kernel<<<4 * 148, 256, 0, st>>>(nmodes, S, acc);
  return 1;
}

size_t sk_partial_words() { return (size_t)kSkBlocks * 2 * kSkBins; }

// Radial sums and counts of nbins bins of width dk (device arrays), in passes
// of kSkBins bins.
int launch_sk_radial(const Geom &g, const double *acc, int nbins, double dk, double *partials, double *sums,
                     double *counts, cudaStream_t st) {
  int k = 0;
  for (int b0 = 0; b0 < nbins; b0 += kSkBins) {
    const int nb = (nbins - b0 < kSkBins) ? nbins - b0 : kSkBins;
    sk_radial_kernel<<<kSkBlocks, kSkWarps * 32, 0, st>>>(g, acc, dk, b0, nb, partials);
    sk_radial_finish_kernel<<<(nb + 127) / 128, 128, 0, st>>>(partials, kSkBlocks, nb, sums + b0, counts + b0);
    k += 2;
  }
  return k;
}

}  // namespace spme

namespace spme {

// ---------------------------------------------------------------------------
// Cross-correlations of several densities (gmx_ewald.py:76-95): after each
// density's sfac, its structure factor is kept in slot i (FP32 complex);
// once all D slots of a frame are filled, C_k += Q_i conj(Q_j) for every
// pair i <= j (k in row order: (0,0), (0,1), ..., (1,1), ...), FP64 complex,
// one writer per (pair, mode).
__global__ void __launch_bounds__(256) xc_store_kernel(long nmodes, const float2 *__restrict__ S,
                                                       float2 *__restrict__ slot) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nmodes; i += (long)gridDim.x * blockDim.x)
    slot[i] = S[i];
}

__global__ void __launch_bounds__(256) xc_accumulate_kernel(long nmodes, int D, const float2 *__restrict__ Q,
                                                            double2 *__restrict__ C) {
  for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < nmodes; m += (long)gridDim.x * blockDim.x) {
    int k = 0;
    for (int i = 0; i < D; i++) {
      const float2 a = Q[(long)i * nmodes + m];
      for (int j = i; j < D; j++, k++) {
        const float2 b = Q[(long)j * nmodes + m];
        double2 c = C[(long)k * nmodes + m];
        // a * conj(b)
        c.x += (double)a.x * b.x + (double)a.y * b.y;
        c.y += (double)a.y * b.x - (double)a.x * b.y;
        C[(long)k * nmodes + m] = c;
      }
    }
  }
}

int launch_xc_store(long nmodes, const float2 *S, float2 *slot, cudaStream_t st) {
  xc_store_kernel<<<4 * 148, 256, 0, st>>>(nmodes, S, slot);
  return 1;
}

int launch_xc_accumulate(long nmodes, int D, const float2 *Q, double2 *C, cudaStream_t st) {
  xc_accumulate_kernel<<<4 * 148, 256, 0, st>>>(nmodes, D, Q, C);
  return 1;
}

}  // namespace spme
