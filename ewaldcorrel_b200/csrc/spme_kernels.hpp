// Launch interface between the host side of libsfac.so (sfac_capi.cu) and
// the sm_100a kernels.  Internal: not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "spme_common.cuh"

namespace spme {

// ---- sort (k_sort.cu) ----
struct SortBuffers {
  uint32_t *keys[2];   // ping-pong key buffers (cap)
  uint32_t *vals[2];   // ping-pong original indices (cap)
  float4 *rec;         // (frac0, frac1, frac2, charge) in input order (cap)
  float4 *rec_sorted;  // the same in cell order (cap)
  uint32_t *hist;      // radix histograms (sort_scratch_words(cap))
  int *cell_start;     // K0*K1*K2 + 1 offsets into the sorted order
  int cur;             // which keys/vals buffer holds the sorted result
};
size_t sort_scratch_words(int cap);
int launch_cell_sort(const Geom &g, int n, const double *x, const double *w, SortBuffers &b,
                      cudaStream_t st);

// ---- spread (k_spread.cu) ----
int launch_spread(const Geom &g, const Spline &S, const int *cell_start, const float4 *rec_sorted,
                   float *grid, cudaStream_t st);

// ---- FFT (k_fft.cu) ----
struct FftLen {
  int n, nst;
  int rad[32];
  const float2 *tw;  // n twiddles exp(-2 pi i k / n)
};
struct FftPlan3 {
  FftLen len[3];
};
struct DeconvArgs {
  const double *iB0, *iB1, *iB2;  // null: no moduli division
  int ldim;
};
int fft_make_len(FftLen &L, int n, float2 *tw_dev, cudaStream_t st);
int launch_fft_forward(const FftPlan3 &F, const float *real, float2 *cplx, const DeconvArgs &dc,
                        cudaStream_t st);
int launch_fft_inverse(const FftPlan3 &F, float2 *cplx, float *real, cudaStream_t st);

// ---- moduli, influence function, convolution (k_conv.cu) ----
// M_order(j), j = 0..order-1: the B-spline at the integer nodes (FP64).
struct SplineNodes {
  double Mj[kMaxOrder];
};
int launch_bspline_moduli(int n, int order, const SplineNodes &nodes, double *iB, cudaStream_t st);

// Influence function source for the convolution.
struct Influence {
  int mode;          // 1: FP64 tables A/dA from set_A; 2: Ewald evaluated on the device
  const double *A;   // mode 1: K0*K1*ldim
  const double *dA;  // mode 1: 6*K0*K1*ldim
  // mode 2: cell used for m = iL n (the cell current when the kernel was set)
  double iL00, iL10, iL11, iL20, iL21, iL22;
  double beta, max_m;
};
constexpr int kConvBlocks = 592;  // 4 x 148 SMs: fixed, so the reduction order is fixed
constexpr int kRedWords = 8;      // e, v00, v11, v22, v10, v20, v21, pad
// want_scale: 0 = energy only (en); 1 = energy + virial + FQ *= A iB (x2 planes) (de1).
int launch_conv(const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                 const double *iB2, float2 *S, int want_scale, double *partials, double *out,
                 cudaStream_t st);

// ---- gather (k_gather.cu) ----
int launch_gather(const Geom &g, const Spline &S, int n, const double *x, const double *w,
                   const float *grid, double *dx, double *phi, cudaStream_t st);

}  // namespace spme
