// Launch interface between the host side of libsfac.so (sfac_capi.cu) and
// the sm_100a kernels.  Internal: not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "spme_common.cuh"

namespace spme {

// Every device allocation of the library (handles and the serving runtime)
// goes through here, so that a test can make the n-th one fail
// (sfac_debug_fail_alloc) and check the error paths without a GPU fault.
cudaError_t device_malloc(void **p, size_t bytes);

// Index-checking build: each kernel module's error word, read and cleared
// (0 when no check failed, and always 0 in the product build).
unsigned long long check_take_sort();
unsigned long long check_take_spread();
unsigned long long check_take_gather();
unsigned long long check_take_fft();
unsigned long long check_take_serve();
unsigned long long check_take_capi();

// ---- sort (k_sort.cu) ----
struct SortBuffers {
  uint32_t *keys[2];   // [1]: cell key of every atom (input order); [0]: keys in cell order
  uint32_t *vals[2];   // [1]: arrival slot of every atom in its bucket; [0]: the stable permutation
  uint32_t *tkeys;     // keys in bucket-offset + arrival-slot order (cap)
  uint32_t *tmp;       // atom indices in the same order (cap)
  float4 *rec;         // (frac0, frac1, frac2, charge) in input order (cap)
  float4 *rec_sorted;  // the same in cell order (cap)
  uint32_t *hist;      // buckets too large for the in-place fix-up (cap)
  int *cell_start;     // cell_count_words(nb): nb + 1 bucket counts -> offsets, tile counts, control words
  int cur;             // which keys/vals buffer holds the sorted result (0)
};
// Buckets of the sort: runs of 2^zshift z cells of each (x, y) cell row.
// The spread's bucket: 32 z cells (its bricks are 32 points deep in z).
constexpr int kSpreadZShift = 5;
long sort_buckets(const Geom &g, int zshift);
size_t cell_count_words(long nbuckets);
int launch_cell_sort(const Geom &g, int n, const double *x, const double *w, SortBuffers &b, cudaStream_t st,
                     int zshift);

// ---- spread (k_spread.cu) ----
// cell_start: the bucket offsets of a launch_cell_sort with kSpreadZShift.
int launch_spread(const Geom &g, const Spline &S, const int *cell_start, const uint32_t *keys_sorted,
                  const float4 *rec_sorted, float *grid, cudaStream_t st);
void spread_prepare();  // sets the spread's shared-memory limit once (before any graph capture)

struct Influence;  // defined below (influence function source)

// ---- FFT (k_fft.cu) ----
struct FftLen {
  int n, nst;
  int rad[32];       // radix of each stage
  FastDiv ns[32];    // product of the earlier radices, per stage
  const float2 *tw;  // n twiddles exp(-2 pi i k / n)
};
struct FftPlan3 {
  FftLen len[3];
  int x_lines = 0;  // lines per CTA of the x pass (0: heuristic); set by the autotuner
  int zy_mode = 0;  // z/y passes: 0 automatic, 1 fused plane kernels, 2 two-level, 3 Stockham
};
struct DeconvArgs {
  const double *iB0, *iB1, *iB2;  // null: no moduli division
  int ldim;
};
int fft_make_len(FftLen &L, int n, float2 *tw_dev, cudaStream_t st);
void fft_prepare_kernels();  // sets shared-memory limits once (before any graph capture)
bool fft_plane_fits(int K1, int K2);
long fft_x_blocks_max(int K1, int K2);  // upper bound of x-pass CTAs (energy/virial partials)
// sfac path: forward 3D r2c and division by the moduli -> S.
int launch_fft_forward(const FftPlan3 &F, const Geom &g, const float *real, float2 *cplx, const DeconvArgs &dc,
                       cudaStream_t st);
// de1 path: S -> energy/virial (ev, raw sums) and the real potential grid.
int launch_conv_inverse(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0,
                        const double *iB1, const double *iB2, float2 *cplx, float *real, double *partials,
                        double *raw, double *ev, cudaStream_t st);
// de1's first half: x pass with the convolution, and the energy/virial sums
// in raw (the same sums, in the same order, as launch_conv_inverse forms);
// the caller enqueues inv_yz (without partials) afterwards.
int launch_conv_energy(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                       const double *iB2, float2 *cplx, double *partials, double *raw, cudaStream_t st);
// en path: energy/virial sums of S (raw), same order as launch_conv_inverse.
int launch_energy(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                  const double *iB2, float2 *cplx, double *partials, double *raw, cudaStream_t st);
// The three launches of the fused solve, also callable one by one:
// forward z/y; x forward + convolution + x inverse; inverse y/z (+ reduction).
int fwd_zy(const FftPlan3 &F, const float *real, float2 *cplx, cudaStream_t st);
int launch_x_conv(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                  const double *iB2, float2 *cplx, double *partials, int &nblocks, cudaStream_t st);
int inv_yz(const FftPlan3 &F, float2 *cplx, float *real, const double *partials, int nblocks,
           const CellConst *cell, double *raw, double *ev, cudaStream_t st);
// fused solve: spread grid -> energy/virial and potential grid.
int launch_fft_conv_solve(const FftPlan3 &F, const Geom &g, const Influence &inf, const double *iB0,
                          const double *iB1, const double *iB2, const float *real_in, float2 *cplx,
                          float *real_out, double *partials, double *raw, double *ev, cudaStream_t st);

// ---- moduli, influence function, convolution (k_conv.cu) ----
// M_order(j), j = 0..order-1: the B-spline at the integer nodes (FP64).
struct SplineNodes {
  double Mj[kMaxOrder];
};
int launch_bspline_moduli(int n, int order, const SplineNodes &nodes, double *iB, cudaStream_t st);

// Reciprocal-lattice images of one (kx, ky) row of stored modes: the
// (i, j) lattice pairs with i = kx mod K0, j = ky mod K1 inside the cutoff
// sphere, with their x/y components and the z index bounds [k0, k1] of the
// sphere (set_A's loop bounds, sfac.cpp:240-262).  count < 0: more pairs
// than fit; the row is then enumerated in full at each use.
constexpr int kRowPairs = 4;
struct RowImg {
  int count;
  int k0[kRowPairs], k1[kRowPairs];
  int pad;
  double mx[kRowPairs], my[kRowPairs], m21[kRowPairs], mz0[kRowPairs];
};

// Constants of the device Ewald influence function (device memory): the
// cell used for m = iL n (the one current when the function was set; later
// box changes do not touch it, as with set_A), the Ewald parameters and the
// exponent factor fac = -(pi / beta)^2.
struct InfConst {
  double iL00, iL10, iL11, iL20, iL21, iL22, beta, max_m, fac;
};

// Influence function source for the convolution.
// Mode 4 is mode 2 with a compact per-mode table (one double per mode: A
// with the lattice shift of the mode's single image inside the cutoff sphere
// in its lowest mantissa bits, 0 for no image, -1 for several), from which
// dA follows without evaluating f again; modes with several images use mode
// 2's row tables.
struct Influence {
  int mode;                // 1: FP64 tables A/dA; 2: Ewald on the device; 4: mode 2 + compact table
  const double *A;         // mode 1: K0*K1*ldim tables; mode 4: the packed compact table
  const double *dA;        // mode 1: 6*K0*K1*ldim
  const InfConst *ic;      // mode 2, 4: device constants
  const RowImg *rows;      // mode 2, 4: K0*K1 row image tables (rebuilt when the function is set)
  FastDiv K2d;             // division by K2
};
// Builds the row image tables of an Ewald influence function (mode 2).
int launch_ewald_rows(const Geom &g, const Influence &inf, RowImg *rows, cudaStream_t st);
// Tabulates a mode-2 influence function as FP64 tables A (nmodes) and dA
// (6 per mode), the layout of mode 1.
int launch_ewald_table(const Geom &g, const Influence &inf, double *A, double *dA, cudaStream_t st);
// Compact table of a mode-2 Ewald influence function (mode 4), packed per mode.
int launch_ewald_compact(const Geom &g, const Influence &inf, double *A, cudaStream_t st);
// Tables A / dA (mode 1 layout) of a caller-sampled radial function f, f'
// at m^2 = k dm2 (k < nt), over set_A's image set within ic.max_m.
int launch_radial_table(const Geom &g, const InfConst &ic, const double *f, const double *df, int nt, double dm2,
                        double *A, double *dA, cudaStream_t st);
constexpr int kConvBlocks = 592;  // 4 x 148 SMs: fixed, so the reduction order is fixed
constexpr int kRedWords = 8;      // e, v00, v11, v22, v10, v20, v21, pad
// Energy/virial sums over S without modifying it (en): raw sums -> out,
// and ev (may be null).  want_scale = 1 also applies the de1 scaling in place.
int launch_conv(const Geom &g, const Influence &inf, const double *iB0, const double *iB1,
                const double *iB2, float2 *S, int want_scale, double *partials, double *out, double *ev,
                cudaStream_t st);
// Sum of per-CTA partials -> raw (7) and ev (7), one small kernel.
int launch_finish(const double *partials, int nblocks, const CellConst *cell, double *raw, double *ev,
                  cudaStream_t st);

// ---- gather (k_gather.cu) ----
// perm/keys/rec (optional): the cell-sorted view of the same points (from
// launch_cell_sort) -- points are then gathered in cell order.
int launch_gather(const Geom &g, const Spline &S, int n, const double *x, const double *w,
                  const float *grid, double *dx, double *phi, cudaStream_t st, const uint32_t *perm = nullptr,
                  const uint32_t *keys = nullptr, const float4 *rec = nullptr);
// Gather + cell adjoint: dE/dL (6 doubles, device) from dE/dx, the virial in ev
// and the positions; cellp is scratch of gather_cell_words(n) doubles.
int launch_gather_cell(const Geom &g, const Spline &S, int n, const double *x, const double *w,
                       const float *grid, double *dx, double *phi, double *cellp, const double *ev, double *dEdL,
                       cudaStream_t st, const uint32_t *perm = nullptr, const uint32_t *keys = nullptr,
                       const float4 *rec = nullptr);
size_t gather_cell_words(int cap);

// ---- structure-factor analysis (k_sk.cu) ----
int launch_sk_accumulate(long nmodes, const float2 *S, double *acc, cudaStream_t st);
size_t sk_partial_words();
int launch_sk_radial(const Geom &g, const double *acc, int nbins, double dk, double *partials, double *sums,
                     double *counts, cudaStream_t st);

// cross-correlations of D densities: slot i <- S; C_k += Q_i conj(Q_j), i <= j
int launch_xc_store(long nmodes, const float2 *S, float2 *slot, cudaStream_t st);
int launch_xc_accumulate(long nmodes, int D, const float2 *Q, double2 *C, cudaStream_t st);

// ---- real-space term (k_real.cu) ----
// Coarse cells of the real-space cell list are at least rcut / kRealSub wide;
// the pair kernel searches kRealSub cells either side.
constexpr int kRealSub = 2;
// Intervals of the erfcx table of the pair kernel (float4 each).
constexpr int kRealTab = 256;
// Cell sort of the points on the coarse grid `coarse` (cells >= rcut wide),
// then the minimum-image erfc pair sum: dx (n x 3, input order, may be null)
// and out (device, 10 doubles: E_real, E_self, E_net, virial[6], net-charge
// virial diagonal).  partials: real_partial_words(n) doubles; tab: kRealTab
// float4.
int launch_real_space(const Geom &coarse, const double L[6], int n, const double *x, const double *w, float eta,
                      float rcut, SortBuffers &sb, double4 *rec, float4 *tab, double *dx, double *partials,
                      double eta_d, double *out, cudaStream_t st);
size_t real_partial_words(int cap);

}  // namespace spme
