// K1: integer cell keys and the stable cell sort (SFac::sort, sfac.cpp:92-111).
//
// The reference inserts every atom into a std::multimap keyed by
// cid = (n0*K1 + n1)*K2 + n2; equal keys keep insertion order, so the result
// is the STABLE sort of atoms by cid.  Two sorts produce that order here:
//   - the main path (launch_cell_sort, below) is a counting sort over
//     buckets of cells (runs of z cells of one cell row), which also yields
//     the per-bucket offsets the spread and the real-space walk need;
//   - the allocation-free entry point (end of file) is an LSD radix sort
//     whose scratch is bounded by the atom count:
//       1. key_hist_kernel: FP64 cell keys (rounding identical to the host,
//          so boundary atoms land in the same cell), in-cell fractions, and
//          the per-tile histogram of the first 8-bit digit;
//       2. per digit: hist_scan_kernel (exclusive scan of that digit's tile
//          histograms), then radix_scatter_kernel, which ranks ties in input
//          order (stable by construction, so bit-exact against the CPU sort)
//          and counts the NEXT digit of every key at the tile it lands in.
// Integer counts only (their sums do not depend on order).
#include <cstdio>
#include <mutex>

#include "../../include/sfac.h"
#include "spme_kernels.hpp"

namespace spme {

SPME_CHECK_READER(sort)

constexpr int RS_THREADS = 128;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 1024 keys per tile
constexpr int RS_BINS = 256;
constexpr int RS_MAX_PASSES = 4;

// Cell index and in-cell fraction exactly as SFac::sort computes them
// (sfac.cpp:98-106): u = s*K, n = (int)u, u -= n.  A coordinate that wrapped
// to exactly 1.0 (Cell::wrap of a tiny negative number) is mapped to its
// periodic image 0 instead of forming the out-of-range key K.
__device__ __forceinline__ uint32_t cell_key(const Geom &g, const CellConst &c, double x0, double x1, double x2,
                                             float4 &r, float w) {
  double s0, s1, s2;
  frac_coords(c, x0, x1, x2, s0, s1, s2);
  const double u0 = __dmul_rn(s0, (double)g.K0), u1 = __dmul_rn(s1, (double)g.K1),
               u2 = __dmul_rn(s2, (double)g.K2);
  int n0 = __double2int_rz(u0), n1 = __double2int_rz(u1), n2 = __double2int_rz(u2);
  double f0 = __dsub_rn(u0, (double)n0), f1 = __dsub_rn(u1, (double)n1), f2 = __dsub_rn(u2, (double)n2);
  if (n0 >= g.K0) { n0 = 0; f0 = 0.0; }
  if (n1 >= g.K1) { n1 = 0; f1 = 0.0; }
  if (n2 >= g.K2) { n2 = 0; f2 = 0.0; }
  r = make_float4((float)f0, (float)f1, (float)f2, w);
  return (uint32_t)((n0 * g.K1 + n1) * g.K2 + n2);
}

// Keys, records and the first digit's per-tile histogram.  Histograms are
// stored pass-major then digit-major: hist[(p * 256 + d) * ntiles + tile];
// the later passes' columns of this tile are zeroed here and filled by the
// preceding scatter pass.
// totals[p][d] (zeroed beforehand) receives the global count of digit d of
// pass p: a permutation-invariant sum, so every pass's digit bases are known
// after this kernel.
__global__ void __launch_bounds__(RS_THREADS) key_hist_kernel(Geom g, int n, const double *__restrict__ x,
                                                              const double *__restrict__ w,
                                                              uint32_t *__restrict__ keys,
                                                              float4 *__restrict__ rec,
                                                              uint32_t *__restrict__ hist, int ntiles,
                                                              int npass, uint32_t *__restrict__ totals) {
  __shared__ uint32_t h[RS_MAX_PASSES][RS_BINS];
  for (int i = threadIdx.x; i < RS_MAX_PASSES * RS_BINS; i += RS_THREADS) (&h[0][0])[i] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE;
  const CellConst cc = *g.cell;
#pragma unroll 2
  for (int it = 0; it < RS_ITEMS; it++) {
    const int a = base + it * RS_THREADS + threadIdx.x;
    if (a < n) {
      float4 r;
      const uint32_t key = cell_key(g, cc, x[3 * a], x[3 * a + 1], x[3 * a + 2], r, (float)w[a]);
      keys[a] = key;
      rec[a] = r;
      for (int p = 0; p < npass; p++) atomicAdd(&h[p][(key >> (8 * p)) & 0xff], 1u);
    }
  }
  __syncthreads();
  for (int d = threadIdx.x; d < RS_BINS; d += RS_THREADS) {
    hist[d * ntiles + blockIdx.x] = h[0][d];
    for (int p = 1; p < npass; p++) hist[(p * RS_BINS + d) * ntiles + blockIdx.x] = 0u;
    for (int p = 0; p < npass; p++)
      if (h[p][d]) atomicAdd(&totals[p * RS_BINS + d], h[p][d]);
  }
}

// In place, one block per digit d of one pass:
//   offsets[d][tile] = sum_{d'<d} totals[d'] + sum_{t<tile} hist[d][t].
__global__ void __launch_bounds__(256) hist_scan_kernel(uint32_t *__restrict__ hist, int ntiles,
                                                        const uint32_t *__restrict__ totals) {
  __shared__ uint32_t wsum[8];
  __shared__ uint32_t base_s;
  const int d = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (warp == 0) {  // base = sum of the totals of smaller digits
    uint32_t v = 0;
    for (int e = lane; e < d; e += 32) v += totals[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) base_s = v;
  }
  __syncthreads();
  uint32_t run = base_s;
  uint32_t *row = hist + (size_t)d * ntiles;
  for (int t0 = 0; t0 < ntiles; t0 += 256) {
    const int t = t0 + threadIdx.x;
    const uint32_t v = (t < ntiles) ? row[t] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0, blk = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const uint32_t ws = wsum[k];
      if (k < warp) wpre += ws;
      blk += ws;
    }
    if (t < ntiles) row[t] = run + wpre + incl - v;
    run += blk;
    __syncthreads();
  }
}

// Stable scatter of one 8-bit digit.  Each warp owns a contiguous run of
// 32*RS_ITEMS keys of the tile and walks it in memory order; ties inside a
// round of 32 are ranked by lane, ties across rounds and warps by a running
// per-warp digit count, ties across tiles by the scanned histogram.
// vin == nullptr: values are the input positions (first pass).  With
// hist_next != nullptr the next digit (shift + 8) of every key is counted at
// the output tile it lands in.  With rec_sorted != nullptr (last pass) the
// atom record of each key is gathered to its sorted position too.
__global__ void __launch_bounds__(RS_THREADS) radix_scatter_kernel(
    const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint32_t *__restrict__ kout,
    uint32_t *__restrict__ vout, int n, int shift, const uint32_t *__restrict__ offs, int ntiles,
    uint32_t *__restrict__ hist_next, const float4 *__restrict__ rec, float4 *__restrict__ rec_sorted) {
  __shared__ uint32_t whist[RS_WARPS][RS_BINS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < RS_WARPS * RS_BINS; i += RS_THREADS) (&whist[0][0])[i] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE + warp * (32 * RS_ITEMS);
  const uint32_t lt_mask = (1u << lane) - 1u;
  uint32_t key[RS_ITEMS], val[RS_ITEMS], rank[RS_ITEMS];
#pragma unroll
  for (int it = 0; it < RS_ITEMS; it++) {
    const int i = base + it * 32 + lane;
    const bool valid = i < n;
    key[it] = valid ? kin[i] : 0u;
    val[it] = valid ? (vin ? vin[i] : (uint32_t)i) : 0u;
    const uint32_t d = valid ? ((key[it] >> shift) & 0xff) : RS_BINS;  // sentinel group
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t prev = 0;
    if (lane == leader && valid) {
      prev = whist[warp][d];
      whist[warp][d] = prev + __popc(peers);
    }
    prev = __shfl_sync(0xffffffffu, prev, leader);
    rank[it] = prev + __popc(peers & lt_mask);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < RS_BINS; d += RS_THREADS) {  // exclusive prefix over warps
    uint32_t run = offs[d * ntiles + blockIdx.x];
#pragma unroll
    for (int wp = 0; wp < RS_WARPS; wp++) {
      const uint32_t c = whist[wp][d];
      whist[wp][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < RS_ITEMS; it++) {
    const int i = base + it * 32 + lane;
    if (i < n) {
      const uint32_t d = (key[it] >> shift) & 0xff;
      const uint32_t pos = whist[warp][d] + rank[it];
      kout[pos] = key[it];
      vout[pos] = val[it];
      if (hist_next) atomicAdd(&hist_next[((key[it] >> (shift + 8)) & 0xff) * ntiles + pos / RS_TILE], 1u);
      if (rec_sorted) rec_sorted[pos] = rec[val[it]];
    }
  }
}

static int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

static int key_passes(long ncell) {
  int bits = 1;
  while (bits < 32 && ((ncell - 1) >> bits) > 0) bits++;
  return (bits + 7) / 8;
}

// ---------------------------------------------------------------------------
// Main-path cell sort: a counting sort over buckets of cells.
//
// A bucket is a run of 2^zshift consecutive z cells of one (x, y) cell row:
// bucket = (n0 K1 + n1) nzb + (n2 >> zshift), nzb = ceil(K2 / 2^zshift), so
// buckets are ordered like the keys they hold.  zshift = 0 gives one bucket
// per cell (the real-space cell list needs per-cell offsets); the spread
// takes runs of 32 cells, which keeps the count array at K0 K1 K2 / 32 words
// (2 MB at 256^3 instead of 67 MB), resident in L2.
//
//   1. key_count_kernel: keys and records (as above); every atom takes an
//      arrival slot in its bucket with an integer atomic (count[bucket]++).
//   2. tile_sum_kernel + cell_offsets_kernel: exclusive scan of the
//      per-bucket counts, in place, into cell_start (cell_start[nb] = n):
//      the sum of every tile of 2^tshift buckets, then each tile scans its
//      buckets from the sum of the tiles before it (at most ~2048 tiles).
//   3. cell_scatter_kernel: every atom goes to cell_start[bucket] + its
//      arrival slot, with its key; an atom alone in its bucket is final.
//   4. cell_fixup_kernel: the atoms of each shared bucket are put in
//      (key, input index) order -- rank = number of the bucket's atoms with a
//      smaller (key, index) pair -- which is exactly the stable order of the
//      reference's multimap.  Buckets with more than kBigCell atoms are
//      listed and merge-sorted by the last CTA to finish (no waiting on other
//      CTAs).
// Only integer atomics (counts) are used; the result is the same bits on
// every run.

constexpr int kBigCell = 256;
constexpr int kScanThreads = 512;
constexpr int kScanItems = 16;
constexpr int kScanChunk = kScanThreads * kScanItems;  // buckets per CTA pass

static int cell_tile_shift(long ncell) {
  int s = 13;  // log2(kScanChunk)
  while (((ncell + 1 + (1L << s) - 1) >> s) > 2048) s++;
  return s;
}
static long cell_tiles(long ncell) {
  const int s = cell_tile_shift(ncell);
  return (ncell + 1 + (1L << s) - 1) >> s;
}

long sort_buckets(const Geom &g, int zshift) {
  const long nzb = ((long)g.K2 + (1L << zshift) - 1) >> zshift;
  return (long)g.K0 * g.K1 * nzb;
}

// Word layout of the bucket-count region (everything before the tile sums is
// zeroed before every sort):
//   [0, nb + 1)            counts, then offsets
//   [nb + 1, nb + 3)       control: large buckets, finished fix-up CTAs
//   [nb + 3, 2 nb + 3)     head: atoms of each bucket in its first H - 1 cells
//   [2 nb + 3, 3 nb + 3)   tail: atoms of each bucket in its last H cells
//   [3 nb + 3, + T)        tile sums
// (head and tail: the spread's halo of an interior brick starts H cells
// before a bucket boundary and ends H - 1 cells after one, H = order / 2.)
size_t cell_count_words(long nb) { return (size_t)(3 * nb + 3 + cell_tiles(nb)); }

// Bucket of a cell key (see above).
struct BucketMap {
  FastDiv K2d;
  uint32_t nzb, zshift;
  uint32_t nb;  // buckets (for the index-checking build)
  __device__ __forceinline__ uint32_t operator()(uint32_t key) const {
    uint32_t row, n2;
    K2d.divmod(key, row, n2);
    return row * nzb + (n2 >> zshift);
  }
};

static BucketMap bucket_map(const Geom &g, int zshift) {
  BucketMap m;
  m.K2d = FastDiv((uint32_t)g.K2);
  m.nzb = (uint32_t)(((long)g.K2 + (1L << zshift) - 1) >> zshift);
  m.zshift = (uint32_t)zshift;
  m.nb = (uint32_t)sort_buckets(g, zshift);
  return m;
}

// head/tail (may be null): see the word layout above; ht_h = H.
__global__ void __launch_bounds__(256) key_count_kernel(Geom g, int n, const double *__restrict__ x,
                                                        const double *__restrict__ w, uint32_t *__restrict__ keys,
                                                        uint32_t *__restrict__ slot, float4 *__restrict__ rec,
                                                        uint32_t *__restrict__ count, BucketMap bm,
                                                        uint32_t *__restrict__ head, uint32_t *__restrict__ tail,
                                                        int ht_h) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const CellConst cc = *g.cell;
  float4 r;
  const uint32_t key = cell_key(g, cc, x[3 * a], x[3 * a + 1], x[3 * a + 2], r, (float)w[a]);
  keys[a] = key;
  rec[a] = r;
  uint32_t row, n2;
  bm.K2d.divmod(key, row, n2);
  const uint32_t b = row * bm.nzb + (n2 >> bm.zshift);
  if (!SPME_IN(b, bm.nb, CK_SORT_BUCKET)) return;
  slot[a] = atomicAdd(&count[b], 1u);
  if (head) {
    const int off = (int)(n2 & ((1u << bm.zshift) - 1u));
    if (off < ht_h - 1) atomicAdd(&head[b], 1u);
    if (off >= (1 << bm.zshift) - ht_h) atomicAdd(&tail[b], 1u);
  }
}

// Block-wide sum (every thread gets the result); red: one word per warp.
template <int NT>
__device__ __forceinline__ uint32_t block_sum_u32(uint32_t v, uint32_t *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint32_t t = 0;
#pragma unroll
  for (int k = 0; k < NT / 32; k++) t += red[k];
  return t;
}

// Loads kScanItems consecutive counts at c (16-byte aligned), zero past nscan.
__device__ __forceinline__ bool load_counts(const uint32_t *cs, long c, long nscan, uint32_t (&a)[kScanItems]) {
  const bool full = c + kScanItems - 1 < nscan;
  if (full) {
#pragma unroll
    for (int v = 0; v < kScanItems / 4; v++) {
      const uint4 q = *reinterpret_cast<const uint4 *>(cs + c + 4 * v);
      a[4 * v] = q.x; a[4 * v + 1] = q.y; a[4 * v + 2] = q.z; a[4 * v + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; k++) a[k] = (c + k < nscan) ? cs[c + k] : 0u;
  }
  return full;
}

// tsum[t] = sum of the counts of tile t (buckets [t << tshift, (t + 1) << tshift)).
__global__ void __launch_bounds__(kScanThreads) tile_sum_kernel(const uint32_t *__restrict__ cs, long nscan,
                                                                int tshift, uint32_t *__restrict__ tsum) {
  __shared__ uint32_t red[kScanThreads / 32];
  const long t0 = (long)blockIdx.x << tshift;
  const long t1 = min(t0 + (1L << tshift), nscan);
  uint32_t s = 0;
  for (long c = t0 + (long)kScanItems * threadIdx.x; c < t1; c += kScanChunk) {
    uint32_t a[kScanItems];
    load_counts(cs, c, t1, a);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) s += a[k];
  }
  s = block_sum_u32<kScanThreads>(s, red);
  if (threadIdx.x == 0) tsum[blockIdx.x] = s;
}

// cs[0 .. nscan): per-bucket counts in, exclusive prefix sums out, one CTA
// per tile; the tile's base is the sum of the earlier tiles' sums.
__global__ void __launch_bounds__(kScanThreads) cell_offsets_kernel(uint32_t *__restrict__ cs, long nscan,
                                                                    int tshift, const uint32_t *__restrict__ tsum) {
  constexpr int NW = kScanThreads / 32;
  __shared__ uint32_t wsum[NW];
  __shared__ uint32_t red[NW];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t b = 0;
  for (int i = threadIdx.x; i < (int)blockIdx.x; i += kScanThreads) b += tsum[i];
  uint32_t run = block_sum_u32<kScanThreads>(b, red);
  const long t0 = (long)blockIdx.x << tshift;
  const long t1 = min(t0 + (1L << tshift), nscan);
  for (long cb = t0; cb < t1; cb += kScanChunk) {
    const long c = cb + (long)kScanItems * threadIdx.x;
    uint32_t a[kScanItems];
    const bool full = load_counts(cs, c, t1, a);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) s += a[k];
    uint32_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    __syncthreads();  // wsum of the previous pass has been read
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0, blk = 0;
#pragma unroll
    for (int k = 0; k < NW; k++) {
      const uint32_t ws = wsum[k];
      if (k < warp) wpre += ws;
      blk += ws;
    }
    uint32_t e = run + wpre + incl - s;
    uint32_t o[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      o[k] = e;
      e += a[k];
    }
    if (full) {
#pragma unroll
      for (int v = 0; v < kScanItems / 4; v++)
        *reinterpret_cast<uint4 *>(cs + c + 4 * v) = make_uint4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
    } else {
#pragma unroll
      for (int k = 0; k < kScanItems; k++)
        if (c + k < t1) cs[c + k] = o[k];
    }
    run += blk;
  }
}

// Atom a -> offset of its bucket + its arrival slot.  Every atom leaves its
// key and index there in tkeys/tmp (arrival order); an atom alone in its
// bucket is already final (skeys, perm, rec_sorted).
__global__ void __launch_bounds__(256) cell_scatter_kernel(int n, const uint32_t *__restrict__ keys,
                                                           const uint32_t *__restrict__ slot,
                                                           const float4 *__restrict__ rec,
                                                           const int *__restrict__ cs, BucketMap bm,
                                                           uint32_t *__restrict__ skeys, uint32_t *__restrict__ perm,
                                                           uint32_t *__restrict__ tkeys, uint32_t *__restrict__ tmp,
                                                           float4 *__restrict__ rec_sorted) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const uint32_t key = keys[a];
  const uint32_t b = bm(key);
  if (!SPME_IN(b, bm.nb, CK_SORT_BUCKET)) return;
  const int lo = cs[b], hi = cs[b + 1];
  const int pos = lo + (int)slot[a];
  if (!SPME_IN(pos - lo, hi - lo, CK_SORT_SCATTER) || !SPME_IN(hi - 1, n, CK_SORT_SCATTER)) return;
  tkeys[pos] = key;
  tmp[pos] = (uint32_t)a;
  if (hi - lo == 1) {
    skeys[pos] = key;
    perm[pos] = (uint32_t)a;
    rec_sorted[pos] = rec[a];
  }
}

__device__ __forceinline__ bool pair_less(uint32_t ka, uint32_t ia, uint32_t kb, uint32_t ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// Merge sort of one large bucket's (key, index) pairs (distinct pairs) by
// one CTA, ping-ponging between (tkeys, tmp)[lo..) and (skeys, perm)[lo..);
// then the records.
__device__ void big_cell_sort(int lo, int c, uint32_t *tkeys, uint32_t *tmp, uint32_t *skeys, uint32_t *perm,
                              const float4 *__restrict__ rec, float4 *__restrict__ rec_sorted) {
  uint32_t *sk = tkeys + lo, *si = tmp + lo, *dk = skeys + lo, *di = perm + lo;
  for (int wd = 1; wd < c; wd <<= 1) {
    for (int i = threadIdx.x; i < c; i += blockDim.x) {
      const int run = i / wd, rs = run * wd;
      const bool left = (run & 1) == 0;
      const int os = left ? rs + wd : rs - wd;  // partner run
      const int oe = min(os + wd, c);
      const uint32_t vk = sk[i], vi = si[i];
      int l = os, h = (os < c) ? oe : os;  // number of partner pairs below (vk, vi)
      while (l < h) {
        const int m = (l + h) >> 1;
        if (pair_less(sk[m], si[m], vk, vi)) l = m + 1; else h = m;
      }
      const int d = (left ? rs : os) + (i - rs) + (l - os);
      if (!SPME_IN(d, c, CK_SORT_MERGE)) continue;
      dk[d] = vk;
      di[d] = vi;
    }
    __syncthreads();
    uint32_t *t = sk; sk = dk; dk = t;
    t = si; si = di; di = t;
  }
  for (int i = threadIdx.x; i < c; i += blockDim.x) {
    const uint32_t k = sk[i], a = si[i];
    skeys[lo + i] = k;
    perm[lo + i] = a;
    rec_sorted[lo + i] = rec[a];
  }
  __syncthreads();
}

// ctl[0]: number of listed large buckets, ctl[1]: finished CTAs (both zero on
// entry; the last CTA resets ctl[1]).  big: listed bucket indices (capacity n).
__global__ void __launch_bounds__(256) cell_fixup_kernel(int n, const int *__restrict__ cs, BucketMap bm,
                                                         uint32_t *tkeys, uint32_t *tmp, uint32_t *skeys,
                                                         uint32_t *perm, const float4 *__restrict__ rec,
                                                         float4 *__restrict__ rec_sorted, uint32_t *ctl,
                                                         uint32_t *big) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const uint32_t key = tkeys[i];
    const uint32_t b = bm(key);
    const bool ok = SPME_IN(b, bm.nb, CK_SORT_BUCKET);
    const int lo = ok ? cs[b] : 0, c = ok ? cs[b + 1] - lo : 1;
    if (c > kBigCell) {
      if (i == lo) big[atomicAdd(&ctl[0], 1u)] = b;
    } else if (c > 1) {
      const uint32_t a = tmp[i];
      int r = 0;
      for (int j = lo; j < lo + c; j++) r += pair_less(tkeys[j], tmp[j], key, a) ? 1 : 0;
      if (SPME_IN(r, c, CK_SORT_FIXUP) && SPME_IN(lo + c - 1, n, CK_SORT_FIXUP)) {
        skeys[lo + r] = key;
        perm[lo + r] = a;
        rec_sorted[lo + r] = rec[a];
      }
    }
  }
  // the last CTA to finish sorts the listed large buckets
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&ctl[1], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const uint32_t nb = *((volatile uint32_t *)&ctl[0]);
  for (uint32_t k = 0; k < nb; k++) {
    const uint32_t b = *((volatile uint32_t *)&big[k]);
    const int lo = cs[b], c = cs[b + 1] - lo;
    big_cell_sort(lo, c, tkeys, tmp, skeys, perm, rec, rec_sorted);
  }
  if (threadIdx.x == 0) ctl[1] = 0u;
}

// Computes keys/fractions, sorts, and builds the per-bucket offsets.
// On return (stream order): keys[0] / vals[0] hold the stable order,
// rec_sorted the records in that order, cell_start the bucket offsets
// (sort_buckets(g, zshift) + 1 of them).
int launch_cell_sort(const Geom &g, int n, const double *x, const double *w, SortBuffers &b, cudaStream_t st,
                     int zshift) {
  const long nb = sort_buckets(g, zshift);
  const long ntiles = cell_tiles(nb);
  const int tshift = cell_tile_shift(nb);
  const BucketMap bm = bucket_map(g, zshift);
  uint32_t *count = reinterpret_cast<uint32_t *>(b.cell_start);
  uint32_t *ctl = count + (nb + 1);
  uint32_t *head = count + (nb + 3), *tail = count + (2 * nb + 3);
  uint32_t *tsum = count + (3 * nb + 3);
  const int ht_h = zshift > 0 ? g.order / 2 : 0;  // head/tail counts for the spread's buckets only
  b.cur = 0;
  cudaMemsetAsync(count, 0, sizeof(uint32_t) * ((ht_h ? 3 * nb : nb) + 3), st);
  int launches = 0;
  if (n > 0) {
    key_count_kernel<<<ceil_div(n, 256), 256, 0, st>>>(g, n, x, w, b.keys[1], b.vals[1], b.rec, count, bm,
                                                       ht_h ? head : nullptr, tail, ht_h);
    launches++;
  }
  if (ntiles > 1) {  // one tile (grids up to about 64^3): its scan starts from 0, no tile sums needed
    tile_sum_kernel<<<(unsigned)ntiles, kScanThreads, 0, st>>>(count, nb + 1, tshift, tsum);
    launches++;
  }
  cell_offsets_kernel<<<(unsigned)ntiles, kScanThreads, 0, st>>>(count, nb + 1, tshift, tsum);
  launches++;
  if (n > 0) {
    cell_scatter_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, b.keys[1], b.vals[1], b.rec, b.cell_start, bm,
                                                          b.keys[0], b.vals[0], b.tkeys, b.tmp, b.rec_sorted);
    cell_fixup_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, b.cell_start, bm, b.tkeys, b.tmp, b.keys[0], b.vals[0],
                                                        b.rec, b.rec_sorted, ctl, b.hist);
    launches += 2;
  }
  return launches;
}

}  // namespace spme

// ---------------------------------------------------------------------------
// Cell sort that allocates nothing.
//
// Some host programs cannot let a library allocate device memory: an MD
// engine or a serving process that has already handed the whole device to
// its own memory pool, or a time-critical loop that must never pay for the
// device-wide synchronisation cudaMalloc and cudaFree imply.  For them,
// sfac_cell_sort_noalloc() runs the same stable cell sort as sfac() with all
// of its scratch in one fixed file-scope device array, sized for at most
// kNoAllocMaxAtoms atoms (about 1.6 MB).  Every GPU that loads this library
// holds that array until the process exits.  The caller passes the device
// inputs and outputs.
namespace {

using namespace spme;

constexpr int kNoAllocMaxAtoms = 1 << 16;
constexpr int kNoAllocTiles = kNoAllocMaxAtoms / RS_TILE;
constexpr size_t kNaKeys = 0;                                                  // u32 keys, one side of the ping-pong
constexpr size_t kNaVals = kNaKeys + sizeof(uint32_t) * kNoAllocMaxAtoms;      // u32 indices, same side
constexpr size_t kNaRec = kNaVals + sizeof(uint32_t) * kNoAllocMaxAtoms;       // float4 records (not returned)
constexpr size_t kNaHist = kNaRec + sizeof(float4) * kNoAllocMaxAtoms;         // per-tile digit histograms
constexpr size_t kNaTotals = kNaHist + sizeof(uint32_t) * RS_MAX_PASSES * RS_BINS * kNoAllocTiles;
constexpr size_t kNaCell = kNaTotals + sizeof(uint32_t) * RS_MAX_PASSES * RS_BINS;  // box constants
constexpr size_t kNoAllocBytes = kNaCell + 256;

static __device__ __align__(256) unsigned char g_sort_scratch[kNoAllocBytes];

// Device address of g_sort_scratch, looked up once per device (the host-side
// symbol is only a stand-in: a kernel must be given this address instead).
// The cached address belongs to the device's primary context: it does not
// survive cudaDeviceReset, after which this entry point must not be called.
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Writes the box constants (a kernel argument) to device memory.
__global__ void store_cell_kernel(CellConst c, CellConst *dst) { *dst = c; }

unsigned char *noalloc_scratch() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess) {
      fprintf(stderr, "sfac_cell_sort_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
              cudaGetErrorString(e));
      return nullptr;
    }
    g_noalloc_ptr[dev] = static_cast<unsigned char *>(p);
  }
  return g_noalloc_ptr[dev];
}

}  // namespace

extern "C" int sfac_cell_sort_noalloc(const double L[6], const int K[3], int n, const double *x, int *keys,
                                      int *perm, void *stream) {
  if (!L || !K || n < 0 || (n > 0 && (!x || !keys || !perm))) {
    fprintf(stderr, "sfac_cell_sort_noalloc: bad arguments\n");
    return 1;
  }
  if (K[0] < 1 || K[1] < 1 || K[2] < 1 || (long)K[0] * K[1] * K[2] >= 0x7fffffffL) {
    fprintf(stderr, "sfac_cell_sort_noalloc: bad grid %d %d %d\n", K[0], K[1], K[2]);
    return 1;
  }
  if (n > kNoAllocMaxAtoms) {
    fprintf(stderr,
            "sfac_cell_sort_noalloc: %d atoms exceed the fixed scratch capacity of %d atoms "
            "(use sfac() on a handle for larger systems)\n",
            n, kNoAllocMaxAtoms);
    return 1;
  }
  if (n == 0) return 0;
  unsigned char *base = noalloc_scratch();
  if (!base) return 2;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // Box constants with the reference's expressions (sfac.hpp:45-51), written
  // into the scratch array by a one-thread kernel that takes them by value:
  // no host address is handed to the stream.
  CellConst *dcell = reinterpret_cast<CellConst *>(base + kNaCell);
  store_cell_kernel<<<1, 1, 0, st>>>(make_cell(L), dcell);
  Geom g{};
  g.K0 = K[0];
  g.K1 = K[1];
  g.K2 = K[2];
  g.ldim = K[2] / 2 + 1;
  g.cell = dcell;

  const long ncell = (long)K[0] * K[1] * K[2];
  const int npass = key_passes(ncell);
  const int ntiles = ceil_div(n, RS_TILE);
  uint32_t *hist = reinterpret_cast<uint32_t *>(base + kNaHist);
  uint32_t *totals = reinterpret_cast<uint32_t *>(base + kNaTotals);
  float4 *rec = reinterpret_cast<float4 *>(base + kNaRec);
  // Ping-pong between the scratch side (0) and the caller's outputs (1),
  // starting on the side that makes the last pass land in the outputs.
  uint32_t *kb[2] = {reinterpret_cast<uint32_t *>(base + kNaKeys), reinterpret_cast<uint32_t *>(keys)};
  uint32_t *vb[2] = {reinterpret_cast<uint32_t *>(base + kNaVals), reinterpret_cast<uint32_t *>(perm)};
  int src = (npass & 1) ? 0 : 1;

  // The array keeps the previous call's contents: the digit totals must
  // start at zero (every other scratch word is written before it is read).
  if (cudaMemsetAsync(totals, 0, sizeof(uint32_t) * RS_BINS * npass, st) != cudaSuccess) return 2;
  // The records are not returned; x stands in for the weights they carry.
  key_hist_kernel<<<ntiles, RS_THREADS, 0, st>>>(g, n, x, x, kb[src], rec, hist, ntiles, npass, totals);
  for (int p = 0; p < npass; p++) {
    const int dst = src ^ 1;
    const bool last = (p == npass - 1);
    uint32_t *hp = hist + (size_t)p * RS_BINS * ntiles;
    hist_scan_kernel<<<RS_BINS, 256, 0, st>>>(hp, ntiles, totals + p * RS_BINS);
    radix_scatter_kernel<<<ntiles, RS_THREADS, 0, st>>>(kb[src], p == 0 ? nullptr : vb[src], kb[dst], vb[dst], n,
                                                        8 * p, hp, ntiles,
                                                        last ? nullptr : hp + (size_t)RS_BINS * ntiles, rec,
                                                        nullptr);
    src = dst;
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "sfac_cell_sort_noalloc: %s\n", cudaGetErrorString(e));
    return 2;
  }
  return 0;
}
