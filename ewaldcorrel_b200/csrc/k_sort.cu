// K1: integer cell keys and the stable cell sort (SFac::sort, sfac.cpp:92-111).
//
// The reference inserts every atom into a std::multimap keyed by
// cid = (n0*K1 + n1)*K2 + n2; equal keys keep insertion order, so the result
// is the STABLE sort of atoms by cid.  Here: one FP64 key kernel (rounding
// identical to the host, so boundary atoms land in the same cell), then an
// LSD radix sort with 8-bit digits whose scatter ranks ties in input order
// (stable by construction, bit-exact against the CPU sort), then per-cell
// start offsets by binary search over the sorted keys.
#include "spme_kernels.hpp"

namespace spme {

// ---------------------------------------------------------------- keys ---
// Cell index and in-cell fraction, exactly as SFac::sort computes them
// (sfac.cpp:98-106): u = s*K, n = (int)u, u -= n.  A coordinate that wrapped
// to exactly 1.0 (Cell::wrap of a tiny negative number) is mapped to its
// periodic image 0 instead of forming the out-of-range key K.
__global__ void __launch_bounds__(256) cell_key_kernel(Geom g, int n, const double *__restrict__ x,
                                                       const double *__restrict__ w,
                                                       uint32_t *__restrict__ keys,
                                                       uint32_t *__restrict__ idx,
                                                       float4 *__restrict__ rec) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  double s0, s1, s2;
  frac_coords(g, x[3 * a + 0], x[3 * a + 1], x[3 * a + 2], s0, s1, s2);
  double u0 = __dmul_rn(s0, (double)g.K0), u1 = __dmul_rn(s1, (double)g.K1),
         u2 = __dmul_rn(s2, (double)g.K2);
  int n0 = __double2int_rz(u0), n1 = __double2int_rz(u1), n2 = __double2int_rz(u2);
  double f0 = __dsub_rn(u0, (double)n0), f1 = __dsub_rn(u1, (double)n1),
         f2 = __dsub_rn(u2, (double)n2);
  if (n0 >= g.K0) { n0 = 0; f0 = 0.0; }
  if (n1 >= g.K1) { n1 = 0; f1 = 0.0; }
  if (n2 >= g.K2) { n2 = 0; f2 = 0.0; }
  keys[a] = (uint32_t)((n0 * g.K1 + n1) * g.K2 + n2);
  idx[a] = (uint32_t)a;
  rec[a] = make_float4((float)f0, (float)f1, (float)f2, (float)w[a]);
}

// ------------------------------------------------------------ radix sort ---
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 2048 keys per tile
constexpr int RS_BINS = 256;

// Per-tile digit histogram, stored digit-major: hist[d * ntiles + tile].
__global__ void __launch_bounds__(RS_THREADS) radix_hist_kernel(const uint32_t *__restrict__ keys,
                                                                int n, int shift,
                                                                uint32_t *__restrict__ hist,
                                                                int ntiles) {
  __shared__ uint32_t h[RS_BINS];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE;
#pragma unroll
  for (int it = 0; it < RS_ITEMS; it++) {
    int i = base + it * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xff], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of `count` entries in place, one block of 1024 threads.
// Integer sums: the result does not depend on the order of additions.
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(uint32_t *__restrict__ data, int count) {
  __shared__ uint32_t part[1024];
  const int t = threadIdx.x;
  const int chunk = (count + 1023) / 1024;
  const int lo = min(count, t * chunk), hi = min(count, lo + chunk);
  uint32_t s = 0;
  for (int i = lo; i < hi; i++) s += data[i];
  part[t] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan over the 1024 partial sums.
  for (int off = 1; off < 1024; off <<= 1) {
    uint32_t v = (t >= off) ? part[t - off] : 0u;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint32_t run = (t == 0) ? 0u : part[t - 1];
  for (int i = lo; i < hi; i++) {
    uint32_t v = data[i];
    data[i] = run;
    run += v;
  }
}

// Stable scatter of one 8-bit digit.  Each warp owns a contiguous run of
// 32*RS_ITEMS keys of the tile and walks it in memory order; ties inside a
// round of 32 are ranked by lane, ties across rounds and warps by a running
// per-warp digit count, ties across tiles by the scanned histogram.
__global__ void __launch_bounds__(RS_THREADS) radix_scatter_kernel(
    const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint32_t *__restrict__ kout,
    uint32_t *__restrict__ vout, int n, int shift, const uint32_t *__restrict__ offs, int ntiles) {
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
    val[it] = valid ? vin[i] : 0u;
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
  {  // exclusive prefix over warps, one thread per digit
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) {
      uint32_t c = whist[w][d];
      whist[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < RS_ITEMS; it++) {
    const int i = base + it * 32 + lane;
    if (i < n) {
      const uint32_t d = (key[it] >> shift) & 0xff;
      const uint32_t pos = offs[d * ntiles + blockIdx.x] + whist[warp][d] + rank[it];
      kout[pos] = key[it];
      vout[pos] = val[it];
    }
  }
}

// rec_sorted[r] = rec[perm[r]]: atom records in cell order.
__global__ void __launch_bounds__(256) gather_records_kernel(int n, const uint32_t *__restrict__ perm,
                                                             const float4 *__restrict__ rec,
                                                             float4 *__restrict__ rec_sorted) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) rec_sorted[r] = rec[perm[r]];
}

// cell_start[c] = first sorted rank whose key >= c, for c in [0, ncell].
__global__ void __launch_bounds__(256) cell_start_kernel(int n, const uint32_t *__restrict__ keys,
                                                         long ncell, int *__restrict__ cell_start) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ncell) return;
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if ((long)keys[mid] < c) lo = mid + 1; else hi = mid;
  }
  cell_start[c] = lo;
}

static int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

size_t sort_scratch_words(int cap) {
  const int ntiles = ceil_div(cap > 0 ? cap : 1, RS_TILE);
  return (size_t)ntiles * RS_BINS;
}

// Computes keys/fractions, sorts, and builds the per-cell offsets.
// On return (stream order): keys_sorted / perm hold the stable order,
// rec_sorted the records in that order, cell_start the cell offsets.
int launch_cell_sort(const Geom &g, int n, const double *x, const double *w, SortBuffers &b,
                     cudaStream_t st) {
  const long ncell = (long)g.K0 * g.K1 * g.K2;
  int launches = 0;
  if (n > 0) {
    cell_key_kernel<<<ceil_div(n, 256), 256, 0, st>>>(g, n, x, w, b.keys[0], b.vals[0], b.rec);
    launches++;
    int bits = 1;
    while (bits < 32 && ((ncell - 1) >> bits) > 0) bits++;
    const int ntiles = ceil_div(n, RS_TILE);
    int cur = 0;
    for (int shift = 0; shift < bits; shift += 8) {
      radix_hist_kernel<<<ntiles, RS_THREADS, 0, st>>>(b.keys[cur], n, shift, b.hist, ntiles);
      exclusive_scan_kernel<<<1, 1024, 0, st>>>(b.hist, ntiles * RS_BINS);
      radix_scatter_kernel<<<ntiles, RS_THREADS, 0, st>>>(b.keys[cur], b.vals[cur], b.keys[cur ^ 1],
                                                          b.vals[cur ^ 1], n, shift, b.hist, ntiles);
      cur ^= 1;
      launches += 3;
    }
    b.cur = cur;
    gather_records_kernel<<<ceil_div(n, 256), 256, 0, st>>>(n, b.vals[cur], b.rec, b.rec_sorted);
    launches++;
  } else {
    b.cur = 0;
  }
  cell_start_kernel<<<ceil_div(ncell + 1, 256), 256, 0, st>>>(n, b.keys[b.cur], ncell, b.cell_start);
  return launches + 1;
}

}  // namespace spme
