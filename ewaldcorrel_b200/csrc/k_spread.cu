// K2: B-spline charge spreading (SFac::operator() + accum_spline,
// sfac.cpp:113-124,141-168).
//
// Owner-computes, like the reference's accum_spline: every grid point has
// exactly one writer, which adds the contributions of the atoms in its
// order^3 neighbouring cells in a fixed order.  No atomics, so the grid is
// bit-for-bit reproducible.
//
// Blocking: a warp owns an 8 x 8 x 16 brick of grid points in registers.
// Lane (lx, ly) holds the two neighbouring columns x = 2 lx, 2 lx + 1 at
// y = ly, 16 z points each, as packed FP32 pairs along z (z = 2j, 2j + 1),
// so that one packed FMA (fma.rn.f32x2) adds an atom's weight times two
// consecutive z taps to one column.  Pairs along z rather than across the
// two columns: the taps then need no duplication (2 instead of 3 shared
// loads per atom and brick at order 6), with the same products in the same
// order, so the same bits.  The brick is 16 deep rather than 32 so that the
// kernel fits in 64 registers: 8 CTAs of 4 warps per SM hide the shared-memory
// latency of the walk better than 5 at 96 registers outweigh the longer z
// halo.  The atoms of the brick's halo (the cells whose stencils reach it)
// are the sorted atoms of (x, y) cell rows, found through the bucket offsets
// of the cell sort (runs of 32 z cells per row); a brick's halo starts H = p/2
// cells before a bucket boundary (even bricks) or ends H - 1 cells after one
// (odd bricks), where the sort's per-bucket tail/head counts give the cut
// without a search.
//
// The atoms are staged 32 at a time, one per lane, at the row given by a
// counting sort of the chunk on its window case (the place of the atom's z
// taps in the brick, the same for every lane; ties in lane order).  Staging
// evaluates the order-p B-spline taps of the three fractions (the charge
// folded into x) once and stores what the lanes will read: the weights of
// the brick's 8 x columns (as the 4 pairs the lanes hold) and 8 y rows,
// written straight to their columns of rows the warp has zeroed, and the z
// taps as consecutive pairs from the even z at or below the first tap.  The
// walk goes window case by window case in a compile-time unrolled chain,
// each case a plain loop over its contiguous rows: per atom, the lane's x
// pair and y weight, two multiplies, the z pairs and two packed FMAs per
// pair into fixed registers -- no indirect jump, no divergent branch.  Small
// grids split one brick's atoms over 2 or 4 warps (equal contiguous shares,
// summed in warp order through shared memory: still a fixed order).
#include "spme_kernels.hpp"

namespace spme {

SPME_CHECK_READER(spread)

constexpr int SP_TX = 8, SP_TY = 8, SP_TZ = 16;  // brick of one warp
constexpr int SP_MIN_CTAS = 8;                  // resident CTAs per SM (64 registers)
constexpr int SP_WARPS = 4;                     // warps per CTA

typedef unsigned long long f2r;  // two FP32 values in one 64-bit register (low word first)

__device__ __forceinline__ f2r pack2(float lo, float hi) {
  f2r r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void unpack2(f2r r, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(r));
}
// d = a * b + c on both halves, round to nearest (two FP32 FMAs).
__device__ __forceinline__ f2r ffma2(f2r a, f2r b, f2r c) {
  f2r d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

template <int P>
struct SpCfg {
  static constexpr int H = P / 2;
  // halo cell rows of a brick: cells [x0 - H, x0 + TX - 2 + H] (RX of them)
  static constexpr int RX = SP_TX + P - 1, RY = SP_TY + P - 1, NR = RX * RY;
  static constexpr int NC = SP_TZ + P - 1;  // window cases: first z tap rz in [1 - P, TZ - 1]
  // z taps as consecutive pairs (z, z + 1) from the even z at or below the first
  // tap: P + 2 values, ZQ pairs, rows rounded to whole 16-byte loads (ZQE pairs)
  static constexpr int ZQ = P / 2 + 1;
  static constexpr int ZQE = (ZQ + 1) / 2 * 2;
};

// Shared memory of one warp.
template <int P>
struct SpStage {
  using C = SpCfg<P>;
  f2r zq[32][C::ZQE];  // (w(zs + 2m), w(zs + 2m + 1)): z taps from the even zs <= rz, zero off the stencil
  __align__(16) f2r wxl[32][5];  // x weights of columns (2 lx, 2 lx + 1), lx = 0..3 (row padded to 5 pairs)
  __align__(16) float wyl[32][9]; // y weights of rows 0..7 (padded to 9: the staging stores spread over the banks)
  int cnt[64];         // atoms per window case in the chunk, then the case starts
};
constexpr int kRowMap = 512;
static_assert(SpCfg<8>::NR <= 256, "halo rows fit a byte");
template <int P>
struct SpGroup {  // per brick: the halo rows' atom ranges of one z piece
  int start[SpCfg<P>::NR];
  int pref[SpCfg<P>::NR + 1];
  uint8_t rowmap[kRowMap];  // halo row of each of the piece's atoms (pieces of at most kRowMap atoms)
};
template <int P, int NS>
constexpr size_t sp_stage_bytes() {
  if (NS == 1) return sizeof(SpStage<P>);
  return sizeof(SpStage<P>) > 2 * SP_TZ * 33 * 4 ? sizeof(SpStage<P>) : 2 * SP_TZ * 33 * 4;
}
template <int P, int NS>
constexpr size_t sp_smem_bytes() {
  return SP_WARPS * (sp_stage_bytes<P, NS>() + sizeof(SpGroup<P>));
}

// acc[c][j] += d_c * zq[m] for the pairs m whose z = zs + 2m lies in the brick
// (zs: the even z at or below the first tap rz = C - (P - 1); all indices
// compile-time); pairs that hold no tap of this case are skipped.
template <int P, int C>
__device__ __forceinline__ void sp_taps(f2r (&acc)[2][SP_TZ / 2], f2r d0, f2r d1,
                                        const f2r (&zq)[SpCfg<P>::ZQE]) {
  constexpr int rz = C - (P - 1);
  constexpr int par = rz & 1;
  constexpr int zs = rz - par;
  constexpr int used = (P + par + 1) / 2;  // pairs holding taps
#pragma unroll
  for (int m = 0; m < used; m++) {
    const int jz = zs / 2 + m;
    if (jz >= 0 && jz < SP_TZ / 2) {
      acc[0][jz] = ffma2(d0, zq[m], acc[0][jz]);
      acc[1][jz] = ffma2(d1, zq[m], acc[1][jz]);
    }
  }
}

// The walk over one staged chunk, window case by window case: case C (all
// compile-time, so every accumulator index is fixed) adds the staged rows
// [start[C], start[C + 1]); a case absent from the chunk costs one test.
template <int P, int C>
__device__ __forceinline__ void sp_walk(f2r (&acc)[2][SP_TZ / 2], const SpStage<P> &st, int lx, int ly, int k) {
  if constexpr (C < SpCfg<P>::NC) {
    const int e = st.cnt[C + 1];
#pragma unroll 1
    for (; k < e; k++) {
      const float2 xp = *reinterpret_cast<const float2 *>(&st.wxl[k][lx]);
      const float wy = st.wyl[k][ly];
      const float w0 = xp.x * wy, w1 = xp.y * wy;
      const f2r d0 = pack2(w0, w0), d1 = pack2(w1, w1);
      f2r zq[SpCfg<P>::ZQE];
#pragma unroll
      for (int v = 0; v < SpCfg<P>::ZQE / 2; v++) {
        const ulonglong2 q = *reinterpret_cast<const ulonglong2 *>(&st.zq[k][2 * v]);
        zq[2 * v] = q.x;
        zq[2 * v + 1] = q.y;
      }
      sp_taps<P, C>(acc, d0, d1, zq);
    }
    sp_walk<P, C + 1>(acc, st, lx, ly, k);
  }
}

// Barrier of the NS warps that share one brick (named barrier 1 + group).
template <int NS>
__device__ __forceinline__ void group_sync(int group) {
  if constexpr (NS == 1) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + group), "n"(32 * NS) : "memory");
  }
}

// First index in [lo, hi) whose key is >= k (keys sorted).
__device__ __forceinline__ int keys_lower_bound(const uint32_t *__restrict__ keys, int lo, int hi, uint32_t k) {
  while (lo < hi) {
    const int m = (lo + hi) >> 1;
    if (__ldg(keys + m) < k) lo = m + 1; else hi = m;
  }
  return lo;
}

// v mod K: one test each way for v in [-K, 2K) (near), the full modulus otherwise.
__device__ __forceinline__ int wrap_near(int v, int K, bool near) {
  if (near) return v < 0 ? v + K : (v >= K ? v - K : v);
  return imod(v, K);
}

struct SpArgs {
  Geom g;
  const int *cs;          // bucket offsets (runs of 32 z cells per row)
  const uint32_t *head;   // per bucket: atoms in its first H - 1 cells
  const uint32_t *tail;   // per bucket: atoms in its last H cells
  const uint32_t *keys;   // sorted cell keys
  const float4 *rec;      // sorted (fx, fy, fz, q)
  float *grid;
  int ntx, nty, ntz, nbricks;
  int nzb;
  long nb;                // buckets (cs holds nb + 1 offsets; cs[nb] = atoms)
  FastDiv K2d;
};

template <int P, int NS>
__global__ void __launch_bounds__(SP_WARPS * 32, SP_MIN_CTAS) spread_kernel(SpArgs A, Spline S) {
  using C = SpCfg<P>;
  constexpr int H = C::H, RX = C::RX, RY = C::RY, NR = C::NR, NC = C::NC;
  constexpr int ZB = kSpreadZShift, ZW = 1 << ZB;  // bucket of the sort: 32 z cells
  extern __shared__ __align__(16) unsigned char sp_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int group = warp / NS, member = warp % NS;
  SpStage<P> &st = *reinterpret_cast<SpStage<P> *>(sp_smem + warp * sp_stage_bytes<P, NS>());
  SpGroup<P> &gr = *reinterpret_cast<SpGroup<P> *>(sp_smem + SP_WARPS * sp_stage_bytes<P, NS>() +
                                                   group * sizeof(SpGroup<P>));
  const long brick = (long)blockIdx.x * (SP_WARPS / NS) + group;
  if (brick >= A.nbricks) return;  // the whole group leaves together
  const Geom &g = A.g;
  const int K0 = g.K0, K1 = g.K1, K2 = g.K2;
  const int tz = (int)(brick % A.ntz), ty = (int)((brick / A.ntz) % A.nty), tx = (int)(brick / ((long)A.ntz * A.nty));
  const int x0 = tx * SP_TX, y0 = ty * SP_TY, z0 = tz * SP_TZ;
  const int lx = lane & 3, ly = lane >> 2;
  const int gt = member * 32 + lane, gn = 32 * NS;  // thread index and size of the group
  const bool nearx = K0 >= RX, neary = K1 >= RY;


  f2r acc[2][SP_TZ / 2];  // column 2 lx + c at z = 2j, 2j + 1
#pragma unroll
  for (int j = 0; j < SP_TZ / 2; j++) acc[0][j] = acc[1][j] = 0ull;

  // extended z cells whose stencils reach [z0, z0 + TZ): [z0 - H, z0 + TZ + H - 2],
  // walked in pieces that do not cross the periodic boundary
  const int ez_lo = z0 - H, ez_hi = z0 + SP_TZ + H - 2;
  for (int ezs = ez_lo; ezs <= ez_hi;) {
    const int n2a = imod(ezs, K2);
    const int len = min(ez_hi - ezs + 1, K2 - n2a);
    const int n2e = n2a + len;  // one past the piece's last cell
    group_sync<NS>(group);  // the previous piece's ranges are no longer read
    for (int r = gt; r < NR; r += gn) {
      const int ex = x0 - H + r / RY, ey = y0 - H + r % RY;
      const int row = wrap_near(ex, K0, nearx) * K1 + wrap_near(ey, K1, neary);
      const int b0 = row * A.nzb + (n2a >> ZB), b1 = row * A.nzb + ((n2e - 1) >> ZB);
      const uint32_t kbase = (uint32_t)row * (uint32_t)K2;
      if (!SPME_IN(b0, A.nb, CK_SPREAD_BUCKET) || !SPME_IN(b1, A.nb, CK_SPREAD_BUCKET)) {
        gr.start[r] = 0;
        gr.pref[r + 1] = 0;
        continue;
      }
      int lo, hi;
      const int lo_off = n2a & (ZW - 1), hi_off = n2e & (ZW - 1);
      if (lo_off == 0) lo = __ldg(A.cs + b0);
      else if (lo_off == ZW - H) lo = __ldg(A.cs + b0 + 1) - (int)__ldg(A.tail + b0);
      else lo = keys_lower_bound(A.keys, __ldg(A.cs + b0), __ldg(A.cs + b0 + 1), kbase + n2a);
      if (hi_off == 0 || n2e == K2) hi = __ldg(A.cs + b1 + 1);
      else if (hi_off == H - 1) hi = __ldg(A.cs + b1) + (int)__ldg(A.head + b1);
      else hi = keys_lower_bound(A.keys, __ldg(A.cs + b1), __ldg(A.cs + b1 + 1), kbase + n2e);
      if (!SPME_IN(lo - A.cs[b0], A.cs[b1 + 1] - A.cs[b0] + 1, CK_SPREAD_RANGE) ||
          !SPME_IN(hi - lo, A.cs[b1 + 1] - lo + 1, CK_SPREAD_RANGE))
        hi = lo;
      gr.start[r] = lo;
      gr.pref[r + 1] = hi - lo;
    }
    group_sync<NS>(group);
    if (member == 0) {
      int running = 0;
      for (int c = 0; c < NR; c += 32) {
        const int r = c + lane;
        int v = (r < NR) ? gr.pref[r + 1] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int u = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += u;
        }
        if (r < NR) gr.pref[r + 1] = running + v;
        running += __shfl_sync(0xffffffffu, v, 31);
      }
      if (lane == 0) gr.pref[0] = 0;
    }
    group_sync<NS>(group);
    const int total = gr.pref[NR];
    const int zoff = ezs - n2a + 1 - H - z0;  // first z tap of an atom in stored cell n2: n2 + zoff
    const bool mapped = total <= kRowMap;
    if (mapped) {
      for (int r = gt; r < NR; r += gn)
        for (int k = gr.pref[r], e = gr.pref[r + 1]; k < e; k++) gr.rowmap[k] = (uint8_t)r;
      group_sync<NS>(group);
    }
    const int w_lo = (int)((long)total * member / NS), w_hi = (int)((long)total * (member + 1) / NS);
    for (int chunk = w_lo; chunk < w_hi; chunk += 32) {
      const int t = chunk + lane;
      bool valid = t < w_hi;
      int a = 0, hr = 0, mycase = NC;  // NC: no atom (sorts last, never walked)
      float4 u = make_float4(0.f, 0.f, 0.f, 0.f);
      if (valid) {
        int lo;
        if (mapped) {
          lo = gr.rowmap[t];
        } else {
          lo = 0;  // largest r with pref[r] <= t
          int hi = NR - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (gr.pref[mid] <= t) lo = mid; else hi = mid - 1;
          }
        }
        a = gr.start[lo] + (t - gr.pref[lo]);
        hr = lo;
        if (SPME_IN(a, A.cs[A.nb], CK_SPREAD_ATOM)) {
          uint32_t qk, n2;
          const uint32_t key = __ldg(A.keys + a);
          u = __ldg(A.rec + a);
          A.K2d.divmod(key, qk, n2);
          mycase = (int)n2 + zoff + P - 1;  // in [0, NC): first z tap rz = mycase - (P - 1)
          if (!SPME_IN(mycase, NC, CK_SPREAD_CASE)) valid = false, mycase = NC;
        } else {
          valid = false;
        }
      }
      // counting sort of the chunk on the window case, ties in lane order:
      // cnt[c] = atoms of case c, then (exclusive scan) the first row of case c
      st.cnt[lane] = 0;
      st.cnt[lane + 32] = 0;
      __syncwarp();
      const uint32_t peers = __match_any_sync(0xffffffffu, mycase);
      if (lane == __ffs(peers) - 1) st.cnt[mycase] = __popc(peers);
      __syncwarp();
      {
        const int e0 = st.cnt[2 * lane], e1 = st.cnt[2 * lane + 1];
        int incl = e0 + e1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int u = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += u;
        }
        __syncwarp();
        st.cnt[2 * lane] = incl - e0 - e1;
        st.cnt[2 * lane + 1] = incl - e1;
      }
      // zero the chunk's x/y weight rows with contiguous stores of the whole warp
      {
        float4 *zx = reinterpret_cast<float4 *>(&st.wxl[0][0]);
        float4 *zy = reinterpret_cast<float4 *>(&st.wyl[0][0]);
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        constexpr int NX = sizeof(st.wxl) / 16, NY = sizeof(st.wyl) / 16;
        static_assert(sizeof(st.wxl) % 16 == 0 && sizeof(st.wyl) % 16 == 0, "whole 16-byte stores");
#pragma unroll
        for (int v = 0; v < 3; v++) {
          if (v * 32 + lane < NX) zx[v * 32 + lane] = z4;
          if (v * 32 + lane < NY) zy[v * 32 + lane] = z4;
        }
      }
      __syncwarp();
      if (valid) {
        int row = st.cnt[mycase] + __popc(peers & ((1u << lane) - 1u));
        if (!SPME_IN(row, 32, CK_SPREAD_ROW)) row = 0;
        // tap i of each axis: the weight of point first + i, M(f + P - 1 - i);
        // the brick's column c = i + rx - (P - 1) takes tap i (zero elsewhere)
        float *wxr = reinterpret_cast<float *>(&st.wxl[row][0]);
        float *wyr = &st.wyl[row][0];
        const int cx = hr / RY - (P - 1), cy = hr % RY - (P - 1);
        float zt[P];
#pragma unroll
        for (int i = 0; i < P; i++) {
          const float wx = u.w * bspl_eval(S, P, u.x, P - 1 - i);
          const float wy = bspl_eval(S, P, u.y, P - 1 - i);
          const float wz = bspl_eval(S, P, u.z, P - 1 - i);
          if ((unsigned)(cx + i) < 8u) wxr[cx + i] = wx;
          if ((unsigned)(cy + i) < 8u) wyr[cy + i] = wy;
          zt[i] = wz;
        }
        // pair m holds taps 2m - par and 2m + 1 - par (par: parity of the first tap's z)
        const int par = (mycase - (P - 1)) & 1;
        float zv[2 * SpCfg<P>::ZQE];
#pragma unroll
        for (int q = 0; q < 2 * SpCfg<P>::ZQE; q++) {
          const float a = (q < P) ? zt[q] : 0.f;                      // par 0: tap q
          const float b = (q >= 1 && q - 1 < P) ? zt[q - 1] : 0.f;   // par 1: tap q - 1
          zv[q] = par ? b : a;
        }
#pragma unroll
        for (int v = 0; v < SpCfg<P>::ZQE / 2; v++)
          *reinterpret_cast<ulonglong2 *>(&st.zq[row][2 * v]) =
              make_ulonglong2(pack2(zv[4 * v], zv[4 * v + 1]), pack2(zv[4 * v + 2], zv[4 * v + 3]));
      }
      __syncwarp();
      sp_walk<P, 0>(acc, st, lx, ly, 0);
      __syncwarp();  // the next chunk's staging overwrites these atoms
    }
    ezs += len;
  }

  if constexpr (NS == 1) {
    // one writer per brick: each lane stores its two columns from registers
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int gx = x0 + 2 * lx + c, gy = y0 + ly;
      if (gx >= K0 || gy >= K1) continue;
      float *col = A.grid + ((long)gx * K1 + gy) * K2 + z0;
      if (!SPME_IN(((long)gx * K1 + gy) * K2 + min(z0 + SP_TZ, K2) - 1, (long)K0 * K1 * K2, CK_SPREAD_GRID)) continue;
      if ((K2 & 3) == 0 && z0 + SP_TZ <= K2) {
#pragma unroll
        for (int z = 0; z < SP_TZ; z += 4)  // a pair holds (z, z + 1), low word first: the grid's own order
          *reinterpret_cast<ulonglong2 *>(col + z) = make_ulonglong2(acc[c][z / 2], acc[c][z / 2 + 1]);
      } else {
#pragma unroll
        for (int z = 0; z < SP_TZ; z++) {
          float lo, hi;
          unpack2(acc[c][z / 2], lo, hi);
          if (z0 + z < K2) col[z] = (z & 1) ? hi : lo;
        }
      }
    }
  } else {
    // partial bricks to shared memory (over the staging rows), summed over the
    // group's warps in warp order, stored with consecutive threads on
    // consecutive z (coalesced)
    group_sync<NS>(group);
    float *part = reinterpret_cast<float *>(&st);  // [k * SP_TZ + z][33]: column 2 lx + k of lane
#pragma unroll
    for (int j = 0; j < SP_TZ / 2; j++) {
      float a0, a1, b0, b1;
      unpack2(acc[0][j], a0, a1);  // column 2 lx at z = 2j, 2j + 1
      unpack2(acc[1][j], b0, b1);  // column 2 lx + 1
      part[(2 * j) * 33 + lane] = a0;
      part[(2 * j + 1) * 33 + lane] = a1;
      part[(SP_TZ + 2 * j) * 33 + lane] = b0;
      part[(SP_TZ + 2 * j + 1) * 33 + lane] = b1;
    }
    group_sync<NS>(group);
    const float *gpart = reinterpret_cast<const float *>(sp_smem + (size_t)group * NS * sp_stage_bytes<P, NS>());
    const size_t mstride = sp_stage_bytes<P, NS>() / sizeof(float);
    for (int p = gt; p < SP_TX * SP_TY * SP_TZ; p += gn) {
      const int z = p % SP_TZ, col = p / SP_TZ;
      const int xr = col >> 3, yr = col & 7;
      const int src = ((xr & 1) * SP_TZ + z) * 33 + (xr >> 1) + 4 * yr;
      float v = gpart[src];
#pragma unroll
      for (int m = 1; m < NS; m++) v += gpart[m * mstride + src];
      const int gx = x0 + xr, gy = y0 + yr, gz = z0 + z;
      if (gx < K0 && gy < K1 && gz < K2) A.grid[((long)gx * K1 + gy) * K2 + gz] = v;
    }
  }
}

template <int P, int NS>
static void spread_ps(const SpArgs &A, const Spline &S, cudaStream_t st) {
  constexpr int per_cta = SP_WARPS / NS;
  const long ctas = (A.nbricks + per_cta - 1) / per_cta;
  spread_kernel<P, NS><<<(unsigned)ctas, SP_WARPS * 32, sp_smem_bytes<P, NS>(), st>>>(A, S);
}

template <int P>
static void spread_p(const SpArgs &A, int nsplit, const Spline &S, cudaStream_t st) {
  if (nsplit == 1) spread_ps<P, 1>(A, S, st);
  else if (nsplit == 2) spread_ps<P, 2>(A, S, st);
  else spread_ps<P, 4>(A, S, st);
}

template <int P>
static void spread_attr() {
  cudaFuncSetAttribute(spread_kernel<P, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<P, 1>());
  cudaFuncSetAttribute(spread_kernel<P, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<P, 2>());
  cudaFuncSetAttribute(spread_kernel<P, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<P, 4>());
}

void spread_prepare() {
  spread_attr<2>();
  spread_attr<4>();
  spread_attr<6>();
  spread_attr<8>();
}

static int sm_count() {
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
      nsm = v;
    else
      nsm = 148;
  }
  return nsm;
}

int launch_spread(const Geom &g, const Spline &S, const int *cell_start, const uint32_t *keys_sorted,
                  const float4 *rec_sorted, float *grid, cudaStream_t st) {
  static_assert((1 << kSpreadZShift) % SP_TZ == 0, "a brick's z range lies within one bucket");
  SpArgs A{};
  A.g = g;
  A.cs = cell_start;
  const long nb = sort_buckets(g, kSpreadZShift);
  A.head = reinterpret_cast<const uint32_t *>(cell_start) + nb + 3;  // layout of cell_count_words
  A.tail = A.head + nb;
  A.keys = keys_sorted;
  A.rec = rec_sorted;
  A.grid = grid;
  A.ntx = (g.K0 + SP_TX - 1) / SP_TX;
  A.nty = (g.K1 + SP_TY - 1) / SP_TY;
  A.ntz = (g.K2 + SP_TZ - 1) / SP_TZ;
  A.nbricks = A.ntx * A.nty * A.ntz;
  A.nzb = (g.K2 + (1 << kSpreadZShift) - 1) >> kSpreadZShift;
  A.nb = nb;
  A.K2d = FastDiv((uint32_t)g.K2);
  // Split a brick's atoms over more warps while the bricks alone would not
  // fill the SMs (SP_MIN_CTAS CTAs of 4 warps resident per SM).
  const long want = (long)sm_count() * SP_WARPS * SP_MIN_CTAS;
  int nsplit = 1;
  while (nsplit < SP_WARPS && (long)A.nbricks * nsplit < want) nsplit *= 2;
  switch (g.order) {
    case 2: spread_p<2>(A, nsplit, S, st); break;
    case 4: spread_p<4>(A, nsplit, S, st); break;
    case 6: spread_p<6>(A, nsplit, S, st); break;
    case 8: spread_p<8>(A, nsplit, S, st); break;
    default: return 0;
  }
  return 1;
}

}  // namespace spme
