// K2: B-spline charge spreading (SFac::operator() + accum_spline,
// sfac.cpp:113-124,141-168).
//
// Owner-computes, like the reference's accum_spline: every grid point has
// exactly one writer, which adds the contributions of the atoms in its
// order^3 neighbouring cells in a fixed order.  No atomics, so the grid is
// bit-for-bit reproducible.
//
// Blocking: a warp owns an 8 x 8 x 32 brick of grid points in registers.
// Lane (lx, ly) holds the two neighbouring columns x = 2 lx, 2 lx + 1 at
// y = ly, 32 z points each, as 32 packed FP32 pairs, so that one packed FMA
// (fma.rn.f32x2) adds an atom's z tap to both columns.  The atoms of the
// brick's halo (the cells whose stencils reach it) are the sorted atoms of
// (x, y) cell rows, found through the bucket offsets of the cell sort (runs
// of 32 z cells per row) and trimmed to the halo's z cells by a search on the
// sorted keys.  They are staged 32 at a time, one per lane: the order-p
// B-spline taps of the three fractions (the charge folded into x), the z taps
// as duplicated pairs ready for the packed FMA.  A branch-free pass then
// forms each lane's two column weights wx * wy for every staged atom (a tap
// index outside [0, p) weighs zero).  The walk goes window case by window
// case -- the place of the atom's z taps in the brick, the same for every
// lane -- in a compile-time unrolled chain: each case present in the chunk
// takes its atoms from a warp ballot and adds them with p packed FMAs into
// fixed registers, so there is no indirect jump and no divergent branch.
// Small grids split one brick's atoms over 2 or 4 warps (equal contiguous
// shares, summed in warp order through shared memory: still a fixed order).
#include "spme_kernels.hpp"

namespace spme {

constexpr int SP_TX = 8, SP_TY = 8, SP_TZ = 32;  // brick of one warp
constexpr int SP_WARPS = 4;                     // warps per CTA
constexpr int SP_MAXC = SP_TZ + kMaxOrder - 1;  // window cases of the largest order

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
__device__ __forceinline__ f2r fmul2(f2r a, f2r b) {
  f2r d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

template <int P>
struct SpCfg {
  static constexpr int H = P / 2;
  // halo cell rows of a brick: cells [x0 - H, x0 + TX - 2 + H] (RX of them)
  static constexpr int RX = SP_TX + P - 1, RY = SP_TY + P - 1, NR = RX * RY;
  static constexpr int NC = SP_TZ + P - 1;  // window cases: first z tap rz in [1 - P, TZ - 1]
  static constexpr int ZL = (P + 1) / 2 * 2;  // z pairs per atom (even: rows stay 16-byte aligned)
};

// Shared memory of one warp: the staged atoms during the walk, its partial
// brick (64 x 33 floats) for the final sum.
template <int P>
struct SpStage {
  using C = SpCfg<P>;
  f2r zp[32][C::ZL];   // (wz[t], wz[t]), t < P: weight of z = rz + t
  f2r wxc[32][P + 1];  // (w[j - 1], w[j]), j = 0..P, of the x taps (charge included; w[-1] = w[P] = 0)
  float wyc[32][9];    // y taps (odd row stride: conflict-free staging stores)
  int2 off[32];        // (P - 1 - rx, P - 1 - ry): tap index of column 0 / row 0 of the brick
  f2r wxy[32][32];     // [atom][lane]: the lane's two column weights wx * wy
};
template <int P>
struct SpGroup {  // per brick: the halo rows' atom ranges of one z piece
  int start[SpCfg<P>::NR];
  int pref[SpCfg<P>::NR + 1];
};
template <int P>
constexpr size_t sp_stage_bytes() {
  return sizeof(SpStage<P>) > 64 * 33 * 4 ? sizeof(SpStage<P>) : 64 * 33 * 4;
}
template <int P>
constexpr size_t sp_smem_bytes() {
  return SP_WARPS * (sp_stage_bytes<P>() + sizeof(SpGroup<P>));
}

// acc[z] += wxy * zp[t] for the taps t whose z = C - (P - 1) + t lies in the
// brick (all indices compile-time).
template <int P, int C>
__device__ __forceinline__ void sp_taps(f2r (&acc)[SP_TZ], f2r wxy, const f2r (&zp)[SpCfg<P>::ZL]) {
#pragma unroll
  for (int t = 0; t < P; t++) {
    const int z = C - (P - 1) + t;
    if (z >= 0 && z < SP_TZ) acc[z] = ffma2(wxy, zp[t], acc[z]);
  }
}

// The walk over one staged chunk, window case by window case: case C (all
// compile-time, so every accumulator index is fixed) takes the chunk's atoms
// whose first z tap is C - (P - 1), in lane order, from a warp ballot.  No
// indirect jump: a case absent from the chunk costs one uniform test.
template <int P, int C>
__device__ __forceinline__ void sp_walk(f2r (&acc)[SP_TZ], const SpStage<P> &st, int lane, int mycase,
                                        uint32_t plo, uint32_t phi) {
  if constexpr (C < SpCfg<P>::NC) {
    const uint32_t bit = C < 32 ? (plo >> (C & 31)) : (phi >> (C & 31));
    if (bit & 1u) {
      uint32_t am = __ballot_sync(0xffffffffu, mycase == C);
      while (am) {
        const int a = __ffs(am) - 1;
        am &= am - 1u;
        const f2r wxy = st.wxy[a][lane];
        f2r zp[SpCfg<P>::ZL];
#pragma unroll
        for (int v = 0; v < SpCfg<P>::ZL / 2; v++) {
          const ulonglong2 q = *reinterpret_cast<const ulonglong2 *>(&st.zp[a][2 * v]);
          zp[2 * v] = q.x;
          zp[2 * v + 1] = q.y;
        }
        sp_taps<P, C>(acc, wxy, zp);
      }
    }
    sp_walk<P, C + 1>(acc, st, lane, mycase, plo, phi);
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

struct SpArgs {
  Geom g;
  const int *cs;          // bucket offsets (runs of 2^zshift z cells per row)
  const uint32_t *keys;   // sorted cell keys
  const float4 *rec;      // sorted (fx, fy, fz, q)
  float *grid;
  int ntx, nty, ntz, nbricks;
  int nzb, zshift;
  FastDiv K2d;
};

template <int P, int NS>
__global__ void __launch_bounds__(SP_WARPS * 32, 4) spread_kernel(SpArgs A, Spline S) {
  using C = SpCfg<P>;
  constexpr int H = C::H, RY = C::RY, NR = C::NR;
  extern __shared__ __align__(16) unsigned char sp_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int nsplit = NS;
  const int group = warp / nsplit, member = warp % nsplit;
  SpStage<P> &st = *reinterpret_cast<SpStage<P> *>(sp_smem + warp * sp_stage_bytes<P>());
  SpGroup<P> &gr = *reinterpret_cast<SpGroup<P> *>(sp_smem + SP_WARPS * sp_stage_bytes<P>() +
                                                   group * sizeof(SpGroup<P>));
  const long brick = (long)blockIdx.x * (SP_WARPS / nsplit) + group;
  if (brick >= A.nbricks) return;  // the whole group leaves together
  const Geom &g = A.g;
  const int K0 = g.K0, K1 = g.K1, K2 = g.K2;
  const int tz = (int)(brick % A.ntz), ty = (int)((brick / A.ntz) % A.nty), tx = (int)(brick / ((long)A.ntz * A.nty));
  const int x0 = tx * SP_TX, y0 = ty * SP_TY, z0 = tz * SP_TZ;
  const int lx = lane & 3, ly = lane >> 2;
  const int gt = member * 32 + lane, gn = 32 * nsplit;  // thread index and size of the group

  f2r acc[SP_TZ];
#pragma unroll
  for (int z = 0; z < SP_TZ; z++) acc[z] = 0ull;

  const uint32_t zmask = (1u << A.zshift) - 1u;
  // extended z cells whose stencils reach [z0, z0 + TZ): [z0 - H, z0 + TZ + H - 2],
  // walked in pieces that do not cross the periodic boundary
  const int ez_lo = z0 - H, ez_hi = z0 + SP_TZ + H - 2;
  for (int ezs = ez_lo; ezs <= ez_hi;) {
    const int n2a = imod(ezs, K2);
    const int len = min(ez_hi - ezs + 1, K2 - n2a);
    group_sync<NS>(group);  // the previous piece's ranges are no longer read
    for (int r = gt; r < NR; r += gn) {
      const int ex = x0 - H + r / RY, ey = y0 - H + r % RY;
      const int row = imod(ex, K0) * K1 + imod(ey, K1);
      const int b0 = row * A.nzb + (n2a >> A.zshift), b1 = row * A.nzb + ((n2a + len - 1) >> A.zshift);
      int lo = __ldg(A.cs + b0), hi = __ldg(A.cs + b1 + 1);
      const uint32_t kbase = (uint32_t)row * (uint32_t)K2;
      // trim the partial first and last buckets to cells [n2a, n2a + len)
      if (n2a & zmask) lo = keys_lower_bound(A.keys, lo, __ldg(A.cs + b0 + 1), kbase + n2a);
      if (((n2a + len) & zmask) && n2a + len < K2)
        hi = keys_lower_bound(A.keys, __ldg(A.cs + b1), hi, kbase + n2a + len);
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
    const int w_lo = (int)((long)total * member / nsplit), w_hi = (int)((long)total * (member + 1) / nsplit);
    for (int chunk = w_lo; chunk < w_hi; chunk += 32) {
      const int t = chunk + lane;
      int mycase = -1;  // window case of this lane's staged atom (-1: none)
      if (t < w_hi) {
        int lo = 0, hi = NR - 1;  // largest r with pref[r] <= t
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (gr.pref[mid] <= t) lo = mid; else hi = mid - 1;
        }
        const int a = gr.start[lo] + (t - gr.pref[lo]);
        const float4 u = __ldg(A.rec + a);
        uint32_t qk, n2;
        A.K2d.divmod(__ldg(A.keys + a), qk, n2);
        const int rx = lo / RY, ry = lo % RY;
        // tap i of each axis: the weight of point first + i, M(f + P - 1 - i);
        // stored as soon as it is formed (the 64 accumulator registers stay live)
        float prev = 0.f;
#pragma unroll
        for (int i = 0; i < P; i++) {
          const float wx = u.w * bspl_eval(S, P, u.x, P - 1 - i);
          st.wxc[lane][i] = pack2(prev, wx);
          prev = wx;
          st.wyc[lane][i] = bspl_eval(S, P, u.y, P - 1 - i);
          const float wz = bspl_eval(S, P, u.z, P - 1 - i);
          st.zp[lane][i] = pack2(wz, wz);
        }
        st.wxc[lane][P] = pack2(prev, 0.f);
        st.off[lane] = make_int2(P - 1 - rx, P - 1 - ry);
        mycase = (int)n2 + zoff + P - 1;  // in [0, NC): first z tap rz = mycase - (P - 1)
      }
      __syncwarp();
      const int na = min(32, w_hi - chunk);
      // this lane's column weights for every staged atom (branch-free pass):
      // columns 2 lx, 2 lx + 1 take x taps ix, ix + 1 = pair ix + 1 of wxc,
      // row ly takes y tap iy; taps outside [0, P) weigh zero
      for (int a = 0; a < na; a++) {
        const int2 o = st.off[a];
        const int jx = o.x + 2 * lx + 1, iy = o.y + ly;
        const f2r xp = ((unsigned)jx <= (unsigned)P) ? st.wxc[a][jx] : 0ull;
        const float wy = ((unsigned)iy < (unsigned)P) ? st.wyc[a][iy] : 0.f;
        st.wxy[a][lane] = fmul2(xp, pack2(wy, wy));
      }
      const uint32_t plo = __reduce_or_sync(0xffffffffu, (mycase >= 0 && mycase < 32) ? 1u << mycase : 0u);
      const uint32_t phi = __reduce_or_sync(0xffffffffu, mycase >= 32 ? 1u << (mycase - 32) : 0u);
      __syncwarp();
      sp_walk<P, 0>(acc, st, lane, mycase, plo, phi);
      __syncwarp();  // the next chunk's staging overwrites these atoms
    }
    ezs += len;
  }

  // partial bricks to shared memory (over the staging rows), summed over the
  // group's warps in warp order, stored with consecutive threads on
  // consecutive z (coalesced)
  group_sync<NS>(group);
  float *part = reinterpret_cast<float *>(&st);  // [k * 32 + z][33]: column 2 lx + k of lane
#pragma unroll
  for (int z = 0; z < SP_TZ; z++) {
    float v0, v1;
    unpack2(acc[z], v0, v1);
    part[z * 33 + lane] = v0;
    part[(32 + z) * 33 + lane] = v1;
  }
  group_sync<NS>(group);
  const float *gpart = reinterpret_cast<const float *>(sp_smem + (size_t)group * nsplit * sp_stage_bytes<P>());
  const size_t mstride = sp_stage_bytes<P>() / sizeof(float);
  for (int p = gt; p < SP_TX * SP_TY * SP_TZ; p += gn) {
    const int z = p & 31, col = p >> 5;
    const int xr = col >> 3, yr = col & 7;
    const int src = ((xr & 1) * 32 + z) * 33 + (xr >> 1) + 4 * yr;
    float v = gpart[src];
    for (int m = 1; m < nsplit; m++) v += gpart[m * mstride + src];
    const int gx = x0 + xr, gy = y0 + yr, gz = z0 + z;
    if (gx < K0 && gy < K1 && gz < K2) A.grid[((long)gx * K1 + gy) * K2 + gz] = v;
  }
}

template <int P, int NS>
static void spread_ps(const SpArgs &A, const Spline &S, cudaStream_t st) {
  constexpr int per_cta = SP_WARPS / NS;
  const long ctas = (A.nbricks + per_cta - 1) / per_cta;
  spread_kernel<P, NS><<<(unsigned)ctas, SP_WARPS * 32, sp_smem_bytes<P>(), st>>>(A, S);
}

template <int P>
static void spread_p(const SpArgs &A, int nsplit, const Spline &S, cudaStream_t st) {
  if (nsplit == 1) spread_ps<P, 1>(A, S, st);
  else if (nsplit == 2) spread_ps<P, 2>(A, S, st);
  else spread_ps<P, 4>(A, S, st);
}

template <int P>
static void spread_attr() {
  cudaFuncSetAttribute(spread_kernel<P, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<P>());
  cudaFuncSetAttribute(spread_kernel<P, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<P>());
  cudaFuncSetAttribute(spread_kernel<P, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<P>());
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
  SpArgs A{};
  A.g = g;
  A.cs = cell_start;
  A.keys = keys_sorted;
  A.rec = rec_sorted;
  A.grid = grid;
  A.ntx = (g.K0 + SP_TX - 1) / SP_TX;
  A.nty = (g.K1 + SP_TY - 1) / SP_TY;
  A.ntz = (g.K2 + SP_TZ - 1) / SP_TZ;
  A.nbricks = A.ntx * A.nty * A.ntz;
  A.zshift = kSpreadZShift;
  A.nzb = (g.K2 + (1 << kSpreadZShift) - 1) >> kSpreadZShift;
  A.K2d = FastDiv((uint32_t)g.K2);
  // Split a brick's atoms over more warps while the bricks alone would not
  // fill the SMs (4 CTAs of 4 warps resident per SM).
  const long want = (long)sm_count() * 16;
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
