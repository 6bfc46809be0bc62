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
// B-spline weights of the three fractions (the charge folded into x) are
// written to shared memory as zero-padded rows, so that every lane reads its
// own column's weight at a per-atom offset without a range test; the z taps
// are stored as duplicated pairs, ready for the packed FMA.  The walk then
// costs per atom: one broadcast load of its offsets and window case, the
// lane's x-pair and y weights, one packed multiply, the z taps, and one
// jump (the window's place in the brick is the same for every lane, so it
// selects an unrolled code path, not a divergent branch) into p packed
// FMAs.  Small grids split one brick's atoms over 2 or 4 warps (equal
// contiguous shares, summed in warp order through shared memory: still a
// fixed order).
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
  // Tap rows: tap i of an atom sits at [OFF + i]; a lane reads [off + col]
  // with off = OFF + P - 1 - (the atom's halo row), which stays in [1, P + 14].
  static constexpr int OFF = 8;
  static constexpr int WL = (P + 15) | 1;
  static constexpr int ZL = (P + 1) / 2 * 2;  // z pairs per atom (even: rows stay 16-byte aligned)
};

// Shared memory of one warp: the staged atoms during the walk, its partial
// brick (64 x 33 floats) for the final sum.
template <int P>
struct SpStage {
  using C = SpCfg<P>;
  f2r zp[32][C::ZL];   // (wz[t], wz[t]), t < P: weight of z = rz + t
  f2r wxp[32][C::WL];  // (w[j], w[j + 1]) of the zero-padded x taps, charge included
  f2r wyd[32][C::WL];  // (w[j], w[j]) of the zero-padded y taps
  int4 meta[32];       // x pair offset, y offset, window case
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

#define SPC(C)                                                     \
  case C:                                                          \
    if constexpr (C < SpCfg<P>::NC) sp_taps<P, C>(acc, wxy, zp);   \
    break;

template <int P>
__device__ __forceinline__ void sp_dispatch(int c, f2r (&acc)[SP_TZ], f2r wxy, const f2r (&zp)[SpCfg<P>::ZL]) {
  switch (c) {
    SPC(0) SPC(1) SPC(2) SPC(3) SPC(4) SPC(5) SPC(6) SPC(7) SPC(8) SPC(9)
    SPC(10) SPC(11) SPC(12) SPC(13) SPC(14) SPC(15) SPC(16) SPC(17) SPC(18) SPC(19)
    SPC(20) SPC(21) SPC(22) SPC(23) SPC(24) SPC(25) SPC(26) SPC(27) SPC(28) SPC(29)
    SPC(30) SPC(31) SPC(32) SPC(33) SPC(34) SPC(35) SPC(36) SPC(37) SPC(38)
    default: break;
  }
}
#undef SPC
static_assert(SP_MAXC <= 39, "window cases");

// Barrier of the nsplit warps that share one brick (named barrier 1 + group).
__device__ __forceinline__ void group_sync(int group, int nsplit) {
  if (nsplit == 1) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + group), "r"(32 * nsplit) : "memory");
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
  int ntx, nty, ntz, nbricks, nsplit;
  int nzb, zshift;
  FastDiv K2d;
};

template <int P>
__global__ void __launch_bounds__(SP_WARPS * 32, 4) spread_kernel(SpArgs A, Spline S) {
  using C = SpCfg<P>;
  constexpr int H = C::H, RY = C::RY, NR = C::NR, WL = C::WL, OFF = C::OFF;
  extern __shared__ __align__(16) unsigned char sp_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nsplit = A.nsplit;
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

  // zero the padded tap rows once (staging overwrites only the tap positions;
  // wxp and wyd are adjacent)
  {
    f2r *p = &st.wxp[0][0];
    for (int i = lane; i < 2 * 32 * WL; i += 32) p[i] = 0ull;
  }
  __syncwarp();

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
    group_sync(group, nsplit);  // the previous piece's ranges are no longer read
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
    group_sync(group, nsplit);
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
    group_sync(group, nsplit);
    const int total = gr.pref[NR];
    const int zoff = ezs - n2a + 1 - H - z0;  // first z tap of an atom in stored cell n2: n2 + zoff
    const int w_lo = (int)((long)total * member / nsplit), w_hi = (int)((long)total * (member + 1) / nsplit);
    for (int chunk = w_lo; chunk < w_hi; chunk += 32) {
      const int t = chunk + lane;
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
          st.wxp[lane][OFF - 1 + i] = pack2(prev, wx);
          prev = wx;
          const float wy = bspl_eval(S, P, u.y, P - 1 - i);
          st.wyd[lane][OFF + i] = pack2(wy, wy);
          const float wz = bspl_eval(S, P, u.z, P - 1 - i);
          st.zp[lane][i] = pack2(wz, wz);
        }
        st.wxp[lane][OFF + P - 1] = pack2(prev, 0.f);
        st.meta[lane] = make_int4(lane * WL + OFF + P - 1 - rx, lane * WL + OFF + P - 1 - ry,
                                  (int)n2 + zoff + P - 1, 0);
      }
      __syncwarp();
      const int na = min(32, w_hi - chunk);
      const f2r *wxl = &st.wxp[0][0] + 2 * lx;
      const f2r *wyl = &st.wyd[0][0] + ly;
      for (int a = 0; a < na; a++) {
        const int4 m = st.meta[a];
        const f2r wxy = fmul2(wxl[m.x], wyl[m.y]);
        f2r zp[C::ZL];
#pragma unroll
        for (int v = 0; v < C::ZL / 2; v++) {
          const ulonglong2 q = *reinterpret_cast<const ulonglong2 *>(&st.zp[a][2 * v]);
          zp[2 * v] = q.x;
          zp[2 * v + 1] = q.y;
        }
        sp_dispatch<P>(m.z, acc, wxy, zp);
      }
      __syncwarp();  // the next chunk's staging overwrites these atoms
    }
    ezs += len;
  }

  // partial bricks to shared memory (over the staging rows), summed over the
  // group's warps in warp order, stored with consecutive threads on
  // consecutive z (coalesced)
  group_sync(group, nsplit);
  float *part = reinterpret_cast<float *>(&st);  // [k * 32 + z][33]: column 2 lx + k of lane
#pragma unroll
  for (int z = 0; z < SP_TZ; z++) {
    float v0, v1;
    unpack2(acc[z], v0, v1);
    part[z * 33 + lane] = v0;
    part[(32 + z) * 33 + lane] = v1;
  }
  group_sync(group, nsplit);
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

template <int P>
static void spread_p(const SpArgs &A, const Spline &S, cudaStream_t st) {
  const int per_cta = SP_WARPS / A.nsplit;
  const long ctas = (A.nbricks + per_cta - 1) / per_cta;
  spread_kernel<P><<<(unsigned)ctas, SP_WARPS * 32, sp_smem_bytes<P>(), st>>>(A, S);
}

void spread_prepare() {
  cudaFuncSetAttribute(spread_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<2>());
  cudaFuncSetAttribute(spread_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<4>());
  cudaFuncSetAttribute(spread_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<6>());
  cudaFuncSetAttribute(spread_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sp_smem_bytes<8>());
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
  A.nsplit = 1;
  while (A.nsplit < SP_WARPS && (long)A.nbricks * A.nsplit < want) A.nsplit *= 2;
  switch (g.order) {
    case 2: spread_p<2>(A, S, st); break;
    case 4: spread_p<4>(A, S, st); break;
    case 6: spread_p<6>(A, S, st); break;
    case 8: spread_p<8>(A, S, st); break;
    default: return 0;
  }
  return 1;
}

}  // namespace spme
