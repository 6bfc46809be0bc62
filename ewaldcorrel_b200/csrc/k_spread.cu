// K2: B-spline charge spreading (SFac::operator() + accum_spline,
// sfac.cpp:113-124,141-168).
//
// Owner-computes, like the reference's accum_spline: every grid point has
// exactly one writer, which adds the contributions of the atoms in its
// order^3 neighbouring cells in a fixed order.  No atomics, so the grid is
// bit-for-bit reproducible.
//
// Blocking: one CTA owns a 4 x 8 x 32 brick of grid points; in each of its
// four warps, lane (cx, cy) holds the 32 points of its (x, y) column in
// registers.  The atoms of the brick's halo (the cells whose stencils reach
// it) are found through the per-cell offsets of the sorted order; the warps
// split them into equal contiguous shares, staged 32 at a time: each lane
// stages one atom in shared memory (cell offsets relative to the brick, the
// order-p B-spline weights of its three fractions, the charge folded into the
// x weights, the z weights as a window aligned to 4).  The warp then walks
// the staged atoms in order: each lane forms its column weight wx*wy and adds
// it times the z window to the registers the window covers -- the window's
// place is the same for every lane, so it selects one unrolled code path (a
// jump table of ten), not a divergent branch.  Finally the four partial
// bricks are summed in warp order through shared memory and stored with
// lane = z (coalesced).
#include "spme_kernels.hpp"

namespace spme {

constexpr int SP_TX = 4, SP_TY = 8, SP_TZ = 32;
constexpr int SP_WARPS = 4;

// acc[Z + t] += w * wz[t] for the t with 0 <= Z + t < TZ (all compile-time).
// z weights of a staged atom as a window of NW floats starting at the
// multiple of 4 at or below its first z offset rz (zero outside the P taps):
// the window covers rz .. rz + P - 1 for P <= NW - 3.
template <int P>
struct ZWin {
  static constexpr int NW = (P + 3 + 3) / 4 * 4;  // 8 for P <= 5, 12 for P <= 9
  static constexpr int NV = NW / 4;                // float4 loads
};

// acc[4 G + t] += w * win[t] for the t with 0 <= 4 G + t < TZ (compile time).
template <int NW, int G>
__device__ __forceinline__ void add_win(float (&acc)[SP_TZ], float w, const float (&win)[NW]) {
#pragma unroll
  for (int t = 0; t < NW; t++)
    if (4 * G + t >= 0 && 4 * G + t < SP_TZ) acc[4 * G + t] = fmaf(w, win[t], acc[4 * G + t]);
}

#define SP_CASE(G) \
  case G:          \
    add_win<NW, G>(acc, w, win); \
    break;

// Dispatch on the warp-uniform window group g4 = floor(rz / 4) in [-2, 7]
// (rz >= -(P-1) >= -7): ten code paths of NW fixed-register FMAs each.
template <int NW>
__device__ __forceinline__ void z_dispatch_win(int g4, float (&acc)[SP_TZ], float w, const float (&win)[NW]) {
  switch (g4) {
    SP_CASE(-2) SP_CASE(-1) SP_CASE(0) SP_CASE(1) SP_CASE(2) SP_CASE(3) SP_CASE(4) SP_CASE(5) SP_CASE(6) SP_CASE(7)
    default: break;
  }
}
#undef SP_CASE

template <int P>
struct SpreadSmem {
  static constexpr int H = P / 2;
  static constexpr int RX = SP_TX + P - 1, RY = SP_TY + P - 1, NR = RX * RY;
  // Staged atom, read by every lane in the walk:
  //   rel: rx | ry << 8 | (g4 + 64) << 16 (brick-relative row and window group);
  //   zw: the z-weight window (ZWin) as float4s -- broadcast loads;
  //   wx: q*M(fx+i) at [3 + i], zero elsewhere, so lane cx reads [rx - cx + 3]
  //       with no range test (rx - cx in [-3, RX - 1]);
  //   wy: M(fy+j) at [7 + j], zero elsewhere, read at [ry - cy + 7].
  // The zero entries are written once per CTA; staging writes only the P
  // weights of each axis.  Odd row strides keep the lane-per-atom staging
  // stores free of bank conflicts.
  static constexpr int NZ4 = ZWin<P>::NV;
  static constexpr int WXS = (P + 6) | 1, WYS = (P + 14) | 1;
  int start[NR];                         // first sorted atom of each halo row segment
  int pref[NR + 1];                      // prefix sums of the row segment counts
  union {
    struct {
      float4 zq[SP_WARPS][32][NZ4];
      int rel[SP_WARPS][32];
      float wx[SP_WARPS][32][WXS];
      float wy[SP_WARPS][32][WYS];
    } st;                                // staging (walk phase)
    float part[SP_WARPS][SP_TZ][33];     // per-warp partial bricks for the final sum
  };
};

// One CTA per 4 x 8 x 32 brick; its 4 warps split the brick's atoms into
// equal contiguous shares (staged 32 at a time) and keep private register
// accumulators, summed in warp order at the end (fixed order: deterministic).
template <int P>
__global__ void __launch_bounds__(SP_WARPS * 32, 8) spread_reg_kernel(Geom g, Spline S, const int *__restrict__ cs,
                                                                  const uint32_t *__restrict__ keys,
                                                                  const float4 *__restrict__ rec,
                                                                  float *__restrict__ grid, int ntx, int nty,
                                                                  int ntz, FastDiv K2d) {
  using SM = SpreadSmem<P>;
  constexpr int H = SM::H, RY = SM::RY, NR = SM::NR, NZ4 = SM::NZ4;
  __shared__ SM s;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long tile = blockIdx.x;
  const int tz = (int)(tile % ntz), ty = (int)((tile / ntz) % nty), tx = (int)(tile / ((long)ntz * nty));
  const int x0 = tx * SP_TX, y0 = ty * SP_TY, z0 = tz * SP_TZ;
  const int cx = lane >> 3, cy = lane & 7;
  const int K0 = g.K0, K1 = g.K1, K2 = g.K2;

  // zero the padded weight rows once (the staged weights overwrite only the
  // fixed non-zero positions)
  for (int i = threadIdx.x; i < SP_WARPS * 32 * SM::WXS; i += SP_WARPS * 32) (&s.st.wx[0][0][0])[i] = 0.f;
  for (int i = threadIdx.x; i < SP_WARPS * 32 * SM::WYS; i += SP_WARPS * 32) (&s.st.wy[0][0][0])[i] = 0.f;

  float acc[SP_TZ];
#pragma unroll
  for (int z = 0; z < SP_TZ; z++) acc[z] = 0.f;

  // extended z cells whose stencils reach [z0, z0 + TZ): [z0 - H, z0 + TZ + H - 2]
  const int ez_lo = z0 - H, ez_hi = z0 + SP_TZ + H - 2;
  for (int ezs = ez_lo; ezs <= ez_hi;) {
    const int n2a = imod(ezs, K2);
    const int len = min(ez_hi - ezs + 1, K2 - n2a);
    __syncthreads();  // previous segment's ranges are no longer read
    // atom ranges of the halo rows for cells [n2a, n2a + len)
    for (int r = threadIdx.x; r < NR; r += SP_WARPS * 32) {
      const int ex = x0 - H + r / RY, ey = y0 - H + r % RY;
      const long base = (long)(imod(ex, K0) * K1 + imod(ey, K1)) * K2 + n2a;
      const int a0 = __ldg(cs + base), a1 = __ldg(cs + base + len);
      s.start[r] = a0;
      s.pref[r + 1] = a1 - a0;
    }
    __syncthreads();
    if (warp == 0) {
      int running = 0;
      for (int c = 0; c < NR; c += 32) {
        const int r = c + lane;
        int v = (r < NR) ? s.pref[r + 1] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int u = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += u;
        }
        if (r < NR) s.pref[r + 1] = running + v;
        running += __shfl_sync(0xffffffffu, v, 31);
      }
      if (lane == 0) s.pref[0] = 0;
    }
    __syncthreads();
    const int total = s.pref[NR];
    const int zoff = ezs + H - (P - 1) - z0 - n2a;  // rz = n2 + zoff
    // each warp takes an equal contiguous share of the segment's atoms,
    // staged 32 at a time
    const int w_lo = (int)((long)total * warp / SP_WARPS), w_hi = (int)((long)total * (warp + 1) / SP_WARPS);
    for (int chunk = w_lo; chunk < w_hi; chunk += 32) {
      const int t = chunk + lane;
      if (t < w_hi) {
        int lo = 0, hi = NR - 1;  // largest r with pref[r] <= t
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s.pref[mid] <= t) lo = mid; else hi = mid - 1;
        }
        const int a = s.start[lo] + (t - s.pref[lo]);
        const float4 u = __ldg(rec + a);
        uint32_t qk, n2;
        K2d.divmod(__ldg(keys + a), qk, n2);
        const int rx = lo / RY, ry = lo % RY;
        const int rz = (int)n2 + zoff;
        const int g4 = rz >> 2;  // floor(rz / 4)
        s.st.rel[warp][lane] = rx | (ry << 8) | ((g4 + 64) << 16);
        float zt[P];
#pragma unroll
        for (int i = 0; i < P; i++) {
          s.st.wx[warp][lane][3 + i] = u.w * bspl_eval(S, P, u.x, i);
          s.st.wy[warp][lane][7 + i] = bspl_eval(S, P, u.y, i);
          zt[i] = bspl_eval(S, P, u.z, P - 1 - i);  // weight of z = rz + i
        }
        const int sh = rz - 4 * g4;  // 0..3: first tap's place in the window
        float zw[4 * NZ4];
#pragma unroll
        for (int t = 0; t < 4 * NZ4; t++) {
          float v = 0.f;
#pragma unroll
          for (int i = 0; i < P; i++) v = (t == sh + i) ? zt[i] : v;
          zw[t] = v;
        }
#pragma unroll
        for (int v = 0; v < NZ4; v++)
          s.st.zq[warp][lane][v] = make_float4(zw[4 * v], zw[4 * v + 1], zw[4 * v + 2], zw[4 * v + 3]);
      }
      __syncwarp();
      const int na = min(32, w_hi - chunk);
      const float *wxl = &s.st.wx[warp][0][3 - cx];
      const float *wyl = &s.st.wy[warp][0][7 - cy];
      for (int a = 0; a < na; a++) {
        float win[4 * NZ4];
#pragma unroll
        for (int v = 0; v < NZ4; v++) {
          const float4 q = s.st.zq[warp][a][v];
          win[4 * v] = q.x; win[4 * v + 1] = q.y; win[4 * v + 2] = q.z; win[4 * v + 3] = q.w;
        }
        const int rel = s.st.rel[warp][a];
        const int rx = rel & 0xff, ry = (rel >> 8) & 0xff, g4 = (rel >> 16) - 64;
        const float w = wxl[a * SM::WXS + rx] * wyl[a * SM::WYS + ry];
        z_dispatch_win<4 * NZ4>(g4, acc, w, win);
      }
      __syncwarp();
    }
    ezs += len;
  }

  // partial bricks to shared memory (over the staging arrays), then the
  // fixed-order sum over warps
  __syncthreads();
#pragma unroll
  for (int z = 0; z < SP_TZ; z++) s.part[warp][z][lane] = acc[z];
  __syncthreads();
  const int gz = z0 + lane;
  for (int c = warp; c < 32; c += SP_WARPS) {
    const int gx = x0 + (c >> 3), gy = y0 + (c & 7);
    float v = s.part[0][lane][c];
#pragma unroll
    for (int wp = 1; wp < SP_WARPS; wp++) v += s.part[wp][lane][c];
    if (gx < K0 && gy < K1 && gz < K2) grid[((long)gx * K1 + gy) * K2 + gz] = v;
  }
}

template <int P>
static void spread_p(const Geom &g, const Spline &S, const int *cs, const uint32_t *keys, const float4 *rec,
                     float *grid, cudaStream_t st) {
  const int ntx = (g.K0 + SP_TX - 1) / SP_TX, nty = (g.K1 + SP_TY - 1) / SP_TY, ntz = (g.K2 + SP_TZ - 1) / SP_TZ;
  const long tiles = (long)ntx * nty * ntz;
  spread_reg_kernel<P><<<(unsigned)tiles, SP_WARPS * 32, 0, st>>>(g, S, cs, keys, rec, grid, ntx, nty, ntz,
                                                                  FastDiv((uint32_t)g.K2));
}

int launch_spread(const Geom &g, const Spline &S, const int *cell_start, const uint32_t *keys_sorted,
                  const float4 *rec_sorted, float *grid, cudaStream_t st) {
  switch (g.order) {
    case 2: spread_p<2>(g, S, cell_start, keys_sorted, rec_sorted, grid, st); break;
    case 4: spread_p<4>(g, S, cell_start, keys_sorted, rec_sorted, grid, st); break;
    case 6: spread_p<6>(g, S, cell_start, keys_sorted, rec_sorted, grid, st); break;
    case 8: spread_p<8>(g, S, cell_start, keys_sorted, rec_sorted, grid, st); break;
    default: return 0;
  }
  return 1;
}

}  // namespace spme
