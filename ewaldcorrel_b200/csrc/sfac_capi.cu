// Host side of libsfac.so: the reference's C interface (sfac.hpp:194-211)
// implemented over the sm_100a kernels.  Handle state, argument checks and
// the state machine follow sfac.cpp; every computation on grids or atoms runs
// on the GPU.  No C++ exception crosses the C ABI: failures return NULL/0 and
// are recorded in the handle (sfac_last_error).
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sfac.h"
#include "spme_kernels.hpp"

using namespace spme;

namespace {
// NVTX range over a scope: names each stage and C-API call on a profiler's
// timeline (header-only NVTX; nearly free when no tool is attached).
struct Nvtx {
  explicit Nvtx(const char *name) { nvtxRangePushA(name); }
  ~Nvtx() { nvtxRangePop(); }
};
}  // namespace

namespace spme {

// > 0: the fail_alloc_in-th device allocation from now on fails (and the
// counter stops); 0: allocations go straight to cudaMalloc.
static std::atomic<int> fail_alloc_in{0};

cudaError_t device_malloc(void **p, size_t bytes) {
  int k = fail_alloc_in.load();
  while (k > 0 && !fail_alloc_in.compare_exchange_weak(k, k - 1)) {
  }
  if (k == 1) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

SPME_CHECK_READER(capi)

// Exercises the check machinery: a logical bound of 32 on a 64-float buffer,
// index 40 -- the check fails and skips the store, which would have stayed
// inside the allocation anyway.
__global__ void check_selftest_kernel(float *buf) {
  if (threadIdx.x == 0 && SPME_IN(40, 32, CK_SELFTEST)) buf[40] = 1.f;
}

}  // namespace spme

namespace {

struct Handle {
  int order = 0, K[3] = {0, 0, 0}, ldim = 0;
  long nreal = 0, nmodes = 0, ncell = 0;
  Geom geom{};            // grid constants + device address of the box constants
  CellConst hcell{};      // host copy of the current box constants
  double L[6] = {0, 0, 0, 0, 0, 0};  // current box [ax, by, cz, bx, cx, cy]
  CellConst *d_cell = nullptr;
  InfConst hic{};         // host copy of the device Ewald constants
  InfConst *d_ic = nullptr;
  Spline spline{};
  SplineNodes nodes{};
  int state = -1;  // -1: nothing computed, 0: structure factor, 1: potential grid
  int a_mode = 0;  // 0: no influence function, 1: host tables, 2: Ewald on device, 3: sampled radial function
  int ewald_src = 0;  // sfac_set_ewald: 0 pick by grid size, 2 always evaluate on the device (no table)
  Influence inf{};
  int device = 0;
  cudaStream_t stream = nullptr;      // stream all work is enqueued on
  cudaStream_t own_stream = nullptr;  // the handle's own stream
  cudaEvent_t ev_in = nullptr;
  cudaEvent_t ev_stage[7] = {};
  // device buffers
  float *d_real = nullptr;
  float2 *d_cplx = nullptr;
  double *d_iB[3] = {nullptr, nullptr, nullptr};
  float2 *d_tw[3] = {nullptr, nullptr, nullptr};
  FftPlan3 fft{};
  double *d_A = nullptr;  // 7 * nmodes (table mode)
  RowImg *d_rows = nullptr;  // K0*K1 row image tables (device Ewald mode)
  double *d_partials = nullptr, *d_red = nullptr, *d_ev = nullptr;
  int cap = 0;
  double *d_x = nullptr, *d_w = nullptr;
  SortBuffers sb{};
  int gcap = 0;
  double *d_gx = nullptr, *d_gw = nullptr, *d_gout = nullptr;
  int ccap = 0;
  double *d_cellp = nullptr;  // per-block partials of the cell adjoint
  // structure-factor analysis: sum of |S|^2 over frames, radial binning scratch
  double *d_sk = nullptr;
  long long sk_frames = 0;
  double *d_skpart = nullptr, *d_skres = nullptr;
  int sk_cap = 0;
  // cross-correlations of several densities: D stored S, D(D+1)/2 sums
  int xc_D = 0;
  long long xc_frames = 0;
  float2 *d_xcq = nullptr;
  double2 *d_xcc = nullptr;
  // real-space term: coarse cell sort and per-point records
  struct RealBufs {
    SortBuffers sb{};
    int cap = 0;
    long ncell = 0;
    double4 *rec = nullptr;
    double *x = nullptr, *w = nullptr, *dx = nullptr, *part = nullptr, *out = nullptr;
    float4 *tab = nullptr;  // erfcx table of the pair kernel
  } rs;
  // pipelined de2 / potl: copy-in and copy-out streams, per-chunk events
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_copied[8] = {}, ev_gathered[8] = {};
  int last_n = 0;
  // pinned host buffers
  double *h_S = nullptr;
  float *h_f = nullptr;
  double *h_red = nullptr;
  int err = 0;
  char errstr[256] = {0};
  long long launches = 0;
  // CUDA graph of the device solve, replayed while its key is unchanged
  unsigned long long version = 1;  // bumped by anything that changes kernel arguments
  bool use_graph = true;
  cudaGraphExec_t graph = nullptr;
  int graph_kernels = 0;
  struct Key {
    int n;
    const void *x, *w, *dx, *phi, *ev, *dEdL;
    cudaStream_t stream;
    unsigned long long version;
    bool operator==(const Key &o) const {
      return n == o.n && x == o.x && w == o.w && dx == o.dx && phi == o.phi && ev == o.ev && dEdL == o.dEdL &&
             stream == o.stream && version == o.version;
    }
  } gkey{};
};

Handle *H(void *p) { return reinterpret_cast<Handle *>(p); }

// Pipelined de2 / potl: at most kPipeChunks chunks of at least kPipeMinChunk
// points each.  Every chunk costs a handful of API calls on the host (copies,
// events, a launch), which smaller chunks do not repay; 8 chunks instead of 4
// shorten the pipeline's tail (the last chunk's gather and copy out): de2 at
// 1M points 0.995 vs 1.03 ms, potl 0.65 vs 0.69 ms.
constexpr int kPipeChunks = 8;
constexpr int kPipeMinChunk = 131072;

// Largest tabulated device Ewald influence function (A + 6 dA, FP64): a
// table that stays in L2 is cheaper to read than the images are to evaluate;
// a larger one streamed from HBM every solve is not.
constexpr size_t kEwaldTableMaxBytes = (size_t)64 << 20;  // stays resident in the 126 MB L2

bool check(Handle *h, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return true;
  if (h) {
    h->err = (int)e;
    snprintf(h->errstr, sizeof(h->errstr), "%s: %s", what, cudaGetErrorString(e));
    fprintf(stderr, "sfac: CUDA error in %s: %s\n", what, cudaGetErrorString(e));
  }
  return false;
}
#define CK(h, call) check((h), (call), #call)

bool launched(Handle *h, int n, const char *what) {
  h->launches += n;
  return check(h, cudaGetLastError(), what);
}

template <class T>
bool dalloc(Handle *h, T **p, size_t count) {
  *p = nullptr;
  return CK(h, device_malloc((void **)p, sizeof(T) * (count ? count : 1)));
}
template <class T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

bool check(Handle *h, cudaError_t e, const char *what);

// Cell(L) (sfac.hpp:37-52): host copy, then the device copy on the handle's
// stream (ordered before any later solve; kernel arguments do not change, so
// captured graphs stay valid).
bool set_cell(Handle *h, const double L[6]) {
  for (int i = 0; i < 6; i++) h->L[i] = L[i];
  h->hcell = make_cell(L);
  return check(h, cudaMemcpyAsync(h->d_cell, &h->hcell, sizeof(CellConst), cudaMemcpyHostToDevice, h->stream),
               "set_cell copy");
}

// Coefficients of the cardinal B-spline pieces: row j, column i holds the
// coefficient of t^(n-1-i) of M_n(t+j),
//   C(n-1,i)/(n-1)! * sum_{k=0..j} (-1)^k C(n,k) (j-k)^i
// (the explicit piecewise form that BSpline::mk_bspl_coeffs tabulates,
// sfac.hpp:81-109).  Evaluated in long double, stored FP32 for the kernels
// and as FP64 node values M_n(j) for the moduli.
void make_spline(int n, Spline &S, SplineNodes &nodes) {
  long double binom[kMaxOrder + 1][kMaxOrder + 1] = {};
  for (int a = 0; a <= kMaxOrder; a++) {
    binom[a][0] = 1;
    for (int b = 1; b <= a; b++) binom[a][b] = binom[a - 1][b - 1] + (b <= a - 1 ? binom[a - 1][b] : 0);
  }
  long double fact = 1;
  for (int k = 2; k < n; k++) fact *= k;
  memset(&S, 0, sizeof(S));
  memset(&nodes, 0, sizeof(nodes));
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      long double acc = 0;
      for (int k = 0; k <= j; k++) {
        long double pw = 1;
        for (int e = 0; e < i; e++) pw *= (long double)(j - k);
        acc += ((k & 1) ? -1 : 1) * binom[n][k] * pw;
      }
      const long double c = binom[n - 1][i] / fact * acc;
      S.c[j * n + i] = (float)c;
      if (i == n - 1) nodes.Mj[j] = (double)c;  // constant term: M_n(j)
    }
}

void free_real(Handle *h) {
  Handle::RealBufs &r = h->rs;
  for (int i = 0; i < 2; i++) {
    dfree(r.sb.keys[i]);
    dfree(r.sb.vals[i]);
  }
  dfree(r.sb.tmp);
  dfree(r.sb.tkeys);
  dfree(r.sb.rec);
  dfree(r.sb.rec_sorted);
  dfree(r.sb.hist);
  dfree(r.sb.cell_start);
  dfree(r.rec);
  dfree(r.x);
  dfree(r.w);
  dfree(r.dx);
  dfree(r.part);
  dfree(r.out);
  dfree(r.tab);
  r.cap = 0;
  r.ncell = 0;
}

// Buffers of the real-space term for n points on a coarse grid of ncell cells.
bool ensure_real(Handle *h, int n, long ncell) {
  Handle::RealBufs &r = h->rs;
  if (n <= r.cap && ncell == r.ncell && r.out) return true;
  const int cap = n > r.cap ? n + n / 2 + 64 : r.cap;
  free_real(h);
  bool ok = true;
  for (int i = 0; i < 2 && ok; i++) ok = dalloc(h, &r.sb.keys[i], cap) && dalloc(h, &r.sb.vals[i], cap);
  ok = ok && dalloc(h, &r.sb.tmp, cap) && dalloc(h, &r.sb.tkeys, cap) && dalloc(h, &r.sb.rec, cap) &&
       dalloc(h, &r.sb.rec_sorted, cap) &&
       dalloc(h, &r.sb.hist, cap) && dalloc(h, &r.sb.cell_start, cell_count_words(ncell)) &&
       dalloc(h, &r.rec, cap) && dalloc(h, &r.x, 3 * (size_t)cap) && dalloc(h, &r.w, cap) &&
       dalloc(h, &r.dx, 3 * (size_t)cap) && dalloc(h, &r.part, real_partial_words(cap)) && dalloc(h, &r.out, 16) &&
       dalloc(h, &r.tab, kRealTab);
  if (!ok) {
    free_real(h);
    return false;
  }
  r.cap = cap;
  r.ncell = ncell;
  return true;
}

void free_atoms(Handle *h) {
  dfree(h->d_x);
  dfree(h->d_w);
  for (int i = 0; i < 2; i++) {
    dfree(h->sb.keys[i]);
    dfree(h->sb.vals[i]);
  }
  dfree(h->sb.tmp);
  dfree(h->sb.tkeys);
  dfree(h->sb.rec);
  dfree(h->sb.rec_sorted);
  dfree(h->sb.hist);
  h->cap = 0;
}

bool ensure_atoms(Handle *h, int n) {
  if (n <= h->cap) return true;
  free_atoms(h);
  const int cap = n + n / 2 + 64;
  bool ok = dalloc(h, &h->d_x, 3 * (size_t)cap) && dalloc(h, &h->d_w, cap);
  for (int i = 0; i < 2; i++) ok = ok && dalloc(h, &h->sb.keys[i], cap) && dalloc(h, &h->sb.vals[i], cap);
  ok = ok && dalloc(h, &h->sb.tmp, cap) && dalloc(h, &h->sb.tkeys, cap) && dalloc(h, &h->sb.rec, cap) &&
       dalloc(h, &h->sb.rec_sorted, cap) &&
       dalloc(h, &h->sb.hist, cap);
  if (!ok) {
    free_atoms(h);
    return false;
  }
  h->cap = cap;
  h->version++;  // buffers moved: cached graphs are stale
  return true;
}

bool ensure_cellp(Handle *h, int n) {
  if (n <= h->ccap && h->d_cellp) return true;
  dfree(h->d_cellp);
  const int cap = n + n / 2 + 64;
  if (!dalloc(h, &h->d_cellp, gather_cell_words(cap))) {
    h->ccap = 0;
    return false;
  }
  h->ccap = cap;
  h->version++;
  return true;
}

bool ensure_gather(Handle *h, int n) {
  if (n <= h->gcap) return true;
  dfree(h->d_gx);
  dfree(h->d_gw);
  dfree(h->d_gout);
  const int cap = n + n / 2 + 64;
  if (!(dalloc(h, &h->d_gx, 3 * (size_t)cap) && dalloc(h, &h->d_gw, cap) &&
        dalloc(h, &h->d_gout, 3 * (size_t)cap))) {
    h->gcap = 0;
    return false;
  }
  h->gcap = cap;
  return true;
}

void destroy(Handle *h) {
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  dfree(h->d_real);
  dfree(h->d_cplx);
  for (int d = 0; d < 3; d++) {
    dfree(h->d_iB[d]);
    dfree(h->d_tw[d]);
  }
  dfree(h->d_A);
  dfree(h->d_rows);
  dfree(h->d_partials);
  dfree(h->d_ev);
  dfree(h->d_cell);
  dfree(h->d_ic);
  dfree(h->d_red);
  dfree(h->sb.cell_start);
  free_atoms(h);
  dfree(h->d_gx);
  dfree(h->d_gw);
  dfree(h->d_gout);
  dfree(h->d_cellp);
  if (h->h_S) cudaFreeHost(h->h_S);
  if (h->h_f) cudaFreeHost(h->h_f);
  if (h->h_red) cudaFreeHost(h->h_red);
  if (h->ev_in) cudaEventDestroy(h->ev_in);
  for (auto &e : h->ev_stage)
    if (e) cudaEventDestroy(e);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (int c = 0; c < 8; c++) {
    if (h->ev_copied[c]) cudaEventDestroy(h->ev_copied[c]);
    if (h->ev_gathered[c]) cudaEventDestroy(h->ev_gathered[c]);
  }
  free_real(h);
  dfree(h->d_sk);
  dfree(h->d_skpart);
  dfree(h->d_skres);
  dfree(h->d_xcq);
  dfree(h->d_xcc);
  if (h->s_in) cudaStreamDestroy(h->s_in);
  if (h->s_out) cudaStreamDestroy(h->s_out);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

bool sync(Handle *h) { return CK(h, cudaStreamSynchronize(h->stream)); }

}  // namespace

extern "C" {

void *sfac_ctor(double L[6], int K[3], int order) {
  if (order % 2 != 0 || order < 2 || order > kMaxOrder) {
    printf("Bad order: %d (must be even)\n", order);
    return nullptr;
  }
  if (K[0] < 1 || K[1] < 1 || K[2] < 1) {
    printf("Bad K: %d %d %d\n", K[0], K[1], K[2]);
    return nullptr;
  }
  const long ncell = (long)K[0] * K[1] * K[2];
  if (ncell >= 0x7fffffffL) {
    printf("Bad K: %d %d %d (grid too large)\n", K[0], K[1], K[2]);
    return nullptr;
  }
  int dev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1 || cudaGetDevice(&dev) != cudaSuccess) {
    printf("sfac_ctor: no CUDA device available\n");
    cudaGetLastError();
    return nullptr;
  }
  Handle *h = new (std::nothrow) Handle;
  if (!h) return nullptr;
  h->device = dev;
  h->order = order;
  for (int d = 0; d < 3; d++) h->K[d] = K[d];
  h->ldim = K[2] / 2 + 1;
  h->ncell = ncell;
  h->nreal = ncell;
  h->nmodes = (long)K[0] * K[1] * h->ldim;
  Geom &g = h->geom;
  g.K0 = K[0];
  g.K1 = K[1];
  g.K2 = K[2];
  g.ldim = h->ldim;
  g.order = order;
  make_spline(order, h->spline, h->nodes);
  fft_prepare_kernels();
  spread_prepare();
  if (const char *e = getenv("SFAC_NO_GRAPH")) h->use_graph = !(e[0] && e[0] != '0');
  if (const char *e = getenv("SFAC_ZY_MODE")) {
    const int v = atoi(e);
    if (v >= 0 && v <= 3) h->fft.zy_mode = v;
  }

  bool ok = CK(h, cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking)) &&
            CK(h, cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
  h->stream = h->own_stream;
  for (int i = 0; i < 7 && ok; i++) ok = CK(h, cudaEventCreate(&h->ev_stage[i]));
  ok = ok && dalloc(h, &h->d_real, h->nreal) && dalloc(h, &h->d_cplx, h->nmodes) &&
       dalloc(h, &h->d_partials,
              (size_t)(fft_x_blocks_max(K[1], K[2]) > kConvBlocks ? fft_x_blocks_max(K[1], K[2]) : kConvBlocks) *
                  kRedWords) &&
       dalloc(h, &h->d_red, kRedWords) && dalloc(h, &h->d_ev, kRedWords) && dalloc(h, &h->d_cell, 1) &&
       dalloc(h, &h->d_ic, 1) &&
       dalloc(h, &h->sb.cell_start, cell_count_words(sort_buckets(g, kSpreadZShift)));
  for (int d = 0; d < 3 && ok; d++) ok = dalloc(h, &h->d_iB[d], K[d]) && dalloc(h, &h->d_tw[d], K[d]);
  const size_t hf = (size_t)(2 * h->nmodes > h->nreal ? 2 * h->nmodes : h->nreal);
  ok = ok && CK(h, cudaMallocHost((void **)&h->h_S, sizeof(double) * 2 * h->nmodes)) &&
       CK(h, cudaMallocHost((void **)&h->h_f, sizeof(float) * hf)) &&
       CK(h, cudaMallocHost((void **)&h->h_red, sizeof(double) * kRedWords));
  if (ok) {
    g.cell = h->d_cell;
    ok = set_cell(h, L);
  }
  if (ok) {
    memset(h->h_S, 0, sizeof(double) * 2 * h->nmodes);
    int n = 0;
    for (int d = 0; d < 3; d++) {
      n += fft_make_len(h->fft.len[d], K[d], h->d_tw[d], h->stream);
      n += launch_bspline_moduli(K[d], order, h->nodes, h->d_iB[d], h->stream);
    }
    ok = launched(h, n, "ctor kernels") && CK(h, cudaMemsetAsync(h->d_real, 0, sizeof(float) * h->nreal, h->stream)) &&
         CK(h, cudaMemsetAsync(h->d_cplx, 0, sizeof(float2) * h->nmodes, h->stream)) && sync(h);
  }
  if (!ok) {
    destroy(h);
    cudaGetLastError();
    return nullptr;
  }
  return h;
}

void sfac_dtor(void *p) { destroy(H(p)); }

void sfac(void *p, int n, const double *w, const double *x) {
  Nvtx range("sfac sfac");
  Handle *h = H(p);
  if (!h) return;
  if (n < 0) {
    printf("sfac: bad atom count %d\n", n);
    return;
  }
  if (!ensure_atoms(h, n)) return;
  if (n > 0) {
    if (!CK(h, cudaMemcpyAsync(h->d_x, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream)) ||
        !CK(h, cudaMemcpyAsync(h->d_w, w, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream)))
      return;
  }
  CK(h, cudaEventRecord(h->ev_in, h->stream));
  int k = launch_cell_sort(h->geom, n, h->d_x, h->d_w, h->sb, h->stream, kSpreadZShift);
  k += launch_spread(h->geom, h->spline, h->sb.cell_start, h->sb.keys[h->sb.cur], h->sb.rec_sorted, h->d_real,
                     h->stream);
  DeconvArgs dc{h->d_iB[0], h->d_iB[1], h->d_iB[2], h->ldim};
  k += launch_fft_forward(h->fft, h->geom, h->d_real, h->d_cplx, dc, h->stream);
  if (!launched(h, k, "sfac kernels")) return;
  // The caller may reuse w and x once this returns: wait for the copies only.
  CK(h, cudaEventSynchronize(h->ev_in));
  h->last_n = n;
  h->state = 0;
}

double *get_S(void *p) {
  Handle *h = H(p);
  if (!h) return nullptr;
  if (h->state == 0) {
    if (CK(h, cudaMemcpyAsync(h->h_f, h->d_cplx, sizeof(float2) * h->nmodes, cudaMemcpyDeviceToHost,
                              h->stream)) &&
        sync(h)) {
      for (long i = 0; i < 2 * h->nmodes; i++) h->h_S[i] = (double)h->h_f[i];
    }
  } else if (h->state == 1) {
    if (CK(h, cudaMemcpyAsync(h->h_f, h->d_real, sizeof(float) * h->nreal, cudaMemcpyDeviceToHost, h->stream)) &&
        sync(h)) {
      const long rows = (long)h->K[0] * h->K[1];
      const int K2 = h->K[2], pitch = 2 * h->ldim;
      for (long r = 0; r < rows; r++) {
        double *dst = h->h_S + r * pitch;
        const float *src = h->h_f + r * K2;
        for (int k = 0; k < K2; k++) dst[k] = (double)src[k];
        for (int k = K2; k < pitch; k++) dst[k] = 0.0;
      }
    }
  }
  return h->h_S;
}

void set_L(void *p, double L[6]) {
  Handle *h = H(p);
  if (!h) return;
  set_cell(h, L);
}

// Tabulates A and dA exactly as set_A defines them (sfac.cpp:213-292): every
// lattice vector n with |m| < max_m, m = iL n, is folded onto its stored
// half-space mode (the conjugate partner when n_z mod K2 >= ldim), adding
// f(m^2)/2 to A and f'(m^2) m_a m_b to dA.  f runs on the host (it may be a
// Python callable); the tables are then uploaded as FP64.
int set_A(void *p, rad_fn f, double max_m, void *info) {
  Nvtx range("sfac set_A");
  Handle *h = H(p);
  if (!h) return 2;
  const int K0 = h->K[0], K1 = h->K[1], K2 = h->K[2], ldim = h->ldim;
  const long nm = h->nmodes;
  std::vector<double> tab;
  try {
    tab.assign(7 * (size_t)nm, 0.0);
  } catch (...) {
    return 2;
  }
  double *A = tab.data(), *dA = A + nm;
  const CellConst &g = h->hcell;
  const double R2 = max_m * max_m;
  const int i0 = (int)(max_m / g.iL00);
  for (int i = -i0; i <= i0; i++) {
    const double mx = i * g.iL00;
    const double m20 = mx * mx;
    const double dy = std::sqrt(std::fmax(R2 - m20, 0.0));
    const double my0 = i * g.iL10;
    const int j0 = (int)std::ceil((-dy - my0) / g.iL11);
    const int j1 = (int)std::floor((dy - my0) / g.iL11);
    for (int j = j0; j <= j1; j++) {
      const double my = my0 + j * g.iL11;
      const double m21 = m20 + my * my;
      const double dz = std::sqrt(std::fmax(R2 - m21, 0.0));
      const double mz0 = i * g.iL20 + j * g.iL21;
      const int k0 = (int)std::ceil((-dz - mz0) / g.iL22);
      const int k1 = (int)std::floor((dz - mz0) / g.iL22);
      for (int k = k0; k <= k1; k++) {
        const double mz = mz0 + k * g.iL22;
        const double m2 = m21 + mz * mz;
        const int kz = imod(k, K2);
        long mode;
        if (kz < ldim) mode = ((long)imod(i, K0) * K1 + imod(j, K1)) * ldim + kz;
        else mode = ((long)imod(-i, K0) * K1 + imod(-j, K1)) * ldim + (K2 - kz);
        double s = 0.0;
        A[mode] += 0.5 * f(m2, &s, info);
        double *d = dA + 6 * mode;
        d[0] += s * mx * mx;
        d[1] += s * my * my;
        d[2] += s * mz * mz;
        d[3] += s * my * mx;
        d[4] += s * mz * mx;
        d[5] += s * mz * my;
      }
    }
  }
  const bool fresh = !h->d_A;
  if (!h->d_A && !dalloc(h, &h->d_A, 7 * (size_t)nm)) return 2;
  if (!CK(h, cudaMemcpyAsync(h->d_A, A, sizeof(double) * 7 * nm, cudaMemcpyHostToDevice, h->stream)) || !sync(h))
    return 2;
  h->inf = Influence{};
  h->inf.mode = 1;
  h->inf.A = h->d_A;
  h->inf.dA = h->d_A + nm;
  if (fresh || h->a_mode != 1) h->version++;  // kernel arguments changed
  h->a_mode = 1;
  return 0;
}

double en(void *p) {
  Nvtx range("sfac en");
  Handle *h = H(p);
  if (!h) return 0.0;
  if (h->state != 0) {
    printf("Error: You must call sfac before this routine.\n");
    return 0.0;
  }
  if (h->a_mode == 0) {
    printf("Error: No convolution kernel has been set.\n");
    return 0.0;
  }
  int k = launch_energy(h->fft, h->geom, h->inf, h->d_iB[0], h->d_iB[1], h->d_iB[2], h->d_cplx, h->d_partials,
                        h->d_red, h->stream);
  if (!launched(h, k, "en kernels")) return 0.0;
  if (!CK(h, cudaMemcpyAsync(h->h_red, h->d_red, sizeof(double) * kRedWords, cudaMemcpyDeviceToHost, h->stream)) ||
      !sync(h))
    return 0.0;
  return h->h_red[0] * h->hcell.iV;
}

double de1(void *p, double vir[6]) {
  Nvtx range("sfac de1");
  Handle *h = H(p);
  if (!h) return 0.0;
  if (h->state != 0) {
    printf("Error: You must call sfac before this routine.\n");
    return 0.0;
  }
  if (h->a_mode == 0) {
    printf("Error: No convolution kernel has been set.\n");
    return 0.0;
  }
  // The energy and virial are read as soon as the x pass has summed them; the
  // inverse y/z passes that make the potential grid for de2/potl run on in
  // stream order while this returns (they overlap the caller's next copies).
  int k = launch_conv_energy(h->fft, h->geom, h->inf, h->d_iB[0], h->d_iB[1], h->d_iB[2], h->d_cplx, h->d_partials,
                             h->d_red, h->stream);
  if (!CK(h, cudaMemcpyAsync(h->h_red, h->d_red, sizeof(double) * kRedWords, cudaMemcpyDeviceToHost, h->stream)) ||
      !CK(h, cudaEventRecord(h->ev_in, h->stream)))
    return 0.0;
  k += inv_yz(h->fft, h->d_cplx, h->d_real, nullptr, 0, h->d_cell, nullptr, nullptr, h->stream);
  if (!launched(h, k, "de1 kernels") || !CK(h, cudaEventSynchronize(h->ev_in))) return 0.0;
  const double *r = h->h_red;
  const double fac = h->hcell.iV * h->hcell.iV;
  vir[0] = (r[1] + r[0]) * fac;
  vir[1] = (r[2] + r[0]) * fac;
  vir[2] = (r[3] + r[0]) * fac;
  vir[3] = r[4] * fac;
  vir[4] = r[5] * fac;
  vir[5] = r[6] * fac;
  h->state = 1;
  return r[0] * h->hcell.iV;
}

// True when p is host memory the GPU can copy asynchronously (pinned or
// registered); pageable memory gets the single-copy path.
static bool host_pinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Streams and events of the pipelined gather (created on first use).
static bool ensure_pipeline(Handle *h) {
  if (h->s_in) return true;
  bool ok = CK(h, cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking)) &&
            CK(h, cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking));
  for (int c = 0; c < kPipeChunks && ok; c++)
    ok = CK(h, cudaEventCreateWithFlags(&h->ev_copied[c], cudaEventDisableTiming)) &&
         CK(h, cudaEventCreateWithFlags(&h->ev_gathered[c], cudaEventDisableTiming));
  return ok;
}

// de2 / potl (sfac.cpp:409-545) on host arrays.  With pinned host buffers
// and enough points, the points are split into chunks: chunk c's copy in
// (s_in), gather (the handle's stream) and copy out (s_out) overlap the
// neighbouring chunks', so the two PCIe directions and the gather run at once.
static void gather_call(Handle *h, int n, const double *w, const double *x, double *dx, double *phi) {
  Nvtx range(dx ? "sfac de2" : "sfac potl");
  if (h->state != 1) {
    printf("Error: You must call de1 before this routine.\n");
    return;
  }
  if (n <= 0) return;
  if (!ensure_gather(h, n)) return;
  double *out = dx ? dx : phi;
  const int ow = dx ? 3 : 1;  // output words per point
  const bool pipe = n >= 2 * kPipeMinChunk && host_pinned(x) && (!w || host_pinned(w)) && host_pinned(out) &&
                    ensure_pipeline(h);
  if (!pipe) {
    if (!CK(h, cudaMemcpyAsync(h->d_gx, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream))) return;
    if (w && !CK(h, cudaMemcpyAsync(h->d_gw, w, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream))) return;
    int k = launch_gather(h->geom, h->spline, n, h->d_gx, h->d_gw, h->d_real, dx ? h->d_gout : nullptr,
                          phi ? h->d_gout : nullptr, h->stream);
    if (!launched(h, k, "gather kernel")) return;
    CK(h, cudaMemcpyAsync(out, h->d_gout, sizeof(double) * ow * n, cudaMemcpyDeviceToHost, h->stream));
    sync(h);
    return;
  }
  int nc = n / kPipeMinChunk;
  if (nc > kPipeChunks) nc = kPipeChunks;
  const int per = (n + nc - 1) / nc;
  // copies in may start at once: the previous call on these buffers has
  // completed (every call ends with a synchronisation)
  int k = 0;
  for (int c = 0; c < nc; c++) {
    const int a0 = c * per, m = (a0 + per <= n) ? per : n - a0;
    if (!CK(h, cudaMemcpyAsync(h->d_gx + 3L * a0, x + 3L * a0, sizeof(double) * 3 * m, cudaMemcpyHostToDevice,
                               h->s_in)))
      return;
    if (w && !CK(h, cudaMemcpyAsync(h->d_gw + a0, w + a0, sizeof(double) * m, cudaMemcpyHostToDevice, h->s_in)))
      return;
    if (!CK(h, cudaEventRecord(h->ev_copied[c], h->s_in)) || !CK(h, cudaStreamWaitEvent(h->stream, h->ev_copied[c], 0)))
      return;
    k += launch_gather(h->geom, h->spline, m, h->d_gx + 3L * a0, h->d_gw + a0, h->d_real,
                       dx ? h->d_gout + 3L * a0 : nullptr, phi ? h->d_gout + a0 : nullptr, h->stream);
    if (!CK(h, cudaEventRecord(h->ev_gathered[c], h->stream)) ||
        !CK(h, cudaStreamWaitEvent(h->s_out, h->ev_gathered[c], 0)))
      return;
    if (!CK(h, cudaMemcpyAsync(out + (long)ow * a0, h->d_gout + (long)ow * a0, sizeof(double) * ow * m,
                               cudaMemcpyDeviceToHost, h->s_out)))
      return;
  }
  if (!launched(h, k, "gather kernel")) return;
  CK(h, cudaStreamSynchronize(h->s_out));
  sync(h);
}

void de2(void *p, int n, const double *w, const double *x, double *dx) {
  Handle *h = H(p);
  if (!h) return;
  gather_call(h, n, w, x, dx, nullptr);
}

void potl(void *p, int n, const double *x, double *phi) {
  Handle *h = H(p);
  if (!h) return;
  gather_call(h, n, nullptr, x, nullptr, phi);
}

// Coarse grid of the real-space cell list: cells at least rcut/kRealSub wide along
// every fractional axis (perpendicular widths of the box from iL).  False when
// rcut exceeds half the smallest width (the minimum image would not be unique).
static bool real_grid(const Handle *h, double rcut, int nb[3]) {
  const CellConst &c = h->hcell;
  const double wd[3] = {1.0 / sqrt(c.iL00 * c.iL00 + c.iL10 * c.iL10 + c.iL20 * c.iL20),
                        1.0 / sqrt(c.iL11 * c.iL11 + c.iL21 * c.iL21), 1.0 / fabs(c.iL22)};
  const double wmin = fmin(wd[0], fmin(wd[1], wd[2]));
  if (!(rcut > 0.0) || rcut > 0.5 * wmin) return false;
  for (int d = 0; d < 3; d++) {  // cells at least rcut / kRealSub wide
    const double m = floor(kRealSub * wd[d] / rcut);
    nb[d] = m < 1.0 ? 1 : (m > 1023.0 ? 1023 : (int)m);
  }
  return true;
}

// Checks the arguments and sizes the buffers; fills the coarse geometry.
static int real_prepare(Handle *h, int n, double eta, double rcut, Geom &cg) {
  int nb[3];
  if (n < 0 || !(eta > 0.0)) {
    printf("sfac_real_space: bad atom count %d or eta %g\n", n, eta);
    return 1;
  }
  if (!real_grid(h, rcut, nb)) {
    printf("sfac_real_space: cutoff %g must be positive and at most half the smallest box width\n", rcut);
    return 1;
  }
  if (!ensure_real(h, n, (long)nb[0] * nb[1] * nb[2])) return 2;
  cg = Geom{};
  cg.K0 = nb[0];
  cg.K1 = nb[1];
  cg.K2 = nb[2];
  cg.ldim = nb[2] / 2 + 1;
  cg.order = h->order;
  cg.cell = h->d_cell;
  return 0;
}

int sfac_real_space_device(void *p, int n, const double *x, const double *w, double eta, double rcut, double *out,
                           double *dx) {
  Handle *h = H(p);
  if (!h || !out || (n > 0 && (!x || !w))) return 1;
  Geom cg;
  const int rc = real_prepare(h, n, eta, rcut, cg);
  if (rc) return rc;
  const int k = launch_real_space(cg, h->L, n, x, w, (float)eta, (float)rcut, h->rs.sb, h->rs.rec, h->rs.tab, dx,
                                  h->rs.part, eta, out, h->stream);
  return launched(h, k, "real-space kernels") ? 0 : 2;
}

int sfac_real_space(void *p, int n, const double *w, const double *x, double eta, double rcut, double out[10],
                    double *dx) {
  Handle *h = H(p);
  if (!h || !out || (n > 0 && (!x || !w))) return 1;
  Geom cg;
  const int rc = real_prepare(h, n, eta, rcut, cg);
  if (rc) return rc;
  if (n > 0 && (!CK(h, cudaMemcpyAsync(h->rs.x, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream)) ||
                !CK(h, cudaMemcpyAsync(h->rs.w, w, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream))))
    return 2;
  const int k = launch_real_space(cg, h->L, n, h->rs.x, h->rs.w, (float)eta, (float)rcut, h->rs.sb, h->rs.rec,
                                  h->rs.tab, dx ? h->rs.dx : nullptr, h->rs.part, eta, h->rs.out, h->stream);
  if (!launched(h, k, "real-space kernels")) return 2;
  if (!CK(h, cudaMemcpyAsync(out, h->rs.out, sizeof(double) * 10, cudaMemcpyDeviceToHost, h->stream))) return 2;
  if (dx && n > 0 &&
      !CK(h, cudaMemcpyAsync(dx, h->rs.dx, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream)))
    return 2;
  return sync(h) ? 0 : 2;
}

int sfac_sk_reset(void *p) {
  Handle *h = H(p);
  if (!h) return 1;
  if (!h->d_sk && !dalloc(h, &h->d_sk, (size_t)h->nmodes)) return 2;
  h->sk_frames = 0;
  return CK(h, cudaMemsetAsync(h->d_sk, 0, sizeof(double) * h->nmodes, h->stream)) ? 0 : 2;
}

int sfac_sk_accumulate(void *p) {
  Handle *h = H(p);
  if (!h) return 1;
  if (h->state != 0) {
    printf("Error: You must call sfac before this routine.\n");
    return 1;
  }
  if (!h->d_sk && sfac_sk_reset(p) != 0) return 2;
  const int k = launch_sk_accumulate(h->nmodes, h->d_cplx, h->d_sk, h->stream);
  if (!launched(h, k, "sk accumulate")) return 2;
  h->sk_frames++;
  return 0;
}

int sfac_sk_get(void *p, double *out, long long *frames) {
  Handle *h = H(p);
  if (!h || !out) return 1;
  if (!h->d_sk && sfac_sk_reset(p) != 0) return 2;
  if (frames) *frames = h->sk_frames;
  if (!CK(h, cudaMemcpyAsync(out, h->d_sk, sizeof(double) * h->nmodes, cudaMemcpyDeviceToHost, h->stream))) return 2;
  return sync(h) ? 0 : 2;
}

int sfac_sk_radial(void *p, int nbins, double kmax, double *sums, double *counts) {
  Handle *h = H(p);
  if (!h || !sums || !counts || nbins < 1 || !(kmax > 0.0)) return 1;
  if (!h->d_sk && sfac_sk_reset(p) != 0) return 2;
  if (nbins > h->sk_cap || !h->d_skpart) {
    dfree(h->d_skpart);
    dfree(h->d_skres);
    if (!dalloc(h, &h->d_skpart, sk_partial_words()) || !dalloc(h, &h->d_skres, 2 * (size_t)nbins)) {
      h->sk_cap = 0;
      return 2;
    }
    h->sk_cap = nbins;
  }
  const int k = launch_sk_radial(h->geom, h->d_sk, nbins, kmax / nbins, h->d_skpart, h->d_skres, h->d_skres + nbins,
                                 h->stream);
  if (!launched(h, k, "sk radial")) return 2;
  if (!CK(h, cudaMemcpyAsync(sums, h->d_skres, sizeof(double) * nbins, cudaMemcpyDeviceToHost, h->stream)) ||
      !CK(h, cudaMemcpyAsync(counts, h->d_skres + nbins, sizeof(double) * nbins, cudaMemcpyDeviceToHost, h->stream)))
    return 2;
  return sync(h) ? 0 : 2;
}

int sfac_xc_reset(void *p, int D) {
  Handle *h = H(p);
  if (!h || D < 1 || D > 64) return 1;
  const size_t nm = (size_t)h->nmodes, npair = (size_t)D * (D + 1) / 2;
  if (D != h->xc_D) {
    dfree(h->d_xcq);
    dfree(h->d_xcc);
    h->xc_D = 0;
    if (!dalloc(h, &h->d_xcq, (size_t)D * nm) || !dalloc(h, &h->d_xcc, npair * nm)) return 2;
    h->xc_D = D;
  }
  h->xc_frames = 0;
  return CK(h, cudaMemsetAsync(h->d_xcc, 0, sizeof(double2) * npair * nm, h->stream)) &&
                 CK(h, cudaMemsetAsync(h->d_xcq, 0, sizeof(float2) * (size_t)D * nm, h->stream))
             ? 0
             : 2;
}

int sfac_xc_store(void *p, int i) {
  Handle *h = H(p);
  if (!h || i < 0 || i >= h->xc_D) return 1;
  if (h->state != 0) {
    printf("Error: You must call sfac before this routine.\n");
    return 1;
  }
  const int k = launch_xc_store(h->nmodes, h->d_cplx, h->d_xcq + (size_t)i * h->nmodes, h->stream);
  return launched(h, k, "xc store") ? 0 : 2;
}

int sfac_xc_accumulate(void *p) {
  Handle *h = H(p);
  if (!h || h->xc_D < 1) return 1;
  const int k = launch_xc_accumulate(h->nmodes, h->xc_D, h->d_xcq, h->d_xcc, h->stream);
  if (!launched(h, k, "xc accumulate")) return 2;
  h->xc_frames++;
  return 0;
}

int sfac_xc_get(void *p, int k, double *out, long long *frames) {
  Handle *h = H(p);
  if (!h || !out || h->xc_D < 1 || k < 0 || k >= h->xc_D * (h->xc_D + 1) / 2) return 1;
  if (frames) *frames = h->xc_frames;
  if (!CK(h, cudaMemcpyAsync(out, h->d_xcc + (size_t)k * h->nmodes, sizeof(double2) * h->nmodes,
                             cudaMemcpyDeviceToHost, h->stream)))
    return 2;
  return sync(h) ? 0 : 2;
}

int sfac_set_radial(void *p, int nt, const double *f, const double *df, double m2max, double max_m) {
  Handle *h = H(p);
  if (!h) return 1;
  if (nt < 2 || !f || !df || !(m2max > 0.0) || !(max_m >= 0.0) || max_m * max_m > m2max) {
    printf("sfac_set_radial: need nt >= 2 samples on [0, m2max] with max_m^2 <= m2max\n");
    return 1;
  }
  const size_t nm = (size_t)h->nmodes;
  double *dtab = nullptr;
  if (!h->d_A && !dalloc(h, &h->d_A, 7 * nm)) return 2;
  if (!dalloc(h, &dtab, 2 * (size_t)nt)) return 2;
  const CellConst &c = h->hcell;
  const InfConst ic{c.iL00, c.iL10, c.iL11, c.iL20, c.iL21, c.iL22, 0.0, max_m, 0.0};
  bool ok = CK(h, cudaMemcpyAsync(dtab, f, sizeof(double) * nt, cudaMemcpyHostToDevice, h->stream)) &&
            CK(h, cudaMemcpyAsync(dtab + nt, df, sizeof(double) * nt, cudaMemcpyHostToDevice, h->stream));
  if (ok) {
    const int k = launch_radial_table(h->geom, ic, dtab, dtab + nt, nt, m2max / (nt - 1), h->d_A, h->d_A + nm,
                                      h->stream);
    ok = launched(h, k, "radial table") && sync(h);
  }
  dfree(dtab);
  if (!ok) return 3;
  Influence inf{};
  inf.mode = 1;
  inf.A = h->d_A;
  inf.dA = h->d_A + nm;
  inf.K2d = FastDiv((uint32_t)h->K[2]);
  if (h->a_mode != 3 || memcmp(&inf, &h->inf, sizeof(Influence)) != 0) h->version++;
  h->inf = inf;
  h->a_mode = 3;
  return 0;
}

int sfac_set_ewald(void *p, double beta, double max_m) {
  Handle *h = H(p);
  if (!h) return 1;
  if (!(beta > 0.0) || !(max_m >= 0.0)) {
    printf("sfac_set_ewald: bad beta %g or max_m %g\n", beta, max_m);
    return 1;
  }
  if (!h->d_rows && !dalloc(h, &h->d_rows, (size_t)h->K[0] * h->K[1])) return 2;
  const CellConst &c = h->hcell;
  const double pb = 3.14159265358979323846 / beta;
  h->hic = InfConst{c.iL00, c.iL10, c.iL11, c.iL20, c.iL21, c.iL22, beta, max_m, -(pb * pb)};
  Influence inf{};
  inf.mode = 2;
  inf.ic = h->d_ic;
  inf.rows = h->d_rows;
  inf.K2d = FastDiv((uint32_t)h->K[2]);
  // constants and row tables are rewritten in place on the stream: later
  // solves see them without new kernel arguments
  if (!CK(h, cudaMemcpyAsync(h->d_ic, &h->hic, sizeof(InfConst), cudaMemcpyHostToDevice, h->stream))) return 3;
  int k = launch_ewald_rows(h->geom, inf, h->d_rows, h->stream);
  // Tabulate A and dA once (FP64, 56 bytes per stored mode) when the tables
  // stay within kEwaldTableMaxBytes: every solve then reads them instead of
  // evaluating the images (one exp each) of every mode.  SFAC_EWALD_TABLE=0
  // keeps the per-solve evaluation.
  const size_t nm = (size_t)h->nmodes;
  bool table = 56 * nm <= kEwaldTableMaxBytes;
  bool compact = !table;
  if (h->ewald_src == 2) table = compact = false;  // the box may change on the device (sfac_box_update_device)
  if (const char *e = getenv("SFAC_EWALD_TABLE")) {
    if (e[0] == '0' && e[1] == 0) table = compact = false;  // evaluate the images in every solve
    if (e[0] == 'c' && e[1] == 0) {  // compact table whatever the size
      compact = true;
      table = false;
    }
  }
  if (table) {
    if (!h->d_A && !dalloc(h, &h->d_A, 7 * nm)) return 2;
    k += launch_ewald_table(h->geom, inf, h->d_A, h->d_A + nm, h->stream);
    inf = Influence{};
    inf.mode = 1;
    inf.A = h->d_A;
    inf.dA = h->d_A + nm;
    inf.K2d = FastDiv((uint32_t)h->K[2]);
  } else if (compact) {
    // A per mode with its single image's lattice shift (8 bytes per mode):
    // dA then costs no exp in the solves
    if (!h->d_A && !dalloc(h, &h->d_A, 7 * nm)) return 2;
    k += launch_ewald_compact(h->geom, inf, h->d_A, h->stream);
    inf.mode = 4;
    inf.A = h->d_A;
  }
  if (!launched(h, k, "ewald rows")) return 3;
  if (h->a_mode != 2 || memcmp(&inf, &h->inf, sizeof(Influence)) != 0) h->version++;  // kernel arguments changed
  h->inf = inf;
  h->a_mode = 2;
  return 0;
}

// Box constants from a box L = [ax, by, cz, bx, cx, cy] in device memory,
// with make_cell's expressions and operation order (explicit round-to-nearest
// operations, no contraction: the same bits as the host's Cell), and the
// device Ewald constants of that box (beta, max_m, fac fixed by the handle).
__global__ void box_from_device_kernel(const double *__restrict__ L, CellConst *cell, InfConst *ic, double beta,
                                       double max_m, double fac) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double L0 = L[0], L1 = L[1], L2 = L[2], L3 = L[3], L4 = L[4], L5 = L[5];
  CellConst c{};
  c.iV = __ddiv_rn(1.0, __dmul_rn(__dmul_rn(L0, L1), L2));
  c.iL00 = __ddiv_rn(1.0, L0);
  c.iL11 = __ddiv_rn(1.0, L1);
  c.iL22 = __ddiv_rn(1.0, L2);
  c.iL10 = __dmul_rn(__dmul_rn(-L3, L2), c.iV);
  c.iL20 = __dmul_rn(__dsub_rn(__dmul_rn(L3, L5), __dmul_rn(L1, L4)), c.iV);
  c.iL21 = __dmul_rn(__dmul_rn(-L0, L5), c.iV);
  *cell = c;
  *ic = InfConst{c.iL00, c.iL10, c.iL11, c.iL20, c.iL21, c.iL22, beta, max_m, fac};
}

int sfac_box_update_device(void *p, const double *L_dev) {
  Handle *h = H(p);
  if (!h || !L_dev) return 1;
  if (h->a_mode != 2 || h->inf.mode != 2) {
    printf("sfac_box_update_device: needs sfac_set_ewald with SFAC_TUNE_EWALD_SOURCE = 2\n");
    return 1;
  }
  box_from_device_kernel<<<1, 32, 0, h->stream>>>(L_dev, h->d_cell, h->d_ic, h->hic.beta, h->hic.max_m, h->hic.fac);
  const int k = 1 + launch_ewald_rows(h->geom, h->inf, h->d_rows, h->stream);
  return launched(h, k, "box update") ? 0 : 2;
}

int sfac_set_stream(void *p, void *stream) {
  Handle *h = H(p);
  if (!h) return 1;
  if (!sync(h)) return 1;
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  h->version++;
  return 0;
}

void *sfac_get_stream(void *p) { return p ? (void *)H(p)->stream : nullptr; }

// Full solve on device arrays; with `ev` non-null the stage boundaries are
// recorded into h->ev_stage.
static int enqueue_solve(Handle *h, int n, const double *x, const double *w, double *dx, double *phi,
                         double *ev, double *dEdL, bool timed) {
  cudaStream_t st = h->stream;
  int k = 0;
  if (timed) CK(h, cudaEventRecord(h->ev_stage[0], st));
  {
    Nvtx r("spme cell sort");
    k += launch_cell_sort(h->geom, n, x, w, h->sb, st, kSpreadZShift);
  }
  if (timed) CK(h, cudaEventRecord(h->ev_stage[1], st));
  {
    Nvtx r("spme spread");
    k += launch_spread(h->geom, h->spline, h->sb.cell_start, h->sb.keys[h->sb.cur], h->sb.rec_sorted, h->d_real, st);
  }
  if (timed) CK(h, cudaEventRecord(h->ev_stage[2], st));
  int nb = 0;
  {
    Nvtx r("spme fft forward");
    k += fwd_zy(h->fft, h->d_real, h->d_cplx, st);
  }
  if (timed) CK(h, cudaEventRecord(h->ev_stage[3], st));
  {
    Nvtx r("spme convolution");
    k += launch_x_conv(h->fft, h->geom, h->inf, h->d_iB[0], h->d_iB[1], h->d_iB[2], h->d_cplx, h->d_partials, nb,
                       st);
  }
  if (timed) CK(h, cudaEventRecord(h->ev_stage[4], st));
  {
    Nvtx r("spme fft inverse");
    k += inv_yz(h->fft, h->d_cplx, h->d_real, h->d_partials, nb, h->d_cell, h->d_red, ev, st);
  }
  if (timed) CK(h, cudaEventRecord(h->ev_stage[5], st));
  Nvtx r("spme gather");
  // gather in cell order (the sort of this solve): neighbouring threads share grid lines
  const uint32_t *perm = h->sb.vals[h->sb.cur], *skeys = h->sb.keys[h->sb.cur];
  if (dEdL)
    k += launch_gather_cell(h->geom, h->spline, n, x, w, h->d_real, dx, phi, h->d_cellp, ev, dEdL, st, perm, skeys,
                            h->sb.rec_sorted);
  else if (n > 0 && (dx || phi))
    k += launch_gather(h->geom, h->spline, n, x, w, h->d_real, dx, phi, st, perm, skeys, h->sb.rec_sorted);
  if (timed) CK(h, cudaEventRecord(h->ev_stage[6], st));
  return k;
}

static int solve_device(Handle *h, int n, const double *x, const double *w, double *dx, double *phi,
                        double *ev, double *dEdL, bool timed) {
  if (n < 0 || (n > 0 && (!x || !w)) || !ev || (dEdL && n > 0 && !dx)) return 1;
  if (h->a_mode == 0) {
    printf("Error: No convolution kernel has been set.\n");
    return 1;
  }
  if (!ensure_atoms(h, n)) return 2;
  if (dEdL && !ensure_cellp(h, n)) return 2;
  if (timed || !h->use_graph) {
    const int k = enqueue_solve(h, n, x, w, dx, phi, ev, dEdL, timed);
    if (!launched(h, k, "solve kernels")) return 3;
  } else {
    const Handle::Key key{n, x, w, dx, phi, ev, dEdL, h->stream, h->version};
    if (!(h->graph && key == h->gkey)) {
      if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
      }
      cudaGraph_t gr = nullptr;
      if (!CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal))) return 3;
      const int k = enqueue_solve(h, n, x, w, dx, phi, ev, dEdL, false);
      const bool ok_launch = check(h, cudaGetLastError(), "solve kernels (capture)");
      if (!CK(h, cudaStreamEndCapture(h->stream, &gr)) || !ok_launch) {
        if (gr) cudaGraphDestroy(gr);
        return 3;
      }
      const bool ok = CK(h, cudaGraphInstantiate(&h->graph, gr, 0));
      cudaGraphDestroy(gr);
      if (!ok) {
        h->graph = nullptr;
        return 3;
      }
      h->gkey = key;
      h->graph_kernels = k;
    }
    if (!CK(h, cudaGraphLaunch(h->graph, h->stream))) return 3;
    h->launches += h->graph_kernels;
  }
  h->last_n = n;
  h->state = 1;
  return 0;
}

int sfac_solve_device(void *p, int n, const double *x, const double *w, double *dx, double *phi, double *ev) {
  Handle *h = H(p);
  if (!h) return 1;
  return solve_device(h, n, x, w, dx, phi, ev, nullptr, false);
}

int sfac_solve_device_cell(void *p, int n, const double *x, const double *w, double *dx, double *phi, double *ev,
                           double *dEdL) {
  Handle *h = H(p);
  if (!h || !dEdL) return 1;
  return solve_device(h, n, x, w, dx, phi, ev, dEdL, false);
}

int sfac_solve_device_timed(void *p, int n, const double *x, const double *w, double *dx, double *phi,
                            double *ev, float stage_ms[6]) {
  Handle *h = H(p);
  if (!h) return 1;
  int rc = solve_device(h, n, x, w, dx, phi, ev, nullptr, true);
  if (rc) return rc;
  if (!sync(h)) return 3;
  for (int i = 0; i < 6; i++) {
    float ms = 0.f;
    if (!CK(h, cudaEventElapsedTime(&ms, h->ev_stage[i], h->ev_stage[i + 1]))) return 3;
    stage_ms[i] = ms;
  }
  return 0;
}

int sfac_set_graphs(void *p, int enable) {
  Handle *h = H(p);
  if (!h) return 1;
  h->use_graph = enable != 0;
  return 0;
}

int sfac_set_tuning(void *p, int key, int value) {
  Handle *h = H(p);
  if (!h) return 1;
  if (key == SFAC_TUNE_X_LINES) {
    if (value < 0 || value > 64 || (value & (value - 1))) return 1;
    h->fft.x_lines = value;
    h->version++;
    return 0;
  }
  if (key == SFAC_TUNE_EWALD_SOURCE) {
    if (value != 0 && value != 2) return 1;
    h->ewald_src = value;
    return 0;
  }
  if (key == SFAC_TUNE_ZY_MODE) {
    if (value < 0 || value > 3) return 1;
    h->fft.zy_mode = value;
    h->version++;
    return 0;
  }
  return 1;
}

unsigned long sfac_footprint_bytes(const int K[3], int n) {
  const size_t K0 = K[0], K1 = K[1], K2 = K[2], ldim = K2 / 2 + 1, nn = (size_t)(n > 0 ? n : 1);
  const size_t cap = nn + nn / 2 + 64;
  const long nzb = ((long)K2 + (1L << kSpreadZShift) - 1) >> kSpreadZShift;
  size_t b = 4 * K0 * K1 * K2 + 8 * K0 * K1 * ldim + 4 * cell_count_words((long)(K0 * K1) * nzb);  // grids, buckets
  b += (K0 + K1 + K2) * 16 + sizeof(RowImg) * K0 * K1;                   // moduli, twiddles, rows
  b += 8 * (size_t)fft_x_blocks_max(K[1], K[2]) * kRedWords;               // partials
  b += cap * (24 + 8 + 7 * 4 + 16 + 16);                                   // sort buffers, records
  b += 8 * cap * 8;                                                        // gather staging
  b += 8 * 2 * K0 * K1 * ldim + 4 * K0 * K1 * K2;                          // host mirrors (pinned)
  return b;
}

int sfac_last_error(void *p) { return p ? H(p)->err : -1; }
const char *sfac_error_string(void *p) { return p ? H(p)->errstr : "null handle"; }
int sfac_device(void *p) { return p ? H(p)->device : -1; }
long long sfac_kernel_launches(void *p) { return p ? H(p)->launches : 0; }

int sfac_debug_sort(void *p, int n, int *keys, int *perm) {
  Handle *h = H(p);
  if (!h || n != h->last_n || h->state < 0) return 1;
  if (n == 0) return 0;
  if (!CK(h, cudaMemcpyAsync(keys, h->sb.keys[h->sb.cur], sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream)) ||
      !CK(h, cudaMemcpyAsync(perm, h->sb.vals[h->sb.cur], sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream)))
    return 1;
  return sync(h) ? 0 : 1;
}

int sfac_check_enabled(void) {
#ifdef SPME_CHECK
  return 1;
#else
  return 0;
#endif
}

int sfac_check_take(unsigned long long *word) {
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  unsigned long long (*const take[])() = {spme::check_take_sort,  spme::check_take_spread,
                                          spme::check_take_gather, spme::check_take_fft,
                                          spme::check_take_serve,  spme::check_take_capi};
  int first = 0;
  for (int m = 0; m < (int)(sizeof(take) / sizeof(take[0])); m++) {
    const unsigned long long v = take[m]();
    if (v && !first) {
      first = m + 1;
      if (word) *word = v;
    }
  }
  return first;
}

int sfac_check_selftest(void) {
  if (!sfac_check_enabled()) return -1;
  float *buf = nullptr;
  if (cudaMalloc(&buf, 64 * sizeof(float)) != cudaSuccess) return 2;
  unsigned long long w = 0;
  sfac_check_take(nullptr);  // start from clear words
  spme::check_selftest_kernel<<<1, 32>>>(buf);
  const int m = sfac_check_take(&w);
  cudaFree(buf);
  const unsigned long long want = ((unsigned long long)spme::CK_SELFTEST << 40) | 40ull;
  return (m == 6 && w == want) ? 0 : 1;
}

int sfac_debug_fail_alloc(int nth) {
  fail_alloc_in.store(nth > 0 ? nth : 0);
  return 0;
}

int sfac_debug_spread(void *p, float *grid) {
  Handle *h = H(p);
  if (!h || h->state != 0) return 1;
  if (!CK(h, cudaMemcpyAsync(grid, h->d_real, sizeof(float) * h->nreal, cudaMemcpyDeviceToHost, h->stream)))
    return 1;
  return sync(h) ? 0 : 1;
}

}  // extern "C"
