// Serving runtime: a persistent pool of SPME solvers on one GPU with
// continuous admission.
//
// A slot is one solver handle (resident grids, B-spline moduli, FFT twiddles)
// plus fixed device buffers for one atom-count bucket, on its own stream.  A
// request is admitted into an idle slot of its shape (grid, order, Ewald
// parameters, bucket), or a new slot while the device memory budget allows
// -- idle slots are evicted least-recently-used first.  Admitted requests run
// concurrently on their slots' streams.
//
// Each slot replays one captured CUDA graph per request, and the request
// costs four host calls: one copy in of a packed block [header (box, atom
// count) | positions | charges], the graph launch, one copy out of
// [E, virial, dE/dx, phi], and an event.  The graph itself unpacks the block
// (padding the atoms to the bucket with zero charges, which leaves every
// result unchanged), takes the request's box on the device (box constants
// and Ewald row tables, sfac_box_update_device), runs the solve, and packs
// phi behind dE/dx.  Completion is detected by polling one event per slot.
// Built on the C ABI of include/sfac.h.
#include <cuda.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/sfac.h"
#include "spme_kernels.hpp"

namespace spme {
SPME_CHECK_READER(serve)
}  // namespace spme

namespace {

constexpr int kHdr = 16;  // header doubles of a packed request: L[6], n, fractional flag, unused

// Packed block (device) -> positions and charges of the solve, padded to the
// bucket: padding atoms copy real positions (the spread stays balanced) and
// carry zero charge.
// Header word 7 = 1: the positions are fractional coordinates s of the box
// (x = s0 a + s1 b + s2 c, the box rows of L), turned into Cartesian ones
// here in FP64 (for a cubic box exactly x = s * side).
__global__ void unpack_kernel(const double *__restrict__ blk, double *__restrict__ x, double *__restrict__ q,
                              int ncap) {
  const int n = (int)blk[6];
  if (n > 0 && !SPME_IN(n - 1, ncap, spme::CK_SERVE_ATOM)) return;
  const bool frac = blk[7] != 0.0;
  const double L0 = blk[0], L1 = blk[1], L2 = blk[2], L3 = blk[3], L4 = blk[4], L5 = blk[5];
  const double *xs = blk + kHdr, *qs = xs + 3 * (size_t)n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncap; i += gridDim.x * blockDim.x) {
    const int s = i < n ? i : (n > 0 ? i % n : -1);
    double v0 = s >= 0 ? xs[3 * s + 0] : 0.0, v1 = s >= 0 ? xs[3 * s + 1] : 0.0, v2 = s >= 0 ? xs[3 * s + 2] : 0.0;
    if (frac) {
      const double c0 = __dadd_rn(__dadd_rn(__dmul_rn(v0, L0), __dmul_rn(v1, L3)), __dmul_rn(v2, L4));
      const double c1 = __dadd_rn(__dmul_rn(v1, L1), __dmul_rn(v2, L5));
      const double c2 = __dmul_rn(v2, L2);
      v0 = c0;
      v1 = c1;
      v2 = c2;
    }
    x[3 * i + 0] = v0;
    x[3 * i + 1] = v1;
    x[3 * i + 2] = v2;
    q[i] = i < n ? qs[i] : 0.0;
  }
}

// phi of the first n atoms behind their dE/dx in the output block
// [E, vir(6), dx(3n), phi(n)] (dx already sits at out + 7).
__global__ void pack_phi_kernel(const double *__restrict__ blk, const double *__restrict__ phi,
                                double *__restrict__ out, int ncap) {
  const int n = (int)blk[6];
  if (n > 0 && !SPME_IN(n - 1, ncap, spme::CK_SERVE_OUT)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[7 + 3 * (size_t)n + i] = phi[i];
}

struct Slot {
  void *h = nullptr;
  int K[3] = {0, 0, 0}, order = 0, ncap = 0;
  double beta = 0, max_m = 0;
  double *d_blk = nullptr;   // packed request block (kHdr + 4 ncap)
  double *d_x = nullptr, *d_q = nullptr, *d_phi = nullptr;
  double *d_out = nullptr;   // [E, vir(6), dx(3 ncap) | phi(n) packed after dx(3n)]
  double *h_blk = nullptr;   // pinned staging of the unpacked submit path (kHdr + 4 ncap)
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  cudaGraphExec_t graph = nullptr;
  bool busy = false;
  long long id = -1;
  unsigned long long last = 0;
  size_t bytes = 0;
  double work = 0.0;           // working set of the request in flight (bytes)
  uint32_t *flag_h = nullptr;  // host-mapped word the stream sets to seq once the outputs are back
  CUdeviceptr flag_d = 0;
  uint32_t seq = 0;
};

// cuStreamWriteValue32, from the driver through the runtime (null where
// stream memory operations are unavailable: completion is then polled with
// events only).
typedef CUresult (*WriteValue32)(CUstream, CUdeviceptr, cuuint32_t, unsigned int);
WriteValue32 write_value32() {
  static WriteValue32 fn = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuStreamWriteValue32", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<WriteValue32>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

struct Tune {
  int K[3], order, x_lines;
};

struct Server {
  int device = 0;
  size_t budget = 0, used = 0;
  int max_inflight = 1, inflight = 0;
  double work_budget = 256.0 * (1 << 20), inflight_work = 0.0;  // bytes of working set in flight
  bool graphs = true;
  std::vector<Slot *> slots;
  std::vector<Tune> tunes;
  unsigned long long tick = 0;
  long long solves = 0, created = 0, evicted = 0, errors = 0;
  unsigned polls = 0;  // every 64th poll also asks the events (work that failed never sets its flag)
};

int bucket(int n) {
  // 256 * sqrt(2)^k rounded up to a multiple of 64
  double b = 256.0;
  while (b < n) b *= 1.4142135623730951;
  const int v = (int)b;
  return (v + 63) / 64 * 64;
}

// Device working set of one request (its grids and atom buffers): requests
// in flight together should keep theirs within the L2-sized work budget --
// concurrent solves whose grids stop fitting the 126 MB L2 all run slower.
double request_work(const int K[3], int n) {
  const double G = 4.0 * K[0] * K[1] * K[2], H = 8.0 * K[0] * K[1] * (K[2] / 2 + 1);
  return G + H + 96.0 * n;
}

size_t slot_bytes(const int K[3], int ncap) {
  return sfac_footprint_bytes(K, ncap) + sizeof(double) * (2 * kHdr + 8 + 13 * (size_t)ncap);
}

void destroy_slot(Slot *s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  if (s->done) cudaEventDestroy(s->done);
  for (double *p : {s->d_blk, s->d_x, s->d_q, s->d_phi, s->d_out})
    if (p) cudaFree(p);
  if (s->h_blk) cudaFreeHost(s->h_blk);
  if (s->flag_h) cudaFreeHost(s->flag_h);
  if (s->h) sfac_dtor(s->h);
  delete s;
}

}  // namespace

namespace {

// The device work of one request on its slot (what the slot's graph holds).
bool enqueue_request_work(Slot *s) {
  const int blocks = (s->ncap + 255) / 256 < 1024 ? (s->ncap + 255) / 256 : 1024;
  unpack_kernel<<<blocks, 256, 0, s->st>>>(s->d_blk, s->d_x, s->d_q, s->ncap);
  if (sfac_box_update_device(s->h, s->d_blk) != 0) return false;
  if (sfac_solve_device(s->h, s->ncap, s->d_x, s->d_q, s->d_out + 7, s->d_phi, s->d_out) != 0) return false;
  pack_phi_kernel<<<blocks, 256, 0, s->st>>>(s->d_blk, s->d_phi, s->d_out, s->ncap);
  return cudaGetLastError() == cudaSuccess;
}

Slot *create_slot(Server *sv, int ncap, const int K[3], int order, double beta, double max_m, const double L[6]) {
  Slot *s = new Slot;
  double Lc[6];
  int Kc[3] = {K[0], K[1], K[2]};
  memcpy(Lc, L, sizeof(Lc));
  s->h = sfac_ctor(Lc, Kc, order);
  bool ok = s->h != nullptr;
  ok = ok && sfac_set_tuning(s->h, SFAC_TUNE_EWALD_SOURCE, 2) == 0 && sfac_set_ewald(s->h, beta, max_m) == 0 &&
       sfac_set_graphs(s->h, 0) == 0;
  for (const Tune &t : sv->tunes)
    if (ok && t.K[0] == K[0] && t.K[1] == K[1] && t.K[2] == K[2] && t.order == order)
      sfac_set_tuning(s->h, SFAC_TUNE_X_LINES, t.x_lines);
  const size_t nb = kHdr + 4 * (size_t)ncap;
  ok = ok && spme::device_malloc((void **)&s->d_blk, sizeof(double) * nb) == cudaSuccess &&
       spme::device_malloc((void **)&s->d_x, sizeof(double) * 3 * ncap) == cudaSuccess &&
       spme::device_malloc((void **)&s->d_q, sizeof(double) * ncap) == cudaSuccess &&
       spme::device_malloc((void **)&s->d_phi, sizeof(double) * ncap) == cudaSuccess &&
       spme::device_malloc((void **)&s->d_out, sizeof(double) * (8 + 4 * (size_t)ncap)) == cudaSuccess &&
       cudaMallocHost((void **)&s->h_blk, sizeof(double) * nb) == cudaSuccess &&
       cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming) == cudaSuccess;
  if (ok && write_value32()) {  // completion word (events remain the fallback)
    void *dp = nullptr;
    if (cudaHostAlloc((void **)&s->flag_h, sizeof(uint32_t), cudaHostAllocMapped) == cudaSuccess &&
        cudaHostGetDevicePointer(&dp, s->flag_h, 0) == cudaSuccess) {
      *s->flag_h = 0;
      s->flag_d = reinterpret_cast<CUdeviceptr>(dp);
    } else {
      cudaGetLastError();
      if (s->flag_h) cudaFreeHost(s->flag_h);
      s->flag_h = nullptr;
    }
  }
  if (ok) {
    s->st = static_cast<cudaStream_t>(sfac_get_stream(s->h));
    s->ncap = ncap;
    // a first run with no atoms sizes the handle's buffers (no allocation may
    // happen inside the capture), then the request work is captured once
    memset(s->h_blk, 0, sizeof(double) * kHdr);
    memcpy(s->h_blk, L, sizeof(double) * 6);
    ok = cudaMemcpyAsync(s->d_blk, s->h_blk, sizeof(double) * kHdr, cudaMemcpyHostToDevice, s->st) == cudaSuccess &&
         enqueue_request_work(s) && cudaStreamSynchronize(s->st) == cudaSuccess;
    if (ok && sv->graphs) {
      cudaGraph_t gr = nullptr;
      ok = cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      const bool work = ok && enqueue_request_work(s);
      ok = ok && cudaStreamEndCapture(s->st, &gr) == cudaSuccess && work &&
           cudaGraphInstantiate(&s->graph, gr, 0) == cudaSuccess;
      if (gr) cudaGraphDestroy(gr);
    }
  }
  if (!ok) {
    cudaGetLastError();
    destroy_slot(s);
    return nullptr;
  }
  memcpy(s->K, K, sizeof(s->K));
  s->order = order;
  s->beta = beta;
  s->max_m = max_m;
  s->bytes = slot_bytes(K, ncap);
  sv->created++;
  return s;
}

bool evict_one(Server *sv) {
  int best = -1;
  for (int i = 0; i < (int)sv->slots.size(); i++) {
    Slot *s = sv->slots[i];
    if (!s->busy && (best < 0 || s->last < sv->slots[best]->last)) best = i;
  }
  if (best < 0) return false;
  sv->used -= sv->slots[best]->bytes;
  destroy_slot(sv->slots[best]);
  sv->slots.erase(sv->slots.begin() + best);
  sv->evicted++;
  return true;
}

// An idle slot for the shape, created (evicting idle slots) when none is
// free.  rc: 0 found, 1 no slot or memory free now, 2 error.
Slot *admit(Server *sv, long long id, int n, const int K[3], int order, double beta, double max_m,
            const double L[6], int &rc) {
  rc = 0;
  Slot *s = nullptr;
  for (Slot *c : sv->slots)
    if (!c->busy && c->K[0] == K[0] && c->K[1] == K[1] && c->K[2] == K[2] && c->order == order &&
        c->beta == beta && c->max_m == max_m && c->ncap >= n && (!s || c->ncap < s->ncap))
      s = c;
  if (s) return s;
  const int ncap = bucket(n);
  const size_t need = slot_bytes(K, ncap);
  if (need > sv->budget) {  // can never fit, even with the pool empty
    fprintf(stderr, "spme_server: request %lld needs %zu bytes, above the pool budget %zu\n", id, need, sv->budget);
    sv->errors++;
    rc = 2;
    return nullptr;
  }
  while (sv->used + need > sv->budget)
    if (!evict_one(sv)) {
      rc = 1;  // everything resident is busy: retry after a poll
      return nullptr;
    }
  s = create_slot(sv, ncap, K, order, beta, max_m, L);
  if (!s) {
    sv->errors++;
    rc = 2;
    return nullptr;
  }
  sv->slots.push_back(s);
  sv->used += s->bytes;
  return s;
}

// Copy in (already enqueued by the caller), the request's device work, copy
// out, completion event.
bool launch_request(Server *sv, Slot *s, long long id, int n, double *out, double work) {
  bool ok = s->graph ? cudaGraphLaunch(s->graph, s->st) == cudaSuccess : enqueue_request_work(s);
  ok = ok && cudaMemcpyAsync(out, s->d_out, sizeof(double) * (7 + 4 * (size_t)n), cudaMemcpyDeviceToHost,
                             s->st) == cudaSuccess;
  ok = ok && cudaEventRecord(s->done, s->st) == cudaSuccess;
  if (ok && s->flag_h) ok = write_value32()(reinterpret_cast<CUstream>(s->st), s->flag_d, ++s->seq, 0) == CUDA_SUCCESS;
  if (!ok) {
    cudaGetLastError();
    sv->errors++;
    return false;
  }
  s->busy = true;
  s->id = id;
  s->last = ++sv->tick;
  s->work = work;
  sv->inflight++;
  sv->inflight_work += work;
  return true;
}

}  // namespace

namespace {

// Admits and launches a request whose positions (Cartesian, or fractional
// with frac) and charges are read straight from the caller's host arrays:
// header from the slot's pinned staging, three copies in.
int submit_parts(Server *sv, long long id, int n, const int K[3], int order, double beta, double max_m,
                 const double L[6], const double *x, const double *q, bool frac, double *out) {
  const double work = request_work(K, n);
  if (sv->inflight >= sv->max_inflight) return 1;
  if (sv->inflight > 0 && sv->inflight_work + work > sv->work_budget) return 3;  // a smaller one may fit
  int rc = 0;
  Slot *s = admit(sv, id, n, K, order, beta, max_m, L, rc);
  if (!s) return rc == 1 ? 3 : rc;
  // the slot is idle: the previous copy from its staging has completed
  memset(s->h_blk, 0, sizeof(double) * kHdr);
  memcpy(s->h_blk, L, sizeof(double) * 6);
  s->h_blk[6] = (double)n;
  s->h_blk[7] = frac ? 1.0 : 0.0;
  bool ok = cudaMemcpyAsync(s->d_blk, s->h_blk, sizeof(double) * kHdr, cudaMemcpyHostToDevice, s->st) == cudaSuccess;
  if (ok && n > 0)
    ok = cudaMemcpyAsync(s->d_blk + kHdr, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s->st) == cudaSuccess &&
         cudaMemcpyAsync(s->d_blk + kHdr + 3 * (size_t)n, q, sizeof(double) * n, cudaMemcpyHostToDevice, s->st) ==
             cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    sv->errors++;
    return 2;
  }
  return launch_request(sv, s, id, n, out, work) ? 0 : 2;
}

}  // namespace

extern "C" {

void *spme_server_create(int device, double budget_bytes, int max_inflight, int use_graphs) {
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    fprintf(stderr, "spme_server_create: no CUDA device %d\n", device);
    return nullptr;
  }
  Server *sv = new Server;
  sv->device = device;
  sv->budget = budget_bytes > 0 ? (size_t)budget_bytes : (size_t)8 << 30;
  sv->max_inflight = max_inflight > 0 ? max_inflight : 1;
  sv->graphs = use_graphs != 0;
  return sv;
}

void spme_server_destroy(void *p) {
  Server *sv = static_cast<Server *>(p);
  if (!sv) return;
  cudaSetDevice(sv->device);
  for (Slot *s : sv->slots) destroy_slot(s);
  delete sv;
}

int spme_server_tune(void *p, const int K[3], int order, int x_lines) {
  Server *sv = static_cast<Server *>(p);
  if (!sv) return 1;
  sv->tunes.push_back(Tune{{K[0], K[1], K[2]}, order, x_lines});
  return 0;  // applies to slots created from now on (existing graphs keep their shape)
}

int spme_server_submit(void *p, long long id, int n, const int K[3], int order, double beta, double max_m,
                       const double L[6], const double *x, const double *q, double *out) {
  Server *sv = static_cast<Server *>(p);
  if (!sv || n < 0 || !K || !L || !out || (n > 0 && (!x || !q))) return 2;
  cudaSetDevice(sv->device);
  const int rc = submit_parts(sv, id, n, K, order, beta, max_m, L, x, q, false, out);
  return rc == 3 ? 1 : rc;
}

int spme_server_submit_packed(void *p, long long id, int n, const int K[3], int order, double beta, double max_m,
                              const double *block, double *out) {
  Server *sv = static_cast<Server *>(p);
  if (!sv || n < 0 || !K || !block || !out || (int)block[6] != n) return 2;
  const double work = request_work(K, n);
  if (sv->inflight >= sv->max_inflight) return 1;
  if (sv->inflight > 0 && sv->inflight_work + work > sv->work_budget) return 1;
  cudaSetDevice(sv->device);
  int rc = 0;
  Slot *s = admit(sv, id, n, K, order, beta, max_m, block, rc);
  if (!s) return rc;
  if (cudaMemcpyAsync(s->d_blk, block, sizeof(double) * (kHdr + 4 * (size_t)n), cudaMemcpyHostToDevice, s->st) !=
      cudaSuccess) {
    cudaGetLastError();
    sv->errors++;
    return 2;
  }
  return launch_request(sv, s, id, n, out, work) ? 0 : 2;
}

int spme_server_set_work_budget(void *p, double bytes) {
  Server *sv = static_cast<Server *>(p);
  if (!sv || !(bytes > 0.0)) return 1;
  sv->work_budget = bytes;
  return 0;
}

int spme_server_poll(void *p, long long *ids, int *status, int max_ids) {
  Server *sv = static_cast<Server *>(p);
  if (!sv || !ids) return 0;
  int c = 0;
  const bool ask_events = (++sv->polls & 63u) == 0;
  for (Slot *s : sv->slots) {
    if (c >= max_ids) break;
    if (!s->busy) continue;
    cudaError_t e;
    if (s->flag_h && *reinterpret_cast<volatile uint32_t *>(s->flag_h) == s->seq) {
      std::atomic_thread_fence(std::memory_order_acquire);  // the outputs were written before the word
      e = cudaSuccess;
    } else if (s->flag_h && !ask_events) {
      continue;
    } else {
      e = cudaEventQuery(s->done);
      if (e == cudaErrorNotReady || (e == cudaSuccess && s->flag_h)) continue;  // success: its word is on its way
    }
    int st = 0;
    if (e != cudaSuccess) {  // the request's work failed: its outputs are not valid
      cudaGetLastError();
      sv->errors++;
      st = 2;
    } else {
      sv->solves++;
    }
    s->busy = false;
    sv->inflight--;
    sv->inflight_work -= s->work;
    if (sv->inflight == 0) sv->inflight_work = 0.0;  // no drift from rounding
    if (status) status[c] = st;
    ids[c++] = s->id;
  }
  return c;
}

int spme_server_stats(void *p, double *st) {
  Server *sv = static_cast<Server *>(p);
  if (!sv || !st) return 1;
  st[0] = (double)sv->slots.size();
  st[1] = (double)sv->used;
  st[2] = (double)sv->solves;
  st[3] = (double)sv->created;
  st[4] = (double)sv->evicted;
  st[5] = (double)sv->errors;
  st[6] = (double)sv->inflight;
  st[7] = (double)sv->budget;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Stream runner: a request stream through the server, native end to end.
//
// Request i (cubic box of side side[i]) sends its positions as fractional
// coordinates frac_pool[0 .. 3 n_i) and its charges q_pool[0 .. n_i) from the
// caller's host memory: they are copied in with the request (the graph turns
// them into x = s * side in FP64 on the device), so no host thread rewrites
// inputs per request.  The loop submits requests in arrival order once they
// have arrived and a slot (or memory for one) is free under the in-flight
// limit and the work budget -- a request that does not fit the budget yet
// is passed by later arrived ones that do (up to 64 waiting), so small solves
// fill the GPU beside the large ones -- polls completions, and records each
// latency from arrival to the poll that saw it complete.  Outputs land in
// pinned buffers taken from a free list (one more than the in-flight limit).
extern "C" int spme_server_run_stream(void *p, int nreq, const int *n, const int *K, const int *order,
                                      const double *beta, const double *max_m, const double *side,
                                      const double *arrival, const double *frac_pool, const double *q_pool,
                                      double *latency, double *wall, double *loop_stats) {
  Server *sv = static_cast<Server *>(p);
  if (!sv || nreq < 0 || !n || !K || !order || !beta || !max_m || !side || !arrival || !frac_pool || !q_pool ||
      !latency || !wall)
    return 1;
  cudaSetDevice(sv->device);
  int nmax = 1;
  for (int i = 0; i < nreq; i++) nmax = n[i] > nmax ? n[i] : nmax;
  const int R = sv->max_inflight + 1;
  const size_t out_words = 8 + 4 * (size_t)nmax;
  std::vector<double *> bout(R, nullptr);
  bool ok = true;
  for (int b = 0; b < R && ok; b++) ok = cudaMallocHost((void **)&bout[b], sizeof(double) * out_words) == cudaSuccess;
  std::vector<int> free_out;  // output buffers not held by a request in flight
  for (int b = R - 1; b >= 0; b--) free_out.push_back(b);
  std::vector<int> out_of(nreq, -1);
  std::vector<int> pending;  // arrived, not yet submitted, in arrival order
  constexpr int kLookahead = 64;  // how far a request may be passed by later, smaller ones
  std::vector<long long> ids(1024);
  std::vector<int> status(1024);
  int next = 0, done = 0, rc = 0;
  const auto t0 = std::chrono::steady_clock::now();
  auto elapsed = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
  double t_submit = 0.0, t_poll = 0.0, n_poll = 0.0, n_submit = 0.0;
  while (ok && done < nreq) {
    const double tp = loop_stats ? elapsed() : 0.0;
    const int c = spme_server_poll(sv, ids.data(), status.data(), (int)ids.size());
    if (loop_stats) {
      t_poll += elapsed() - tp;
      n_poll += 1.0;
    }
    if (c > 0) {
      const double now = elapsed();
      for (int k = 0; k < c; k++) {
        const long long id = ids[k];
        if (id < 0 || id >= nreq) continue;  // not one of this stream's requests
        if (status[k] != 0) rc = 2;
        latency[id] = now - arrival[id];
        free_out.push_back(out_of[id]);
        done++;
      }
    }
    if (rc) break;
    const double now = elapsed();
    while (next < nreq && arrival[next] <= now && (int)pending.size() < kLookahead) pending.push_back(next++);
    // in arrival order; a request that does not fit the work budget (or has
    // no idle slot) is passed by later ones that do
    for (size_t j = 0; j < pending.size() && !free_out.empty();) {
      const int i = pending[j];
      const double L[6] = {side[i], side[i], side[i], 0.0, 0.0, 0.0};
      const int b = free_out.back();
      const double ts = loop_stats ? elapsed() : 0.0;
      const int r = submit_parts(sv, i, n[i], K + 3 * (size_t)i, order[i], beta[i], max_m[i], L, frac_pool, q_pool,
                                 true, bout[b]);
      if (loop_stats) {
        t_submit += elapsed() - ts;
        n_submit += 1.0;
      }
      if (r == 1) break;  // the in-flight limit: nothing else fits either
      if (r == 3) {
        j++;
        continue;
      }
      if (r != 0) {
        rc = 2;
        break;
      }
      free_out.pop_back();
      out_of[i] = b;
      pending.erase(pending.begin() + j);
    }
    if (rc) break;
  }
  *wall = elapsed();
  if (loop_stats) {
    loop_stats[0] = t_submit;
    loop_stats[1] = t_poll;
    loop_stats[2] = n_submit;
    loop_stats[3] = n_poll;
  }
  for (Slot *s : sv->slots)  // nothing may still write into the ring buffers
    if (s->st) cudaStreamSynchronize(s->st);
  for (int b = 0; b < R; b++)
    if (bout[b]) cudaFreeHost(bout[b]);
  if (!ok) return 2;
  return rc;
}
