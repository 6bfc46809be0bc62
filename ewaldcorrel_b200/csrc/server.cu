// Serving runtime: a persistent pool of SPME solvers on one GPU with
// continuous admission.
//
// A slot is one solver handle (resident grids, B-spline moduli, FFT twiddles,
// influence tables) plus fixed device buffers for one atom-count bucket, on
// its own stream.  A request is admitted into an idle slot of its shape
// (grid, order, Ewald parameters, bucket), or a new slot while the device
// memory budget allows -- idle slots are evicted least-recently-used first.
// Admitted requests run concurrently on their slots' streams; each slot
// replays its solve as a CUDA graph (the atom count is padded to the bucket
// with zero charges, which leaves every result unchanged; box changes only
// rewrite device constants, so the graph stays valid).  Completion is
// detected by polling one event per slot.  Built only on the C ABI of
// include/sfac.h.
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/sfac.h"
#include "spme_common.cuh"

namespace {

// Padding atoms: copies of real positions (same spatial distribution, so
// the spread stays balanced) with zero charge.
__global__ void pad_atoms_kernel(double *__restrict__ x, double *__restrict__ q, int n, int ncap) {
  const int i = n + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncap) return;
  const int s = n > 0 ? i % n : 0;
  x[3 * i + 0] = n > 0 ? x[3 * s + 0] : 0.0;
  x[3 * i + 1] = n > 0 ? x[3 * s + 1] : 0.0;
  x[3 * i + 2] = n > 0 ? x[3 * s + 2] : 0.0;
  q[i] = 0.0;
}

struct Slot {
  void *h = nullptr;
  int K[3] = {0, 0, 0}, order = 0, ncap = 0;
  double beta = 0, max_m = 0;
  double L[6] = {0, 0, 0, 0, 0, 0};
  double *d_x = nullptr, *d_q = nullptr, *d_out = nullptr;  // d_out: ev (8) | dx (3 ncap) | phi (ncap)
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  long long id = -1;
  unsigned long long last = 0;
  size_t bytes = 0;
};

struct Tune {
  int K[3], order, x_lines;
};

struct Server {
  int device = 0;
  size_t budget = 0, used = 0;
  int max_inflight = 1, inflight = 0;
  bool graphs = true;
  std::vector<Slot *> slots;
  std::vector<Tune> tunes;
  unsigned long long tick = 0;
  long long solves = 0, created = 0, evicted = 0, errors = 0;
};

int bucket(int n) {
  // 256 * sqrt(2)^k rounded up to a multiple of 64
  double b = 256.0;
  while (b < n) b *= 1.4142135623730951;
  const int v = (int)b;
  return (v + 63) / 64 * 64;
}

void destroy_slot(Slot *s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->done) cudaEventDestroy(s->done);
  if (s->d_x) cudaFree(s->d_x);
  if (s->d_q) cudaFree(s->d_q);
  if (s->d_out) cudaFree(s->d_out);
  if (s->h) sfac_dtor(s->h);
  delete s;
}

Slot *create_slot(Server *sv, int ncap, const int K[3], int order, double beta, double max_m, const double L[6]) {
  Slot *s = new Slot;
  double Lc[6];
  int Kc[3] = {K[0], K[1], K[2]};
  memcpy(Lc, L, sizeof(Lc));
  s->h = sfac_ctor(Lc, Kc, order);
  bool ok = s->h != nullptr;
  ok = ok && sfac_set_ewald(s->h, beta, max_m) == 0 && sfac_set_graphs(s->h, sv->graphs ? 1 : 0) == 0;
  for (const Tune &t : sv->tunes)
    if (ok && t.K[0] == K[0] && t.K[1] == K[1] && t.K[2] == K[2] && t.order == order)
      sfac_set_tuning(s->h, SFAC_TUNE_X_LINES, t.x_lines);
  ok = ok && cudaMalloc((void **)&s->d_x, sizeof(double) * 3 * ncap) == cudaSuccess &&
       cudaMalloc((void **)&s->d_q, sizeof(double) * ncap) == cudaSuccess &&
       cudaMalloc((void **)&s->d_out, sizeof(double) * (8 + 4 * (size_t)ncap)) == cudaSuccess &&
       cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    destroy_slot(s);
    return nullptr;
  }
  s->st = static_cast<cudaStream_t>(sfac_get_stream(s->h));
  memcpy(s->K, K, sizeof(s->K));
  s->order = order;
  s->ncap = ncap;
  s->beta = beta;
  s->max_m = max_m;
  memcpy(s->L, L, sizeof(s->L));
  s->bytes = sfac_footprint_bytes(K, ncap) + sizeof(double) * (8 + 8 * (size_t)ncap);
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
  for (Slot *s : sv->slots)
    if (s->K[0] == K[0] && s->K[1] == K[1] && s->K[2] == K[2] && s->order == order && !s->busy)
      sfac_set_tuning(s->h, SFAC_TUNE_X_LINES, x_lines);
  return 0;
}

int spme_server_submit(void *p, long long id, int n, const int K[3], int order, double beta, double max_m,
                       const double L[6], const double *x, const double *q, double *out) {
  Server *sv = static_cast<Server *>(p);
  if (!sv || n < 0 || !K || !L || !out || (n > 0 && (!x || !q))) return 2;
  if (sv->inflight >= sv->max_inflight) return 1;
  cudaSetDevice(sv->device);
  // an idle slot of this shape with the smallest sufficient bucket
  Slot *s = nullptr;
  for (Slot *c : sv->slots)
    if (!c->busy && c->K[0] == K[0] && c->K[1] == K[1] && c->K[2] == K[2] && c->order == order &&
        c->beta == beta && c->max_m == max_m && c->ncap >= n && (!s || c->ncap < s->ncap))
      s = c;
  if (!s) {
    const int ncap = bucket(n);
    const size_t need = sfac_footprint_bytes(K, ncap) + sizeof(double) * (8 + 8 * (size_t)ncap);
    if (need > sv->budget) {  // can never fit, even with the pool empty
      fprintf(stderr, "spme_server_submit: request %lld needs %zu bytes, above the pool budget %zu\n", id, need,
              sv->budget);
      sv->errors++;
      return 2;
    }
    while (sv->used + need > sv->budget)
      if (!evict_one(sv)) return 1;  // everything resident is busy: retry after a poll
    s = create_slot(sv, ncap, K, order, beta, max_m, L);
    if (!s) {
      sv->errors++;
      return 2;
    }
    sv->slots.push_back(s);
    sv->used += s->bytes;
  }
  if (memcmp(s->L, L, sizeof(s->L)) != 0) {  // new box: device constants and row tables only
    double Lc[6];
    memcpy(Lc, L, sizeof(Lc));
    set_L(s->h, Lc);
    if (sfac_set_ewald(s->h, beta, max_m) != 0) {
      sv->errors++;
      return 2;
    }
    memcpy(s->L, L, sizeof(s->L));
  }
  bool ok = true;
  if (n > 0) {
    ok = cudaMemcpyAsync(s->d_x, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s->st) == cudaSuccess &&
         cudaMemcpyAsync(s->d_q, q, sizeof(double) * n, cudaMemcpyHostToDevice, s->st) == cudaSuccess;
  }
  if (ok && s->ncap > n) pad_atoms_kernel<<<(s->ncap - n + 255) / 256, 256, 0, s->st>>>(s->d_x, s->d_q, n, s->ncap);
  double *d_ev = s->d_out, *d_dx = s->d_out + 8, *d_phi = s->d_out + 8 + 3 * (size_t)s->ncap;
  ok = ok && sfac_solve_device(s->h, s->ncap, s->d_x, s->d_q, d_dx, d_phi, d_ev) == 0;
  ok = ok && cudaMemcpyAsync(out, d_ev, sizeof(double) * 7, cudaMemcpyDeviceToHost, s->st) == cudaSuccess;
  if (ok && n > 0)
    ok = cudaMemcpyAsync(out + 7, d_dx, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s->st) == cudaSuccess &&
         cudaMemcpyAsync(out + 7 + 3 * (size_t)n, d_phi, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st) ==
             cudaSuccess;
  ok = ok && cudaEventRecord(s->done, s->st) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    sv->errors++;
    return 2;
  }
  s->busy = true;
  s->id = id;
  s->last = ++sv->tick;
  sv->inflight++;
  return 0;
}

int spme_server_poll(void *p, long long *ids, int *status, int max_ids) {
  Server *sv = static_cast<Server *>(p);
  if (!sv || !ids) return 0;
  int c = 0;
  for (Slot *s : sv->slots) {
    if (c >= max_ids) break;
    if (!s->busy) continue;
    const cudaError_t e = cudaEventQuery(s->done);
    if (e == cudaErrorNotReady) continue;
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
