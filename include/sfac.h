/*
 * sfac.h -- C ABI of libsfac.so, the B200 (sm_100a) SPME reciprocal-space
 * library.
 *
 * The first block is a drop-in for the C interface of the reference
 * (frobnitzem/EwaldCorrel, sfac.hpp:194-211): same symbol names, argument
 * meanings, array layouts, state machine and error behaviour, so the
 * reference's ctypes wrapper (ewald.py:15-68) binds it unchanged.  All
 * arrays are HOST memory, FP64, C-contiguous.  Each handle owns its device
 * buffers and a CUDA stream on the device that was current at sfac_ctor.
 *
 * The second block adds entry points the reference does not have; they never
 * change the behaviour of the first block.
 */
#ifndef SFAC_B200_H
#define SFAC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- reference interface (sfac.hpp:194-211) ---------------- */

/* rad_fn must return f(r2) and store f'(r2) in *dA; info is passed through
 * (sfac.hpp:201-203). */
typedef double (*rad_fn)(double r2, double *dA, void *info);

/* Replaces sfac_ctor (sfac.hpp:196, sfac.cpp:180-183).
 * L = [ax, by, cz, bx, cx, cy] (lower-triangular box rows), K = grid size,
 * order = even B-spline order in [2, 8].  Returns NULL (never throws) on an
 * odd or out-of-range order, K < 1, a grid too large for 32-bit cell keys,
 * no CUDA device, or an allocation failure. */
void *sfac_ctor(double L[6], int K[3], int order);

/* Replaces sfac_dtor (sfac.hpp:197, sfac.cpp:185-188).  Releases only this
 * handle (the reference's global fftw_cleanup has no counterpart). */
void sfac_dtor(void *sfac);

/* Replaces sfac (sfac.hpp:198, sfac.cpp:190-193): spread the n weights w
 * at positions x (n x 3), forward FFT, divide by the B-spline moduli.
 * State becomes 0 (structure factor). */
void sfac(void *sfac, int n, const double *w, const double *x);

/* Replaces get_S (sfac.hpp:199, sfac.cpp:194-197).  Returns a host array
 * owned by the handle, valid until sfac_dtor: in state 0 the structure
 * factor as K0 x K1 x ldim x 2 doubles (ldim = K2/2+1); in state 1 the real
 * potential grid as K0 x K1 x (2*ldim) doubles (first K2 of each row used).
 * The array is refreshed from the device at each call. */
double *get_S(void *sfac);

/* Replaces set_L (sfac.hpp:205, sfac.cpp:199-202): replaces the box only;
 * the influence function is NOT recomputed. */
void set_L(void *sfac, double L[6]);

/* Replaces set_A (sfac.hpp:206, sfac.cpp:213-292): tabulates A = sum f/2 and
 * dA = sum f' m_a m_b over every m = iL n with |m| < max_m, folded onto the
 * stored half space, calling f on the host.  Returns 0, or 2 on an
 * allocation failure. */
int set_A(void *sfac, rad_fn f, double max_m, void *info);

/* Replaces en (sfac.hpp:207, sfac.cpp:304-325): iV * sum A |S|^2.
 * Needs state 0 and an influence function, else prints and returns 0. */
double en(void *sfac);

/* Replaces de1 (sfac.hpp:208, sfac.cpp:339-396): energy, virial
 * vir = [xx, yy, zz, yx, zx, zy], convolution and inverse FFT into the
 * potential grid.  Needs state 0; state becomes 1. */
double de1(void *sfac, double vir[6]);

/* Replaces de2 (sfac.hpp:209, sfac.cpp:409-483): dE/dx (n x 3) of weights
 * w at positions x (any point set).  Needs state 1. */
void de2(void *sfac, int n, const double *w, const double *x, double *dx);

/* Replaces potl (sfac.hpp:210, sfac.cpp:497-545): potential phi (n) at
 * positions x.  Needs state 1. */
void potl(void *sfac, int n, const double *x, double *phi);

/* ---------------- additions (no counterpart in the reference) ----------- */

/* Ewald influence function f(m^2) = exp(-pi^2 m^2/beta^2)/(pi m^2) with the
 * same image set as set_A(ewald_f, max_m) (ewald.py:124-132), evaluated in
 * FP64 on the device at each use instead of tabulated on the host.  Uses the
 * cell current at this call (later set_L calls do not change it, as with
 * set_A).  Returns 0. */
int sfac_set_ewald(void *sfac, double beta, double max_m);

/* Structure-factor analysis over frames, on the device: what the
 * reference's run.py:27-47 does on the host (Q += |get_S()|^2 per frame) and
 * plot.py:9-32's radial binning.  No counterpart in the reference's library.
 *   sfac_sk_reset       zeroes the sum of |S|^2 and the frame count;
 *   sfac_sk_accumulate  after sfac: adds |S(m)|^2 of every stored mode (FP64);
 *   sfac_sk_get         copies the sum (K0 x K1 x ldim doubles, get_S's
 *                       mode order) and the frame count;
 *   sfac_sk_radial      sums and counts of the stored modes in nbins bins of
 *                       |k| = 2 pi |m| (m the reciprocal vector of the
 *                       signed x/y indices and the stored z index, m . x =
 *                       n . s in the current box), width kmax/nbins; modes
 *                       beyond kmax are left out.
 * Return 0, 1 on bad arguments or state, 2 on a CUDA error. */
int sfac_sk_reset(void *sfac);
int sfac_sk_accumulate(void *sfac);
int sfac_sk_get(void *sfac, double *out, long long *frames);
int sfac_sk_radial(void *sfac, int nbins, double kmax, double *sums, double *counts);

/* Cross-correlations of D densities, on the device: what the reference's
 * gmx_ewald.py:76-95 does on the host (Q[i] = S after each density's sfac;
 * C[k] += Q[i] conj(Q[j]) for i <= j, k counting the pairs in row order).
 * No counterpart in the reference's library.
 *   sfac_xc_reset       D slots (1..64), zeroes the sums and the frame count;
 *   sfac_xc_store       after sfac: keeps this density's S in slot i;
 *   sfac_xc_accumulate  adds Q[i] conj(Q[j]) of the stored slots (FP64);
 *   sfac_xc_get         copies sum k (K0 x K1 x ldim complex as interleaved
 *                       doubles, get_S's mode order) and the frame count.
 * Return 0, 1 on bad arguments or state, 2 on a CUDA error. */
int sfac_xc_reset(void *sfac, int D);
int sfac_xc_store(void *sfac, int i);
int sfac_xc_accumulate(void *sfac);
int sfac_xc_get(void *sfac, int k, double *out, long long *frames);

/* Real-space Ewald term and corrections beside the reciprocal sum: with the
 * Ewald influence function of splitting parameter eta (sfac_set_ewald, or
 * ewald.py's ewald_f), E_recip + out[0] + out[1] + out[2] is the full Ewald
 * energy (CGS) and does not depend on eta (notes.tex:68-79 gives E_self;
 * E_real is the erfc complement of f, E_net the neutralising background).
 *   out[0] E_real = 1/2 sum_{i != j, r < rcut} q_i q_j erfc(eta r) / r
 *          (minimum image; rcut <= half the smallest box width),
 *   out[1] E_self = -eta/sqrt(pi) sum q^2,
 *   out[2] E_net  = -pi (sum q)^2 / (2 V eta^2),
 *   out[3..8] virial of E_real in de1's convention ([xx,yy,zz,yx,zx,zy]),
 *   out[9] virial of E_net (add to xx, yy and zz).
 * dx (n x 3, may be null): dE_real/dx.  Host arrays; uses the handle's
 * current box.  Returns 0, 1 on bad arguments, 2 on a CUDA error.
 * No counterpart in the reference (its notes give the correction only). */
int sfac_real_space(void *sfac, int n, const double *w, const double *x, double eta, double rcut, double out[10],
                    double *dx);
/* The same on device arrays (out: 10 device doubles), enqueued on the
 * handle's stream without synchronising. */
int sfac_real_space_device(void *sfac, int n, const double *x, const double *w, double eta, double rcut, double *out,
                           double *dx);

/* Any radial influence function on the device, in place of set_A's host
 * callback (sfac.hpp:201-203): f(m^2) and f'(m^2) sampled by the caller at
 * m^2 = k m2max/(nt-1), k = 0..nt-1, are interpolated (cubic Hermite in m^2,
 * FP64) over the same images set_A visits (|m| < max_m, max_m^2 <= m2max) and
 * tabulated as set_A's A and dA.  Like set_A, later box changes do not
 * re-tabulate.  Returns 0, 1 on bad arguments, 2 or 3 on a CUDA error.
 * No counterpart in the reference (set_A evaluates f on the host). */
int sfac_set_radial(void *sfac, int nt, const double *f, const double *df, double m2max, double max_m);

/* Last CUDA or argument error seen by this handle (0 = none), and its text. */
int sfac_last_error(void *sfac);
const char *sfac_error_string(void *sfac);

/* Device the handle runs on, and the number of kernels it has launched. */
int sfac_device(void *sfac);
long long sfac_kernel_launches(void *sfac);

/* Run all later work of this handle on `stream` (a cudaStream_t of the
 * handle's device, e.g. a torch stream); NULL restores the handle's own
 * stream.  Returns 0. */
int sfac_set_stream(void *sfac, void *stream);
void *sfac_get_stream(void *sfac);

/* One full solve on DEVICE arrays, enqueued on the handle's stream without
 * host copies or synchronisation: cell sort, spread, forward FFT, fused
 * convolution (energy + virial), inverse FFT, and the gather of dE/dx and
 * phi at the same points.  x (n*3), w (n), dx (n*3), phi (n) and
 * ev (7 doubles: E, vir xx, yy, zz, yx, zx, zy) are device pointers; dx
 * and/or phi may be NULL.  Needs an influence function (set_A or
 * sfac_set_ewald).  Leaves state 1 (get_S then returns the potential grid).
 * Returns 0, or nonzero on a bad argument or CUDA error. */
int sfac_solve_device(void *sfac, int n, const double *x, const double *w, double *dx, double *phi,
                      double *ev);

/* sfac_solve_device plus the derivative of the energy with respect to the
 * box at fixed Cartesian positions: dEdL (6 doubles, device) in the order of
 * L = [ax, by, cz, bx, cx, cy].  dx is required (dE/dx feeds the adjoint):
 *   dE/dL = lower triangle of (-V iL^T Pi - sum_a s_a (dE/dx_a)^T),
 * Pi the virial, s_a = iL^T x_a.  No counterpart in the reference. */
int sfac_solve_device_cell(void *sfac, int n, const double *x, const double *w, double *dx, double *phi,
                           double *ev, double *dEdL);

/* The same solve with CUDA events between its stages; synchronises and
 * stores the stage times in stage_ms: [0] cell sort, [1] spread, [2] forward
 * FFT, [3] convolution, [4] inverse FFT, [5] gather (milliseconds). */
int sfac_solve_device_timed(void *sfac, int n, const double *x, const double *w, double *dx,
                            double *phi, double *ev, float stage_ms[6]);

/* Stable cell sort of n atoms that allocates no device memory.  No
 * counterpart in the reference: it serves host programs that cannot let a
 * library allocate device memory (the device is already given to their own
 * memory pool, or their loop must not pay the device-wide synchronisation of
 * cudaMalloc/cudaFree).  Same keys and order as sfac()'s cell sort
 * (sfac.cpp:92-111).  L (6) and K (3) are host arrays; x (n*3 doubles) is a
 * device input, keys and perm (n ints each) are device outputs: the cell key
 * and the original index of each sorted position.  Work is enqueued on
 * `stream` (NULL: the default stream); results are valid once it completes.
 * All scratch lives in one fixed device array per GPU (at most 65,536 atoms,
 * held until the process exits); larger n is rejected with return code 1.
 * Every call on a device shares that array and leaves its contents behind,
 * so calls whose GPU work overlaps (other streams or threads) race.  The
 * first call on a device looks up the array's device address with that
 * device current; make it before any stream capture begins.  That address
 * is kept for the life of the process: do not call this after
 * cudaDeviceReset on that device.
 * Returns 0, 1 (bad arguments or n too large), 2 (CUDA error). */
int sfac_cell_sort_noalloc(const double L[6], const int K[3], int n, const double *x, int *keys, int *perm,
                           void *stream);

/* Replaces the box from DEVICE memory: L_dev (6 doubles on the handle's
 * device, [ax, by, cz, bx, cx, cy]) is read when the enqueued work runs, so a
 * captured CUDA graph can take a new box with each replay.  Updates the
 * device box constants (the same bits as set_L would give) and rebuilds the
 * Ewald row tables; the device solves that follow use the new box.  Needs
 * sfac_set_ewald under SFAC_TUNE_EWALD_SOURCE = 2 (influence evaluated per
 * solve, no table to rebuild).  The host-side calls (sfac, en, de1, de2,
 * potl, sfac_real_space) keep the box last set on the host.  Enqueued on the
 * handle's stream without synchronising.  Returns 0, 1 (wrong influence
 * source), 2 (CUDA error).  No counterpart in the reference. */
int sfac_box_update_device(void *sfac, const double *L_dev);

/* Use (1) or bypass (0) CUDA-graph replay in sfac_solve_device*.
 * Returns 0. */
int sfac_set_graphs(void *sfac, int enable);

/* Tuning knobs chosen by an autotuner (0 restores the heuristic):
 * SFAC_TUNE_X_LINES: x-FFT lines per CTA (power of two, <= 64).
 * SFAC_TUNE_EWALD_SOURCE: 0 (default) lets sfac_set_ewald tabulate the
 *   influence function when the table stays in L2; 2 always evaluates it on
 *   the device per solve (needed by sfac_box_update_device).  Takes effect at
 *   the next sfac_set_ewald.
 * SFAC_TUNE_ZY_MODE: z/y FFT passes: 1 fused x-plane kernels (when a plane
 *   fits in shared memory), 2 two-level register passes, 3 Stockham passes.
 * Returns 0, or 1 for an unknown key or bad value. */
#define SFAC_TUNE_X_LINES 1
#define SFAC_TUNE_ZY_MODE 2
#define SFAC_TUNE_EWALD_SOURCE 3
int sfac_set_tuning(void *sfac, int key, int value);

/* Estimated device + pinned-host bytes of a handle with grid K solving n
 * atoms (for admission by memory footprint). */
unsigned long sfac_footprint_bytes(const int K[3], int n);

/* ---- serving runtime (server.cu) ----------------------------------------
 * A persistent solver pool on one GPU.  Requests (host FP64 arrays) are
 * admitted into slots -- one handle with resident grids, moduli and twiddles
 * and fixed buffers per (grid, order, Ewald parameters, atom-count bucket) --
 * while the pool's device-memory budget allows (idle slots are evicted
 * least-recently-used first); each slot runs on its own stream, so requests
 * overlap on the GPU.  Each request's box may differ: the slot takes it on
 * the device (sfac_box_update_device), so one captured CUDA graph per slot
 * serves every request: copy in, graph launch, copy out, event.  Atoms are
 * padded to the bucket size with zero charges (no effect on results).  out
 * receives [E, vir(6), dE/dx (3n), phi (n)] once spme_server_poll has
 * reported the request id; the host arrays must stay untouched until then
 * (pinned memory makes the copies asynchronous).  Returns of submit: 0
 * admitted, 1 no slot or memory free now (poll, then retry), 2 error.
 * Not thread-safe: one host thread drives a server.  No counterpart in the
 * reference (its library solves one system per handle). */
void *spme_server_create(int device, double budget_bytes, int max_inflight, int use_graphs);
void spme_server_destroy(void *server);
int spme_server_submit(void *server, long long id, int n, const int K[3], int order, double beta, double max_m,
                       const double L[6], const double *x, const double *q, double *out);
/* The same request as one packed host block of 16 + 4n doubles:
 * [L(6), n, f, 8 unused | x (3n) | q (n)], f = 1 when x holds fractional
 * coordinates of the box (else 0); one copy in instead of three. */
int spme_server_submit_packed(void *server, long long id, int n, const int K[3], int order, double beta,
                              double max_m, const double *block, double *out);
/* Completed requests: up to max_ids ids, each with its status (0: out holds
 * the results; 2: the request's GPU work failed and out is not valid).
 * status may be NULL.  Returns the number of ids written. */
int spme_server_poll(void *server, long long *ids, int *status, int max_ids);
/* Admission by working set: a request waits (submit returns 1) while the
 * requests in flight plus it would hold more than `bytes` of grids and atom
 * buffers, unless nothing is in flight.  Concurrent solves whose working
 * sets outgrow the L2 cache all run slower; the default is 256 MB. */
int spme_server_set_work_budget(void *server, double bytes);
/* Sets x-FFT lines per CTA for slots of grid K and order created from now on
 * (autotuner result). */
int spme_server_tune(void *server, const int K[3], int order, int x_lines);
/* stats[0..7] = slots, bytes in use, solves, slots created, slots evicted,
 * errors, in flight, budget. */
int spme_server_stats(void *server, double *stats);
/* A whole request stream, served natively (the serving benchmark): request
 * i (ids 0..nreq-1, in arrival order) has n[i] atoms in a cubic box of side
 * side[i], its positions given as fractional coordinates frac_pool[0 ..
 * 3 n[i]) (copied in with the request and turned into x = s * side on the
 * device) and its charges q_pool[0 .. n[i]), grid K[3i..3i+2], order[i],
 * beta[i], max_m[i]; it arrives at arrival[i] seconds after the start (0: all
 * at once).  The loop submits in arrival order within the server's
 * in-flight limit and work budget (a request that does not fit the budget
 * yet is passed by later arrived ones that do, up to 64 waiting), polls,
 * and stores latency[i] = completion -
 * arrival (seconds) and the wall time.  frac_pool and q_pool should be
 * pinned.  loop_stats (4 doubles, may be NULL): seconds the loop spent in
 * submissions and in polls, submissions tried, polls.  Returns 0, 1 bad
 * arguments, 2 failure. */
int spme_server_run_stream(void *server, int nreq, const int *n, const int *K, const int *order, const double *beta,
                           const double *max_m, const double *side, const double *arrival, const double *frac_pool,
                           const double *q_pool, double *latency, double *wall, double *loop_stats);

/* Debug views (copies to host; for parity tests).
 * sfac_debug_sort: cell keys and original indices in sorted order (n each)
 *   of the last sfac call.
 * sfac_debug_spread: the spread grid of the last sfac call (K0*K1*K2 float),
 *   recomputed from the stored sorted atoms. */
int sfac_debug_sort(void *sfac, int n, int *keys, int *perm);
/* Test hook: the nth device allocation of the library from now on (handles
 * and serving slots) fails as if the device were out of memory, once; 0
 * disarms.  Lets tests drive the allocation-failure paths (sfac_ctor
 * returning NULL, set_A returning 2, spme_server_submit returning 2) without
 * exhausting a GPU.  Returns 0. */
int sfac_debug_fail_alloc(int nth);
/* Index-checking build (libsfac_check.so, compiled with -DSPME_CHECK): the
 * kernels test their grid, bucket, atom and table indices; a failed check
 * records (site << 40 | index) in its module's error word and skips the
 * access instead of trapping.
 * sfac_check_enabled: 1 in the checking build, 0 in the product build.
 * sfac_check_take: after a device synchronize, reads and clears every
 *   module's word; returns 0 if no check failed since the last call, else
 *   the first failing module (1 sort, 2 spread, 3 gather, 4 FFT and
 *   convolution, 5 serving, 6 C API) with its word in *word (may be NULL);
 *   -1 if the device reports an error.
 * sfac_check_selftest: runs one check that must fail (its store stays inside
 *   its buffer either way) and returns 0 if the word came back as expected,
 *   1 if not, 2 on allocation failure, -1 in the product build. */
int sfac_check_enabled(void);
int sfac_check_take(unsigned long long *word);
int sfac_check_selftest(void);
int sfac_debug_spread(void *sfac, float *grid);

#ifdef __cplusplus
}
#endif

#endif /* SFAC_B200_H */
