"""Serving SPME solves with continuous batching on one GPU.

``SpmeServer`` wraps the native serving runtime of libsfac.so
(``spme_server_*`` in include/sfac.h): a persistent pool of solver slots with
resident grids, moduli and twiddles, admission by device memory footprint,
one stream per slot so that admitted requests overlap on the GPU, and one
captured CUDA graph per slot that takes each request's box on the device.

``SpmeServer.run_stream_native`` serves a whole request stream in native code
(each request's positions and charges are copied in from the caller's memory
with the request; the serving loop submits, polls and records latency from
arrival to completion).
``run_stream`` drives the same server from Python, request by request, and
can keep outputs (the tests use it).  ``run_plain`` is the baseline: the plain
one-solve-per-launch path -- one request at a time through the same runner
and graphs, each waited for before the next.  ``autotune`` picks, per (grid,
order) shape, the x-FFT lines per CTA from per-stage CUDA-event timings.
"""
from __future__ import annotations

import ctypes
import math
import statistics
import time
from collections import deque
from ctypes import POINTER, c_double, c_float, c_int, c_longlong, c_ulong, c_void_p

import numpy as np

from . import ewald as _ew

_dbl6 = np.ctypeslib.ndpointer(np.float64, shape=(6,), flags="C_CONTIGUOUS")
_int3 = np.ctypeslib.ndpointer(np.int32, shape=(3,), flags="C_CONTIGUOUS")


def _lib():
    _, _, lib = _ew.describe_sfac()
    if not getattr(lib, "_serve_declared", False):
        lib.spme_server_create.argtypes = [c_int, c_double, c_int, c_int]
        lib.spme_server_create.restype = c_void_p
        lib.spme_server_destroy.argtypes = [c_void_p]
        lib.spme_server_destroy.restype = None
        lib.spme_server_submit.argtypes = [c_void_p, c_longlong, c_int, _int3, c_int, c_double, c_double, _dbl6,
                                           c_void_p, c_void_p, c_void_p]
        lib.spme_server_submit.restype = c_int
        lib.spme_server_poll.argtypes = [c_void_p, POINTER(c_longlong), POINTER(c_int), c_int]
        lib.spme_server_poll.restype = c_int
        lib.spme_server_tune.argtypes = [c_void_p, _int3, c_int, c_int]
        lib.spme_server_tune.restype = c_int
        lib.spme_server_set_work_budget.argtypes = [c_void_p, c_double]
        lib.spme_server_set_work_budget.restype = c_int
        lib.spme_server_stats.argtypes = [c_void_p, POINTER(c_double)]
        lib.spme_server_stats.restype = c_int
        lib.spme_server_run_stream.argtypes = [c_void_p, c_int] + [c_void_p] * 9 + [c_void_p, c_void_p, c_void_p]
        lib.spme_server_run_stream.restype = c_int
        lib.sfac_set_tuning.argtypes = [c_void_p, c_int, c_int]
        lib.sfac_set_tuning.restype = c_int
        lib.sfac_solve_device_timed.argtypes = [c_void_p, c_int] + [c_void_p] * 5 + [POINTER(c_float)]
        lib.sfac_solve_device_timed.restype = c_int
        lib.sfac_footprint_bytes.argtypes = [_int3, c_int]
        lib.sfac_footprint_bytes.restype = c_ulong
        lib._serve_declared = True
    return lib


class Request:
    """One solve request: host FP64 positions (n, 3), charges (n), box L (6),
    grid K, B-spline order, Ewald beta and cutoff max_m."""

    __slots__ = ("id", "n", "K", "order", "beta", "max_m", "L", "x", "q")

    def __init__(self, rid, x, q, L, K, order, beta, max_m):
        self.id = int(rid)
        self.x, self.q = x, q
        self.n = int(q.shape[0])
        self.L = np.ascontiguousarray(L, dtype=np.float64)
        self.K = np.ascontiguousarray(K, dtype=np.int32)
        self.order, self.beta, self.max_m = int(order), float(beta), float(max_m)


class SpmeServer:
    def __init__(self, device=0, budget_bytes=32 << 30, max_inflight=32, graphs=True):
        self.lib = _lib()
        self.h = self.lib.spme_server_create(int(device), float(budget_bytes), int(max_inflight), 1 if graphs else 0)
        if not self.h:
            raise RuntimeError("spme_server_create failed (no CUDA device?)")
        self._ids = (c_longlong * 1024)()
        self._status = (c_int * 1024)()

    def close(self):
        if self.h:
            self.lib.spme_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, req: Request, xbuf, out):
        """0 admitted, 1 busy (retry after poll), 2 error.  xbuf/out: pinned
        numpy arrays holding the positions and receiving [E, vir, dx, phi]."""
        return self.lib.spme_server_submit(self.h, req.id, req.n, req.K, req.order, req.beta, req.max_m, req.L,
                                           xbuf.ctypes.data, req.q.ctypes.data, out.ctypes.data)

    def poll(self):
        """Completed requests as (id, status): status 0 means the output
        buffer holds the results, 2 that the request's GPU work failed."""
        k = self.lib.spme_server_poll(self.h, self._ids, self._status, 1024)
        return [(self._ids[i], self._status[i]) for i in range(k)]

    def run_stream_native(self, specs, arrivals, pool, qpool):
        """Serves the request stream `specs` (cfg5-style dicts: n, side, K,
        order, beta, max_m; request i sends the fractional positions
        pool[:n] of its cubic box of side `side` and charges qpool[:n])
        arriving at `arrivals` seconds (None: all at once) entirely in native
        code (spme_server_run_stream).  Returns (latencies in s, wall s)."""
        m = len(specs)
        n = np.ascontiguousarray([sp["n"] for sp in specs], dtype=np.int32)
        K = np.ascontiguousarray([sp["K"] for sp in specs], dtype=np.int32).reshape(-1)
        order = np.ascontiguousarray([sp["order"] for sp in specs], dtype=np.int32)
        beta = np.ascontiguousarray([sp["beta"] for sp in specs], dtype=np.float64)
        max_m = np.ascontiguousarray([sp["max_m"] for sp in specs], dtype=np.float64)
        side = np.ascontiguousarray([sp["side"] for sp in specs], dtype=np.float64)
        arr = np.zeros(m) if arrivals is None else np.ascontiguousarray(arrivals, dtype=np.float64)
        lat = np.zeros(m)
        wall = np.zeros(1)
        self.loop_stats = np.zeros(4)
        rc = self.lib.spme_server_run_stream(self.h, m, *(a.ctypes.data for a in (n, K, order, beta, max_m, side, arr,
                                                                                   pool, qpool)),
                                             lat.ctypes.data, wall.ctypes.data, self.loop_stats.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"spme_server_run_stream failed ({rc})")
        return lat, float(wall[0])

    def set_work_budget(self, nbytes):
        """Admission by working set (spme_server_set_work_budget)."""
        if self.lib.spme_server_set_work_budget(self.h, float(nbytes)) != 0:
            raise ValueError("bad work budget")

    def tune(self, K, order, x_lines):
        self.lib.spme_server_tune(self.h, np.asarray(K, np.int32), int(order), int(x_lines))

    def stats(self):
        s = (c_double * 8)()
        self.lib.spme_server_stats(self.h, s)
        keys = ["slots", "bytes", "solves", "created", "evicted", "errors", "inflight", "budget"]
        return {k: s[i] for i, k in enumerate(keys)}


def _pinned(shape):
    import torch

    return torch.empty(shape, dtype=torch.float64).pin_memory().numpy()


class _Buffers:
    """Pinned host staging: positions and outputs per in-flight request."""

    def __init__(self, count, nmax):
        self.free = [(_pinned((nmax, 3)), _pinned(7 + 4 * nmax)) for _ in range(count)]


def run_stream(server: SpmeServer, requests, arrivals=None, make_x=None, max_inflight=32, keep=None,
               timeout_s=600.0):
    """Serves `requests` (list of Request) arriving at `arrivals` seconds
    (None: all at once).  make_x(req, buf) fills the pinned position buffer
    (default: copies req.x).  keep: ids whose outputs are returned.
    Returns (latencies in s, wall time, outputs dict)."""
    nmax = max(r.n for r in requests)
    bufs = _Buffers(max_inflight, max(nmax, 1))
    total = len(requests)
    arr = np.zeros(total) if arrivals is None else np.asarray(arrivals, dtype=np.float64)
    lat = np.zeros(total)
    outs = {}
    pending = deque()
    inflight = {}
    nxt = 0
    done = 0
    t0 = time.perf_counter()
    while done < total:
        now = time.perf_counter() - t0
        if now > timeout_s:
            raise TimeoutError(f"serving stream exceeded {timeout_s} s ({done}/{total} done)")
        while nxt < total and arr[nxt] <= now:
            pending.append(nxt)
            nxt += 1
        ids = server.poll()
        if ids:
            tdone = time.perf_counter() - t0
            for rid, st in ids:
                i, xb, ob = inflight.pop(rid)
                if st != 0:
                    raise RuntimeError(f"request {rid} failed on the GPU (status {st})")
                lat[i] = tdone - arr[i]
                if keep is not None and rid in keep:
                    r = requests[i]
                    outs[rid] = (ob[0], ob[1:7].copy(), ob[7:7 + 3 * r.n].reshape(r.n, 3).copy(),
                                 ob[7 + 3 * r.n:7 + 4 * r.n].copy())
                bufs.free.append((xb, ob))
                done += 1
        while pending and bufs.free:
            i = pending[0]
            r = requests[i]
            xb, ob = bufs.free[-1]
            if make_x is not None:
                make_x(r, xb)
            else:
                xb[: r.n] = r.x
            rc = server.submit(r, xb, ob)
            if rc == 1:
                break
            if rc != 0:
                raise RuntimeError(f"spme_server_submit failed for request {r.id}")
            pending.popleft()
            bufs.free.pop()
            inflight[r.id] = (i, xb, ob)
    return lat, time.perf_counter() - t0, outs


def run_plain(specs, pool, qpool, device=0, warm=True):
    """Baseline: the plain one-solve-per-launch GPU path -- one request at a
    time (copy in, its captured CUDA graph, copy out, wait) through the same
    native runner, slots and graphs as the served stream, with resident
    per-shape solvers (a first pass, untimed, creates them)."""
    server = SpmeServer(device=device, max_inflight=1, graphs=True)
    try:
        if warm:
            server.run_stream_native(specs, None, pool, qpool)
        lat, wall = server.run_stream_native(specs, None, pool, qpool)
    finally:
        server.close()
    return lat, wall


def autotune(shapes, device=0, candidates=(0, 4, 8, 16, 32), reps=3):
    """Per (K, order, n) shape: the x-FFT lines per CTA with the fastest
    convolution stage (median of `reps` CUDA-event timings).  Returns
    {(K, order): x_lines}."""
    import torch

    lib = _lib()
    out = {}
    dev = torch.device("cuda", device)
    for K, order, n in shapes:
        K = tuple(int(k) for k in K)
        L = np.array([K[0] * 0.1, K[1] * 0.1, K[2] * 0.1, 0, 0, 0], dtype=np.float64)
        s = _ew.Sfac(L.copy(), np.asarray(K), int(order))
        s.set_ewald(3.12, 6.0)
        rng = np.random.default_rng(0)
        x = torch.tensor(rng.uniform(0, 1, size=(n, 3)) * L[:3], device=dev)
        q = torch.tensor(np.where(np.arange(n) % 2 == 0, 1.0, -1.0), device=dev)
        dx = torch.empty((n, 3), dtype=torch.float64, device=dev)
        phi = torch.empty(n, dtype=torch.float64, device=dev)
        ev = torch.empty(7, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        best, best_t = 0, float("inf")
        ms = (c_float * 6)()
        for c in candidates:
            if lib.sfac_set_tuning(s._data, 1, int(c)) != 0:
                continue
            ts = []
            for _ in range(reps + 1):
                lib.sfac_solve_device_timed(s._data, n, x.data_ptr(), q.data_ptr(), dx.data_ptr(), phi.data_ptr(),
                                            ev.data_ptr(), ms)
                ts.append(ms[3])
            t = statistics.median(ts[1:])
            if t < best_t:
                best, best_t = c, t
        out[(K, int(order))] = best
        del s
    return out


def percentiles(lat):
    srt = np.sort(np.asarray(lat))
    if srt.size == 0:
        return {"p50": None, "p99": None}
    return {"p50": float(srt[int(0.5 * (srt.size - 1))] * 1e3),
            "p99": float(srt[min(srt.size - 1, int(math.ceil(0.99 * srt.size)) - 1)] * 1e3),
            "mean": float(srt.mean() * 1e3)}


def stream_benchmark(count=10000, plain_count=2000, load=0.8, max_inflight=64, device=0, tune=False,
                     budget_bytes=48 << 30, seed=5):
    """The serving-stream measurement: `count` requests (cfg5 shapes: 500 to
    200,000 atoms, 24^3 to 128^3 grids, order 4 or 6) served natively with
    continuous admission (spme_server_run_stream); capacity from a
    closed-loop pass, then Poisson arrivals at `load` x capacity for latency;
    the plain one-at-a-time path on the first `plain_count` requests.
    Returns a dict of results."""
    import collections

    import torch

    from . import configs

    specs = configs.cfg5_specs(count, seed)
    pool = _pinned((configs.CFG5_POOL_ATOMS, 3))
    pool[:] = configs.cfg5_pool(seed)
    qpool = _pinned(configs.CFG5_POOL_ATOMS)
    qpool[:] = configs.cfg5_charges(configs.CFG5_POOL_ATOMS)

    tunes = {}
    t_tune = time.perf_counter()
    if tune:
        by_shape = collections.defaultdict(list)
        for sp in specs:
            by_shape[(tuple(int(k) for k in sp["K"]), sp["order"])].append(sp["n"])
        shapes = [(K, o, int(np.median(ns))) for (K, o), ns in sorted(by_shape.items())]
        tunes = autotune(shapes, device=device)
    t_tune = time.perf_counter() - t_tune

    srv = SpmeServer(device=device, budget_bytes=budget_bytes, max_inflight=max_inflight, graphs=True)
    for (K, o), xl in tunes.items():
        srv.tune(K, o, xl)
    torch.cuda.synchronize(device)
    # warm until a pass creates no slot: every shape the stream needs at its
    # concurrency is resident (grids, plans, graphs), as in steady serving
    t_warm = 0.0
    for _ in range(6):
        c0 = srv.stats()["created"]
        _, t = srv.run_stream_native(specs, None, pool, qpool)
        t_warm += t
        if srv.stats()["created"] == c0:
            break
    _, t_cap = srv.run_stream_native(specs, None, pool, qpool)
    capacity = count / t_cap
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / (load * capacity), size=count))
    lat, t_open = srv.run_stream_native(specs, arrivals, pool, qpool)
    stats = srv.stats()
    srv.close()

    sample = specs[:plain_count]
    plat, t_plain = run_plain(sample, pool, qpool, device=device)
    plain = len(sample) / t_plain
    return {
        "requests": count,
        "capacity_solves_per_s": capacity,
        "served_solves_per_s": count / t_open,
        "offered_load": load,
        "latency_ms": percentiles(lat),
        "plain_solves_per_s": plain,
        "plain_latency_ms": percentiles(plat),
        "served_over_plain": capacity / plain,
        "max_inflight": max_inflight,
        "slots": int(stats["slots"]),
        "pool_bytes": int(stats["bytes"]),
        "errors": int(stats["errors"]),
        "warm_pass_s": t_warm,
        "autotune_s": t_tune,
        "autotuned_shapes": len(tunes),
        "mean_atoms": float(np.mean([sp["n"] for sp in specs])),
        "plain": "one request at a time through the same runner: copy in, captured CUDA graph, copy out, wait",
    }


def main(argv=None):
    """`python -m ewaldcorrel_b200.serve [--count N] [--plain N] [--load F]`:
    runs stream_benchmark on GPU 0 and prints its results as one JSON line."""
    import argparse
    import json

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--count", type=int, default=10000)
    ap.add_argument("--plain", type=int, default=2000)
    ap.add_argument("--load", type=float, default=0.8)
    ap.add_argument("--max-inflight", type=int, default=64)
    ap.add_argument("--tune", action="store_true")
    args = ap.parse_args(argv)
    t0 = time.perf_counter()
    res = stream_benchmark(count=args.count, plain_count=args.plain, load=args.load, max_inflight=args.max_inflight,
                           tune=args.tune)
    res["wall_s"] = time.perf_counter() - t0
    print(json.dumps(res))


if __name__ == "__main__":
    main()
