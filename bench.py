"""SPME reciprocal-space benchmark on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (default ``--workload triclinic``): the largest single-GPU system,
1,048,576 charges N(0, 0.5^2) in a triclinic cell (a=b=c=20 nm, gamma=60
deg), 256^3 grid, B-spline order 6, Ewald beta 3.5 nm^-1, seeded synthetic
data; ``--workload water`` takes the 98,304-atom water box (96^3, order 4)
instead.  One step = one full reciprocal solve: cell sort, spread, forward
FFT, convolution with energy and virial, inverse FFT, and the gather of
forces (dE/dx) and potentials at every atom.

Metric: solves/s (whole job; replicas on N GPUs -- the path does not shard).
``value`` is timed with CUDA events on the launching stream with inputs
resident in HBM and the L2 flushed (256 MiB write) before every step; ``e2e``
is the same metric through the reference-compatible C API (sfac, de1, de2,
potl) with pinned host buffers, host<->device copies inside the timed
region.  The CPU baseline is the reference's own sfac.cpp (oracle/_ref,
compiled -O3 -fopenmp) on this host's cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOADS = {
    "water": ("water box: 98,304 atoms (32,768 rigid 3-site molecules), 10 nm cube, 96^3 grid, "
              "B-spline order 4, Ewald beta 3.12 nm^-1",
              "SPME solves/s (water box 98,304 atoms, 96^3, order 4)"),
    "triclinic": ("triclinic cell: 1,048,576 charges N(0, 0.5^2), a=b=c=20 nm, gamma=60 deg, 256^3 grid, "
                  "B-spline order 6, Ewald beta 3.5 nm^-1",
                  "SPME solves/s (1,048,576 charges, 256^3, order 6, triclinic)"),
}
DEFAULT_WORKLOAD = "triclinic"
L2_FLUSH_BYTES = 256 << 20
# The reference arm runs whole solves on the host's cores; at the 1M-atom size
# one solve takes seconds, so its timed steps stop once this many seconds of
# solves have run (each step stays one whole solve; the line says how many).
REFERENCE_BUDGET_S = float(os.environ.get("SPME_REFERENCE_BUDGET_S", "100"))


def load_workload(name):
    """The seeded system of a workload name (see WORKLOADS)."""
    from ewaldcorrel_b200 import configs

    return configs.cfg2_water() if name == "water" else configs.cfg3_triclinic()


def workload_seed(name):
    return 2 if name == "water" else 3


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ------------------------------------------------------------ clocks --
class ClockSampler:
    """SM clocks and throttle reasons sampled while the GPU works: an NVML
    polling thread (every 2 ms, so that a timed region of a few milliseconds
    still gets samples), with `nvidia-smi -lms 100` written beside it to a
    per-rank CSV as a second record when SPME_BENCH_CLOCKS_DIR names a
    folder for it."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index):
        self.index = index
        self.proc = None
        d = os.environ.get("SPME_BENCH_CLOCKS_DIR")
        self.path = os.path.join(d, f"clocks_rank{index}.csv") if d else None
        self.samples = []  # (sm_mhz, reasons bitmask)
        self.smax = None
        self._stop = None
        self._thread = None

    def _poll(self):
        import pynvml

        try:
            pynvml.nvmlInit()
            hnd = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(hnd, pynvml.NVML_CLOCK_SM))
            while not self._stop.is_set():
                sm = pynvml.nvmlDeviceGetClockInfo(hnd, pynvml.NVML_CLOCK_SM)
                rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(hnd)
                self.samples.append((float(sm), int(rs)))
                self._stop.wait(0.002)
        except Exception:
            pass

    def __enter__(self):
        import threading

        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._poll, daemon=True)
        self._thread.start()
        try:
            if self.path is None:
                raise OSError("no clocks CSV folder")
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        t0 = time.time()
        while time.time() - t0 < 5.0 and not self.samples:
            time.sleep(0.01)
        return self

    def mark(self):
        """Index of the next sample (to summarise only part of the run)."""
        return len(self.samples)

    def __exit__(self, *a):
        if self._stop is not None:
            self._stop.set()
            self._thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, start=0, end=None):
        smp = self.samples[start:end]
        if not smp:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["unsampled"], "samples": 0}
        reasons = sorted(n for n, bit in self.REASONS.items() if any(r & bit for _, r in smp))
        return {"sm_mhz": statistics.median(s for s, _ in smp), "sm_max_mhz": self.smax, "reasons": reasons,
                "samples": len(smp), "source": "NVML, 2 ms polling during the timed steps"}


# ------------------------------------------------- algorithmic bytes --
def algorithmic_bytes(n, K):
    """Algorithmic HBM bytes per stage of one solve (FP64 atom I/O, FP32
    grids): inputs read once by the spread and once by the gather, outputs
    written once; spread writes the real grid G, R2C reads G and writes the
    half-complex grid H, the convolution reads and writes H, C2R reads H and
    writes G, the gather reads G."""
    K0, K1, K2 = K
    G = 4 * K0 * K1 * K2
    H = 8 * K0 * K1 * (K2 // 2 + 1)
    atom_in = n * (3 * 8 + 8)
    atom_out = n * (3 * 8 + 8)
    return {
        "cell_sort": atom_in,
        "spread": G,
        "fft_forward": G + H,
        "convolution": 2 * H,
        "fft_inverse": H + G,
        "gather": G + atom_in + atom_out,
        "solve_total": 2 * atom_in + atom_out + 4 * G + 2 * H,
    }


# DRAM bytes (read + write) per launch of each stage's kernels, from ncu
# captures of a plain solve (cold caches; summaries in profiles/).  Writes
# that stay in the 126 MB L2 past the kernel's end are not counted.  At 256^3
# the sort's figure is from profiles/dram_sort_triclinic1m.md, the spread's
# from profiles/ncu_full_spread_triclinic1m.md, the x pass's and the gather's
# from profiles/ncu_full_gather_x2_triclinic1m.md, the z/y passes' from
# profiles/dram_per_kernel_water_triclinic_fft_gather.md; the water box's from
# profiles/dram_per_kernel_water.md.  None: not captured for the current
# kernels.
NCU_TRAFFIC = {
    "water": {"cell_sort": 7.48e6, "spread": 2.33e6, "fft_forward": 7.30e6, "convolution": 28.99e6,
              "fft_inverse": 7.38e6, "gather": 6.70e6},
    "triclinic": {"cell_sort": 119.30e6, "spread": 44.54e6, "fft_forward": 163.58e6, "convolution": 162.71e6,
                  "fft_inverse": 165.67e6, "gather": 160.72e6},
}
# Kernels of each stage (the roofline is reported for the longest stage that
# is a single kernel launch).
STAGE_KERNELS = {
    "cell_sort": "key_count + tile_sum + cell_offsets + cell_scatter + cell_fixup (+ memset)",
    "spread": "spread_kernel",
    "fft_forward": "fft_zr2c2_kernel + fft_y2_kernel<-1>",
    "convolution": "fft_x2_kernel<XM_FWD_CONV_INV> (x FFT, Ewald convolution, energy/virial, inverse x FFT)",
    "fft_inverse": "fft_y2_kernel<+1> (+ energy/virial reduction) + fft_zc2r2_kernel",
    "gather": "gather_kernel (forces + potentials)",
}
SINGLE_KERNEL_STAGES = ("spread", "convolution", "gather")


def volume(L):
    """Cell volume from the 6-vector [ax, by, cz, bx, cx, cy] (lower-triangular box)."""
    return float(L[0] * L[1] * L[2])


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# -------------------------------------------------------- CPU sides --
def _load_reference_solver():
    """The reference's sfac.cpp compiled unmodified (oracle/_ref), else the
    oracle's C restatement.  Used only for the CPU baseline and the
    reference arm."""
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    from oracle import oracle as O

    if O.ref_available():
        return O.RefSfac, "reference", "reference sfac.cpp (oracle/_ref, g++ -O3 -fopenmp, FFT: project FP64 shim; FFTW unavailable)"
    return O.OracleSfac, "port", "oracle C restatement (oracle/liborc.so, gcc -O3 -fopenmp)"


def cpu_setup(cls, c):
    """Handle + influence function (setup: outside the timed solves)."""
    s = cls(c.L, np.array(c.K), c.order)
    s.set_ewald(c.beta, c.max_m)
    return s


def cpu_solve(s, c):
    s.sfac(c.q, c.x)
    vir = np.zeros(6)
    e = s.de1(vir)
    dx = np.zeros((c.n, 3))
    phi = np.zeros(c.n)
    s.de2(c.n, c.q, c.x, dx)
    s.potl(c.n, c.x, phi)
    return e, vir, dx, phi


def cpu_baseline(c, label, budget_s=20.0, max_solves=10):
    cls, kind, desc = _load_reference_solver()
    s = cpu_setup(cls, c)
    t0 = time.perf_counter()
    res = cpu_solve(s, c)
    t1 = time.perf_counter()
    times = [t1 - t0]
    while sum(times) < budget_s * 0.5 and len(times) < max_solves:
        a = time.perf_counter()
        cpu_solve(s, c)
        times.append(time.perf_counter() - a)
    s.close()
    per = statistics.median(times)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {
        "value": 1.0 / per, "unit": "solves/s", "cores": cores, "kind": kind,
        "sample": f"{len(times)} full {label} solves (sfac+de1+de2+potl, setup excluded), median {per * 1e3:.1f} ms; {desc}",
    }, res


# ------------------------------------------------------------- GPU arm --
# End-to-end timing: at least this many solves through the C API.
E2E_MIN_STEPS = 100


def max_over_ranks(ms, dist, device):
    """The largest of every rank's `ms` (each rank's own device-timed total):
    the whole job ends when its slowest rank does.  dist: torch.distributed
    with an initialised process group, or None for one rank."""
    import torch

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rate_over_ranks(units, ms_max):
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time (ms)."""
    return units / (ms_max / 1e3)


def bind_gpu_local_cpus(local_rank):
    """Binds this process to the CPUs that NVML reports as local to its GPU
    (the NUMA node of the GPU's PCIe root), so that the pinned host buffers
    of the end-to-end run and the threads that drive their copies sit on that
    node; a remote node can halve the host<->device copy rate.  Returns
    (previous affinity or None, CPUs bound)."""
    try:
        import pynvml

        pynvml.nvmlInit()
        ids = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
        if local_rank < len(ids):
            ident = ids[local_rank]
            h = (pynvml.nvmlDeviceGetHandleByUUID(ident) if ident.startswith("GPU-")
                 else pynvml.nvmlDeviceGetHandleByIndex(int(ident)))
        else:
            h = pynvml.nvmlDeviceGetHandleByIndex(local_rank)
        ncpu = os.cpu_count() or 1
        words = pynvml.nvmlDeviceGetCpuAffinity(h, (ncpu + 63) // 64)
        cpus = {64 * i + b for i, m in enumerate(words) for b in range(64) if (int(m) >> b) & 1}
        prev = os.sched_getaffinity(0)
        cpus &= prev
        if not cpus or cpus == prev:
            return None, len(prev)
        os.sched_setaffinity(0, cpus)
        return prev, len(cpus)
    except Exception:
        return None, 0


def run_b200(args, rank, world, local_rank):
    import torch

    from ewaldcorrel_b200 import ewald as ew
    from ewaldcorrel_b200.device import STAGES, SpmeSolver

    prev_cpus, bound_cpus = bind_gpu_local_cpus(local_rank)
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    c = load_workload(args.workload)
    WORKLOAD, METRIC = WORKLOADS[args.workload]
    n = c.n
    stream = torch.cuda.Stream(dev)
    solver = SpmeSolver(c.L, c.K, c.order, c.beta, c.max_m, device=local_rank, stream=stream)
    with torch.cuda.stream(stream):
        x = torch.from_numpy(c.x).to(dev)
        q = torch.from_numpy(c.q).to(dev)
        dx = torch.empty((n, 3), dtype=torch.float64, device=dev)
        phi = torch.empty(n, dtype=torch.float64, device=dev)
        ev = torch.empty(7, dtype=torch.float64, device=dev)
        flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # clocks are sampled from before the warm-up until after the e2e timing
    clk = ClockSampler(local_rank).__enter__()

    # warm-up
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            flush.zero_()
            solver.solve(x, q, dx, phi, ev)
    barrier()

    # timed region: K solves, each bracketed by events, L2 flushed between
    K = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    l0 = solver.launches()
    barrier()
    c0 = clk.mark()
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.zero_()
            starts[k].record(stream)
            solver.solve(x, q, dx, phi, ev)
            ends[k].record(stream)
    barrier()
    c1 = clk.mark()
    launches = solver.launches() - l0
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)
    total_ms_max = max_over_ranks(total_ms, dist, dev)
    value = rate_over_ranks(world * K, total_ms_max)
    srt = sorted(step_ms)
    p50 = srt[len(srt) // 2]
    p99 = srt[min(len(srt) - 1, int(math.ceil(0.99 * len(srt))) - 1)]
    ev_host = ev.cpu().numpy()

    # per-stage times (same solve with events between stages), L2 flushed
    stage_acc = {s: [] for s in STAGES}
    for _ in range(max(3, min(K, 10))):
        with torch.cuda.stream(stream):
            flush.zero_()
        st = solver.solve_timed(x, q, dx, phi, ev)
        for s_, v in st.items():
            stage_acc[s_].append(v)
    stage_ms = {s_: statistics.mean(v) for s_, v in stage_acc.items()}
    alg = algorithmic_bytes(n, c.K)
    dominant = max(SINGLE_KERNEL_STAGES, key=lambda s_: stage_ms[s_])
    peak, peak_kind = measured_peak()
    achieved = alg[dominant] / (stage_ms[dominant] / 1e3) / 1e9

    # the real-space term beside the solve (erfc pair sum, cutoff 1 nm), for
    # the record: not part of the metric
    rdx = torch.empty((n, 3), dtype=torch.float64, device=dev)
    rout = torch.empty(10, dtype=torch.float64, device=dev)
    with torch.cuda.stream(stream):
        for _ in range(3):
            solver.real_space(x, q, c.beta, 1.0, rout, rdx)
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        flush.zero_()
        r0.record(stream)
        solver.real_space(x, q, c.beta, 1.0, rout, rdx)
        r1.record(stream)
    torch.cuda.synchronize(dev)
    real_ms = r0.elapsed_time(r1)

    # end to end through the reference-compatible C API, pinned host buffers
    xh = torch.from_numpy(c.x).pin_memory().numpy()
    qh = torch.from_numpy(c.q).pin_memory().numpy()
    dxh = torch.zeros((n, 3), dtype=torch.float64).pin_memory().numpy()
    phih = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()
    sf = ew.Sfac(c.L, np.array(c.K), c.order)
    sf.set_ewald(c.beta, c.max_m)
    vir = np.zeros(6)
    for _ in range(3):
        sf.sfac(qh, xh)
        sf.de1(vir)
        sf.de2(n, qh, xh, dxh)
        sf.potl(n, xh, phih)
    e2e_ms = []
    KE = max(K, E2E_MIN_STEPS)  # host-side hiccups of a few ms would dominate a short run
    for _ in range(KE):
        flush.zero_()
        torch.cuda.synchronize(dev)
        a = time.perf_counter()
        sf.sfac(qh, xh)
        e_api = sf.de1(vir)
        sf.de2(n, qh, xh, dxh)
        sf.potl(n, xh, phih)
        e2e_ms.append((time.perf_counter() - a) * 1e3)
    clk.__exit__(None, None, None)
    clocks = clk.summary()
    clocks["window"] = "warm-up, timed steps, per-stage timing and the e2e run"
    clocks["timed_steps"] = clk.summary(c0, c1)
    e2e_value = rate_over_ranks(world * KE, max_over_ranks(sum(e2e_ms), dist, dev))

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": K,
        "warmup": args.warmup,
        "ms_per_step": total_ms_max / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (grids, FFT, spline weights); f64 (positions, cell keys, moduli, influence function, energy/virial reductions)",
        "data": f"synthetic (seeded numpy rng({workload_seed(args.workload)}); no dataset)",
        "config": {
            "workload": WORKLOAD,
            "atoms": n,
            "grid": list(c.K),
            "order": c.order,
            "beta": c.beta,
            "max_m": c.max_m,
            "parallelism": f"replicas x{world} (independent solves, no collective)",
            "l2": "flushed before every timed step (256 MiB device write, outside the step events)",
            "host_cpus": (f"bound to the {bound_cpus} CPUs local to the GPU (NVML affinity) for the GPU runs"
                          if prev_cpus is not None else "unbound"),
        },
        "latency_ms": {"p50": p50, "p99": p99, "mean": total_ms_max / K},
        "stage_ms": stage_ms,
        "stage_kernels": STAGE_KERNELS,
        "roofline": {
            "bound": "hbm",
            "kernel": f"{dominant}: {STAGE_KERNELS[dominant]}",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": NCU_TRAFFIC.get(args.workload, {}).get(dominant),
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch (profiles/)",
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6650 GB/s",
            "algorithmic_bytes": alg[dominant],
            "solve_algorithmic_bytes": alg["solve_total"],
            "solve_frac": alg["solve_total"] / (total_ms_max / K / 1e3) / 1e9 / peak,
        },
        "e2e": {
            "value": e2e_value,
            "unit": "solves/s",
            "h2d_bytes_per_step": int(n * (24 + 8) * 2 + n * 24),
            "d2h_bytes_per_step": int(n * 24 + n * 8 + 7 * 8),
            "api": "sfac + de1 + de2 + potl (reference C interface), pinned host arrays",
            "steps": KE,
            "ms_per_step_p50": statistics.median(e2e_ms),
            "ms_per_step_max": max(e2e_ms),
        },
        "gpu_launches": int(launches),
        "real_space": {"ms": real_ms, "rcut_nm": 1.0, "eta": c.beta,
                       # ordered pairs within the cutoff from the mean density
                       # (each pair is evaluated from both sides)
                       "pairs_per_s": n * (n / volume(c.L)) * (4.0 / 3.0) * math.pi * 1.0 ** 3 / (real_ms / 1e3),
                       "note": "erfc pair sum + self/background terms (sfac_real_space_device), cell sort "
                               "included; not in the metric"},
        "energy": float(ev_host[0]),
    }
    if prev_cpus is not None:
        os.sched_setaffinity(0, prev_cpus)  # the CPU baseline uses every host core
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, (e_ref, vir_ref, dx_ref, phi_ref) = cpu_baseline(c, args.workload)
        line["cpu_baseline"] = cb
        dxg = dx.cpu().numpy()
        phig = phi.cpu().numpy()
        line["accuracy_vs_reference"] = {
            "energy_rel_err": abs(float(ev_host[0]) - e_ref) / abs(e_ref),
            "force_rel_rms": float(np.sqrt(np.mean((dxg - dx_ref) ** 2) / np.mean(dx_ref ** 2))),
            "potential_rel_rms": float(np.sqrt(np.mean((phig - phi_ref) ** 2) / np.mean(phi_ref ** 2))),
            "virial_max_rel": float(np.abs(ev_host[1:] - vir_ref).max() / np.abs(vir_ref).max()),
        }
    if world == 1 and not args.no_serving:
        # the serving stream beside the solve (10,000 requests of the
        # serving workload, 500 to 200,000 atoms, 24^3 to 128^3, order 4/6):
        # served (continuous admission) vs the plain one-at-a-time path
        from ewaldcorrel_b200 import serve

        sv = serve.stream_benchmark(count=10000, plain_count=2000, device=local_rank)
        line["serving"] = {
            "workload": "10,000 requests: atoms log-uniform in [500, 200000], cubic boxes at 100 atoms/nm^3, "
                        "grids 24^3..128^3 (2/3/5-smooth, 0.1 nm), order 4 or 6, beta 3.12; Poisson arrivals at "
                        f"{sv['offered_load']:.0%} of capacity",
            "served_over_plain": sv["served_over_plain"],
            "capacity_solves_per_s": sv["capacity_solves_per_s"],
            "served_solves_per_s": sv["served_solves_per_s"],
            "latency_ms": sv["latency_ms"],
            "plain_solves_per_s": sv["plain_solves_per_s"],
            "plain": sv["plain"],
            "errors": sv["errors"],
        }
    line["clocks"] = clocks
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------ reference arm --
def run_reference(args, rank, world):
    """The reference's own CPU implementation of the solve (oracle/_ref: its
    sfac.cpp compiled unmodified; the oracle's C restatement where the
    reference was not built) on this host's cores, on the same workload,
    metric and unit as the GPU arm.  Rank 0 alone runs and prints the line.

    Each step is one whole solve (sfac + de1 + de2 + potl).  At the 1M-atom
    size a solve takes seconds, so the run is bounded: warm-up stops after
    the first solve once W solves or a tenth of REFERENCE_BUDGET_S have run,
    and the timed steps stop once K steps or REFERENCE_BUDGET_S seconds have
    run (at least one step); `steps` is the number timed, `steps_requested`
    the K asked for."""
    if rank != 0:
        return
    try:
        cls, kind, desc = _load_reference_solver()
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"CPU reference not built: {e}"}))
        return
    WORKLOAD, METRIC = WORKLOADS[args.workload]
    c = load_workload(args.workload)
    s = cpu_setup(cls, c)
    warm, t_warm = 0, 0.0
    while warm < max(0, args.warmup) and (warm == 0 or t_warm < 0.1 * REFERENCE_BUDGET_S):
        a = time.perf_counter()
        cpu_solve(s, c)
        t_warm += time.perf_counter() - a
        warm += 1
    times = []
    while len(times) < max(1, args.steps) and (not times or sum(times) < REFERENCE_BUDGET_S):
        a = time.perf_counter()
        cpu_solve(s, c)
        times.append(time.perf_counter() - a)
    s.close()
    steps = len(times)
    total = sum(times)
    value = steps / total
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    srt = sorted(times)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": steps,
        "steps_requested": args.steps,
        "warmup": warm,
        "warmup_requested": args.warmup,
        "ms_per_step": total / steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": f"synthetic (seeded numpy rng({workload_seed(args.workload)}); no dataset)",
        "config": {"workload": WORKLOAD, "atoms": c.n, "grid": list(c.K), "order": c.order, "beta": c.beta,
                   "max_m": c.max_m, "parallelism": "CPU, OpenMP threads"},
        "latency_ms": {"p50": srt[len(srt) // 2] * 1e3, "p99": srt[-1] * 1e3},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": kind,
                         "sample": (f"{steps} full {args.workload} solves (sfac+de1+de2+potl, setup excluded; "
                                    f"run bounded at {REFERENCE_BUDGET_S:.0f} s); {desc}")},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_profile(args):
    """`--profile-solves S`: S plain solves (no CUDA graph, no L2 flush, no
    torch kernels), for profiler captures.  Prints the library's set-up
    launch count and launches per solve, so a capture can skip the set-up and
    the first solve (`-s`) and take exactly one solve (`-c`)."""
    import torch

    from ewaldcorrel_b200 import configs
    from ewaldcorrel_b200.device import SpmeSolver

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    c = load_workload(args.workload)
    stream = torch.cuda.Stream(dev)
    solver = SpmeSolver(c.L, c.K, c.order, c.beta, c.max_m, device=0, stream=stream)
    solver.lib.sfac_set_graphs(solver.handle, 0)
    x = torch.from_numpy(c.x).to(dev)
    q = torch.from_numpy(c.q).to(dev)
    dx = torch.empty((c.n, 3), dtype=torch.float64, device=dev)
    phi = torch.empty(c.n, dtype=torch.float64, device=dev)
    ev = torch.empty(7, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    setup = solver.launches()
    per = []
    for _ in range(args.profile_solves):
        l0 = solver.launches()
        with torch.cuda.stream(stream):
            solver.solve(x, q, dx, phi, ev)
        torch.cuda.synchronize(dev)
        per.append(solver.launches() - l0)
    print(json.dumps({"profile": args.workload, "setup_launches": setup, "launches_per_solve": per,
                      "energy": float(ev[0].item())}), flush=True)


def run_cufft_compare(args):
    """`--cufft-compare`: the solve's own FFT stages (fft_forward = z/y r2c
    passes, fft_inverse = y/z c2r passes, CUDA events per stage, L2 flushed)
    beside cuFFT's full 3-D FP32 r2c and c2r of the same grid (torch.fft, a
    cross-check only: nothing in the library calls cuFFT).  Prints one JSON
    line; the x pass of this library is fused with the convolution, so the
    fair sum is fft_forward + convolution + fft_inverse against
    cuFFT r2c + c2r."""
    import torch

    from ewaldcorrel_b200.device import SpmeSolver

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    c = load_workload(args.workload)
    stream = torch.cuda.Stream(dev)
    solver = SpmeSolver(c.L, c.K, c.order, c.beta, c.max_m, device=0, stream=stream)
    x = torch.from_numpy(c.x).to(dev)
    q = torch.from_numpy(c.q).to(dev)
    dx = torch.empty((c.n, 3), dtype=torch.float64, device=dev)
    phi = torch.empty(c.n, dtype=torch.float64, device=dev)
    ev = torch.empty(7, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    ours = {}
    for i in range(8):
        with torch.cuda.stream(stream):
            flush.zero_()
        st = solver.solve_timed(x, q, dx, phi, ev)
        if i >= 3:
            for k_, v in st.items():
                ours.setdefault(k_, []).append(v)
    ours = {k_: statistics.median(v) for k_, v in ours.items()}
    g = torch.randn(c.K, dtype=torch.float32, device=dev)
    cu = {"r2c": [], "c2r": []}
    for i in range(8):
        flush.zero_()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        F = torch.fft.rfftn(g)
        e1.record()
        torch.fft.irfftn(F, s=c.K)
        e2.record()
        torch.cuda.synchronize(dev)
        if i >= 3:
            cu["r2c"].append(e0.elapsed_time(e1))
            cu["c2r"].append(e1.elapsed_time(e2))
    cu = {k_: statistics.median(v) for k_, v in cu.items()}
    print(json.dumps({"cufft_compare": args.workload, "grid": list(c.K),
                      "ours_ms": {k_: ours[k_] for k_ in ("fft_forward", "convolution", "fft_inverse")},
                      "ours_fft_conv_total_ms": ours["fft_forward"] + ours["convolution"] + ours["fft_inverse"],
                      "cufft_ms": cu, "cufft_total_ms": cu["r2c"] + cu["c2r"],
                      "note": "ours: z/y r2c passes; x pass + Ewald convolution + energy/virial + inverse x pass; "
                              "y/z c2r passes (FP32, deconvolution included). cuFFT: plain 3-D FP32 r2c and c2r"}),
          flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream measurement")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--cufft-compare", action="store_true",
                    help="time the solve's FFT stages beside cuFFT on the same grid and exit (no timing line)")
    ap.add_argument("--profile-solves", type=int, default=0,
                    help="run this many plain solves for a profiler capture and exit (no timing line)")
    args = ap.parse_args(argv)
    if args.profile_solves > 0:
        run_profile(args)
        return
    if args.cufft_compare:
        run_cufft_compare(args)
        return
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_b200(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
