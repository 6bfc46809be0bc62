"""Solves through the index-checking library (libsfac_check.so, loaded because
EWALDCORREL_LIBSFAC names it) on shapes that take every kernel path, and
prints one JSON line: whether the build checks, its self-test, and per case
the first failed index check (module 0 = none) with the parity errors
against the FP64 oracle.  Run as a child process by tests/test_gpu_check.py,
so that the checking library never shares a process with the product one.
"""
from __future__ import annotations

import ctypes
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from ewaldcorrel_b200 import ewald as E  # noqa: E402
from tests import spme_testlib as T  # noqa: E402

TRI = np.array([2.0, 2.1, 1.9, 0.1, 0.0, -0.2])

# (name, L6, K, order, atoms, clustered): grids below one brick, grids whose
# z length is not a multiple of 32, every order, the split-brick spread
# (small grids) and the one-warp-per-brick spread (192^3), and a clustered
# box whose buckets exceed the fix-up's in-place limit (merge-sorted).
CASES = [
    ("tri_12x13x14_p4", TRI, (12, 13, 14), 4, 600, False),
    ("tri_5x6x7_p4", TRI, (5, 6, 7), 4, 200, False),
    ("tri_40x36x64_p6", TRI * 2, (40, 36, 64), 6, 4000, False),
    ("tri_24x24x48_p8", TRI, (24, 24, 48), 8, 3000, False),
    ("tri_33x17x96_p4", TRI * 3, (33, 17, 96), 4, 5000, False),
    ("tri_20x22x70_p2", TRI, (20, 22, 70), 2, 2000, False),
    ("cubic_96_p4", np.array([9.6, 9.6, 9.6, 0, 0, 0]), (96, 96, 96), 4, 30000, False),
    ("cubic_192_p6", np.array([19.2, 19.2, 19.2, 0, 0, 0]), (192, 192, 192), 6, 120000, False),
    ("clustered_16_p4", np.array([3.0, 3.0, 3.0, 0, 0, 0]), (16, 16, 16), 4, 3000, True),
]


def _system(L, n, clustered, seed):
    rng = np.random.default_rng(seed)
    Lm = np.array([[L[0], 0, 0], [L[3], L[1], 0], [L[4], L[5], L[2]]])
    s = rng.uniform(0, 1, size=(n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    if clustered:
        s = 0.3 + 0.02 * s  # every atom within about one cell
        q = np.ones(n)  # like charges: no FP32 cancellation on the few grid points they reach
    x = s @ Lm
    return x, q


def main():
    _, _, lib = E.describe_sfac()
    lib.sfac_check_enabled.restype = ctypes.c_int
    lib.sfac_check_selftest.restype = ctypes.c_int
    lib.sfac_check_take.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)]
    lib.sfac_check_take.restype = ctypes.c_int

    def take():
        w = ctypes.c_ulonglong(0)
        m = lib.sfac_check_take(ctypes.byref(w))
        return m, hex(w.value)

    out = {"library": os.environ.get("EWALDCORREL_LIBSFAC", ""), "enabled": lib.sfac_check_enabled(),
           "selftest": lib.sfac_check_selftest(), "start": take(), "cases": []}
    beta = 3.0
    for i, (name, L, K, order, n, clustered) in enumerate(CASES):
        x, q = _system(L, n, clustered, 100 + i)
        max_m = 1.93205 * beta
        g = T.solve("gpu", L, K, order, x, q, beta=beta, max_m=max_m)
        m, w = take()
        o = T.solve("oracle", L, K, order, x, q, beta=beta, max_m=max_m)
        out["cases"].append({
            "case": name, "module": m, "word": w,
            "energy_rel": abs(g["en"] - o["en"]) / abs(o["en"]),
            "force_rrms": T.rel_rms(g["dx"], o["dx"]),
            "pot_rrms": T.rel_rms(g["phi"], o["phi"]),
        })
        g["handle"].__del__()

    # the graph-replayed device solve (the bench's path) and the serving runtime
    import torch

    from ewaldcorrel_b200.device import SpmeSolver
    from ewaldcorrel_b200.serve import Request, SpmeServer, _pinned

    L = np.array([9.6, 9.6, 9.6, 0, 0, 0])
    x, q = _system(L, 30000, False, 7)
    sv = SpmeSolver(L, (96, 96, 96), 4, beta, 6.0)
    xd = torch.tensor(x, device=sv.device)
    qd = torch.tensor(q, device=sv.device)
    dx = torch.empty_like(xd)
    phi = torch.empty_like(qd)
    for _ in range(3):
        ev = sv.solve(xd, qd, dx, phi)
    torch.cuda.synchronize()
    m, w = take()
    o = T.solve("oracle", L, (96, 96, 96), 4, x, q, beta=beta, max_m=6.0)
    out["cases"].append({"case": "device_solve_96_p4", "module": m, "word": w,
                         "energy_rel": abs(float(ev[0]) - o["en"]) / abs(o["en"]),
                         "force_rrms": T.rel_rms(dx.cpu().numpy(), o["dx"]),
                         "pot_rrms": T.rel_rms(phi.cpu().numpy(), o["phi"])})

    srv = SpmeServer(max_inflight=4)
    errs = []
    for rid, (n, k, order, side) in enumerate([(900, 24, 4, 2.1), (5000, 40, 6, 3.7), (1700, 30, 4, 2.6)]):
        xs, qs = _system(np.array([side, side, side, 0, 0, 0]), n, False, 40 + rid)
        req = Request(rid, xs, qs, np.array([side, side, side, 0, 0, 0]), np.array([k, k, k]), order, beta, 6.0)
        xb = _pinned((n, 3))
        xb[:] = xs
        res = _pinned(7 + 4 * n)
        assert srv.submit(req, xb, res) == 0
        done = []
        while not done:
            done = srv.poll()
        o = T.solve("oracle", req.L, req.K, order, xs, qs, beta=beta, max_m=6.0)
        errs.append(abs(res[0] - o["en"]) / abs(o["en"]))
    srv.close()
    m, w = take()
    out["cases"].append({"case": "serving_3_requests", "module": m, "word": w, "energy_rel": max(errs),
                         "force_rrms": 0.0, "pot_rrms": 0.0})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
