"""GPU tests of the serving runtime (continuous batching): every request's
result is the same served alone and served in a mix of concurrent requests
of other shapes (within the FP32-path tolerance), matches the FP64 oracle,
and survives admission under a small memory budget (slot eviction)."""
import numpy as np
import pytest

from ewaldcorrel_b200 import configs
from tests.spme_testlib import rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _libs(libsfac_path, oracle_built):
    return libsfac_path


def _requests(count=40, nmax=30000):
    from ewaldcorrel_b200.serve import Request

    pool = configs.cfg5_pool()
    specs = [s for s in configs.cfg5_specs(600) if s["n"] <= nmax][:count]
    reqs = []
    for s in specs:
        sysm = configs.cfg5_request(s, pool)
        reqs.append(Request(s["id"], sysm.x, sysm.q, sysm.L, sysm.K, sysm.order, sysm.beta, sysm.max_m))
    return reqs


def _compare(a, b, name):
    ea, va, dxa, pa = a
    eb, vb, dxb, pb = b
    assert abs(ea - eb) <= 1e-6 * abs(eb), (name, ea, eb)
    assert rel_rms(dxa, dxb) <= 1e-5, name
    assert rel_rms(pa, pb) <= 1e-5, name
    assert np.abs(va - vb).max() <= 1e-5 * np.abs(vb).max(), name


def test_each_result_same_alone_and_in_mix():
    from ewaldcorrel_b200.serve import SpmeServer, run_stream

    reqs = _requests()
    ids = {r.id for r in reqs}
    alone = SpmeServer(max_inflight=1)
    _, _, out_alone = run_stream(alone, reqs, keep=ids, max_inflight=1)
    alone.close()
    mix = SpmeServer(max_inflight=16)
    rng = np.random.default_rng(1)
    arrivals = np.cumsum(rng.exponential(20e-6, size=len(reqs)))  # faster than service: overlap
    lat, _, out_mix = run_stream(mix, reqs, arrivals=arrivals, keep=ids, max_inflight=16)
    st = mix.stats()
    mix.close()
    assert st["errors"] == 0 and st["solves"] == len(reqs)
    for r in reqs:
        _compare(out_mix[r.id], out_alone[r.id], f"request {r.id}")
    assert np.all(lat > 0)


def test_served_results_match_oracle():
    from ewaldcorrel_b200.serve import SpmeServer, run_stream
    from oracle.oracle import OracleSfac

    reqs = [r for r in _requests(count=40, nmax=6000)][:4]
    srv = SpmeServer(max_inflight=8)
    _, _, out = run_stream(srv, reqs, keep={r.id for r in reqs}, max_inflight=8)
    srv.close()
    for r in reqs:
        o = OracleSfac(r.L, r.K, r.order)
        o.set_ewald(r.beta, r.max_m)
        o.sfac(r.q, r.x)
        vir = np.zeros(6)
        e = o.de1(vir)
        dx = np.zeros((r.n, 3))
        phi = np.zeros(r.n)
        o.de2(r.n, r.q, r.x, dx)
        o.potl(r.n, r.x, phi)
        _compare(out[r.id], (e, vir, dx, phi), f"request {r.id} vs oracle")


def test_small_budget_evicts_and_stays_correct():
    from ewaldcorrel_b200.serve import SpmeServer, run_stream

    reqs = _requests(count=24, nmax=20000)
    ids = {r.id for r in reqs}
    big = SpmeServer(max_inflight=4)
    _, _, ref = run_stream(big, reqs, keep=ids, max_inflight=4)
    big.close()
    # room for about two slots of the largest shape: forces evictions
    from ewaldcorrel_b200.serve import _lib

    lib = _lib()
    biggest = max(int(lib.sfac_footprint_bytes(np.asarray(r.K, np.int32), 2 * r.n)) + 64 * r.n for r in reqs)
    budget = 2 * biggest + (4 << 20)
    small = SpmeServer(budget_bytes=budget, max_inflight=4)
    _, _, out = run_stream(small, reqs, keep=ids, max_inflight=4)
    st = small.stats()
    small.close()
    assert st["evicted"] > 0 and st["bytes"] <= budget and st["errors"] == 0
    for r in reqs:
        _compare(out[r.id], ref[r.id], f"request {r.id}")


def test_packed_submit_matches_oracle():
    """spme_server_submit_packed (one packed block [box, n, f | x | q]) gives
    the oracle's results, on slots whose box changes on the device between
    requests of the same shape, with Cartesian and with fractional (f = 1)
    positions."""
    import ctypes

    from ewaldcorrel_b200.serve import SpmeServer, _lib, _pinned
    from oracle.oracle import OracleSfac

    lib = _lib()
    lib.spme_server_submit_packed.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                              ctypes.c_void_p]
    lib.spme_server_submit_packed.restype = ctypes.c_int
    rng = np.random.default_rng(3)
    srv = SpmeServer(max_inflight=4)
    K = np.array([32, 32, 32], np.int32)
    cases = []
    for i, side in enumerate((3.0, 3.3, 2.8)):  # same shape, new box each time
        n = 1200
        frac = i == 2  # the last one sends fractional coordinates (flag word 7)
        s = rng.uniform(0, 1, size=(n, 3))
        x = s * side
        q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
        blk = _pinned(16 + 4 * n)
        blk[:] = 0.0
        blk[0:3] = side
        blk[6] = n
        blk[7] = 1.0 if frac else 0.0
        blk[16:16 + 3 * n] = (s if frac else x).ravel()
        blk[16 + 3 * n:] = q
        out = _pinned(7 + 4 * n)
        rc = lib.spme_server_submit_packed(srv.h, i, n, K.ctypes.data, 4, 3.12, 6.0, blk.ctypes.data, out.ctypes.data)
        assert rc == 0
        done = []
        while not done:
            done = srv.poll()
        assert done == [(i, 0)]
        cases.append((side, x, q, out.copy()))
    srv.close()
    for side, x, q, out in cases:
        n = len(q)
        o = OracleSfac(np.array([side, side, side, 0, 0, 0]), K, 4)
        o.set_ewald(3.12, 6.0)
        o.sfac(q, x)
        vir = np.zeros(6)
        e = o.de1(vir)
        dx = np.zeros((n, 3))
        phi = np.zeros(n)
        o.de2(n, q, x, dx)
        o.potl(n, x, phi)
        _compare((out[0], out[1:7], out[7:7 + 3 * n].reshape(n, 3), out[7 + 3 * n:]), (e, vir, dx, phi),
                 f"box {side}")


def test_native_stream_runner():
    """spme_server_run_stream serves a stream (all at once, then with timed
    arrivals) with no errors and a latency for every request."""
    from ewaldcorrel_b200.serve import SpmeServer

    specs = [s for s in configs.cfg5_specs(400) if s["n"] <= 40000][:60]
    pool = configs.cfg5_pool()
    qpool = configs.cfg5_charges(configs.CFG5_POOL_ATOMS)
    srv = SpmeServer(max_inflight=16)
    lat, wall = srv.run_stream_native(specs, None, pool, qpool)
    assert wall > 0 and np.all(lat > 0)
    arrivals = np.cumsum(np.full(len(specs), 100e-6))
    lat, wall = srv.run_stream_native(specs, arrivals, pool, qpool)
    st = srv.stats()
    srv.close()
    assert np.all(lat > 0) and wall >= arrivals[-1]
    assert st["errors"] == 0 and st["solves"] == 2 * len(specs)
