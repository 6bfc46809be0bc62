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
