"""Allocation-failure paths, driven on the host by the library's test hook
(sfac_debug_fail_alloc: the n-th device allocation from now on fails once)
instead of exhausting a GPU: the constructor returns NULL (the wrapper
raises, as the reference's ewald.py:80-81 does), set_A returns 2
(sfac.cpp:223), and a serving request whose slot cannot be allocated is
refused with 2 while the server stays usable."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture()
def lib(libsfac_path):
    from ewaldcorrel_b200 import ewald

    _, _, lib = ewald.describe_sfac()
    lib.sfac_debug_fail_alloc.argtypes = [ctypes.c_int]
    lib.sfac_debug_fail_alloc.restype = ctypes.c_int
    yield lib
    lib.sfac_debug_fail_alloc(0)


L = np.array([2.0, 2.1, 1.9, 0.1, 0.0, -0.2])


@pytest.mark.parametrize("nth", [1, 2, 5])
def test_ctor_returns_null_when_an_allocation_fails(lib, nth):
    from ewaldcorrel_b200 import ewald

    lib.sfac_debug_fail_alloc(nth)
    with pytest.raises(RuntimeError, match="intializing"):
        ewald.Sfac(L.copy(), np.array([16, 16, 16]), 4)
    s = ewald.Sfac(L.copy(), np.array([16, 16, 16]), 4)  # the hook fired once: the next one works
    s.set_ewald(3.0, 6.0)
    rng = np.random.default_rng(1)
    x = rng.uniform(0, 2, size=(50, 3))
    q = rng.normal(size=50)
    s.sfac(q, x)
    assert np.isfinite(s.en())


def test_set_A_returns_2_when_its_table_cannot_be_allocated(lib):
    from ewaldcorrel_b200 import ewald

    s = ewald.Sfac(L.copy(), np.array([12, 13, 14]), 4)
    lib.sfac_debug_fail_alloc(1)  # set_A's first allocation: the A/dA tables
    with pytest.raises(RuntimeError, match=r"Error \(2\) setting A-array"):
        s.set_A(ewald.ewald_f, 1.0)
    s.set_A(ewald.ewald_f, 1.0)  # and works once memory is there
    rng = np.random.default_rng(2)
    x = rng.uniform(0, 2, size=(20, 3))
    s.sfac(np.ones(20), x)
    assert s.en() > 0


def test_server_refuses_a_request_whose_slot_cannot_be_allocated(lib):
    from ewaldcorrel_b200 import configs
    from ewaldcorrel_b200.serve import Request, SpmeServer, _pinned

    pool = configs.cfg5_pool()
    spec = [s for s in configs.cfg5_specs(200) if s["n"] < 4000][0]
    sysm = configs.cfg5_request(spec, pool)
    req = Request(spec["id"], sysm.x, sysm.q, sysm.L, sysm.K, sysm.order, sysm.beta, sysm.max_m)
    xb = _pinned((req.n, 3))
    xb[:] = req.x
    out = _pinned(7 + 4 * req.n)
    srv = SpmeServer(max_inflight=4)
    lib.sfac_debug_fail_alloc(3)
    assert srv.submit(req, xb, out) == 2
    st = srv.stats()
    assert st["errors"] == 1 and st["inflight"] == 0 and st["slots"] == 0 and st["bytes"] == 0
    assert srv.submit(req, xb, out) == 0  # the server is still usable
    done = []
    while not done:
        done = srv.poll()
    assert done == [(req.id, 0)]
    st = srv.stats()
    srv.close()
    assert st["solves"] == 1 and st["errors"] == 1
    assert np.isfinite(out[0]) and out[0] != 0.0
