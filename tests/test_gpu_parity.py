"""GPU parity tests: the B200 path (libsfac.so through its C ABI) against the
FP64 oracle and the reference's golden fixtures.  Bit-exact for the integer
cell sort; FP32-path tolerances (energy 1e-6 relative, forces/potentials
1e-5 relative RMS) for the floating-point outputs."""
import json
import os

import numpy as np
import pytest

from ewaldcorrel_b200 import configs
from oracle import oracle as O
from tests.spme_testlib import assert_parity, rel_rms, solve

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TESTPY_L = np.array([9.0, 10.0, 11.0, 2.0, -0.1, 1.0])
TESTPY_CRDS = np.array([[0.1, 0.5, 0.1], [0.9, 0.4, 0.1], [0.1, 0.4, 0.9], [0.9, 0.5, 0.9]])


@pytest.fixture(scope="module", autouse=True)
def _libs(libsfac_path, oracle_built):
    return libsfac_path


def E():
    from ewaldcorrel_b200 import ewald

    return ewald


# ---------------------------------------------------------------- test.py --
def test_testpy_fixture_against_golden():
    """test.py:test()'s fixture through the reference-compatible wrapper,
    against the reference's own outputs (test.log.ref and the compiled
    reference's fixture)."""
    ew = E()
    g = np.load(os.path.join(GOLD, "testpy_ref.npz"))
    log = json.load(open(os.path.join(GOLD, "test_log_ref.json")))
    x = TESTPY_CRDS @ ew.LofS(TESTPY_L)
    q = np.ones(4)
    s = ew.Sfac(TESTPY_L, np.array([12, 13, 14]), 4)
    s.set_A(ew.ewald_f, 1.0)
    s.sfac(q, x)
    M = s.get_S()
    np.testing.assert_allclose(M, g["S"], rtol=0, atol=2e-6 * np.abs(g["S"]).max())
    np.testing.assert_allclose(M[0, 0].real, log["spl_S00"], atol=2e-6)
    en0 = s.en()
    vir = np.zeros(6)
    en1 = s.de1(vir)
    assert en0 == en1  # test.py:100 asserts |en1 - en0| < 1e-14
    assert abs(en0 - log["E"]) <= 1e-6 * log["E"]
    dx = np.zeros((4, 3))
    s.de2(4, q, x, dx)
    assert rel_rms(dx, g["dx"]) < 1e-5
    np.testing.assert_allclose(dx.ravel(), log["spl_dx"], atol=2e-6)
    assert np.abs(vir - g["vir"]).max() <= 1e-5 * np.abs(g["vir"]).max()
    grid = s.get_grid()
    np.testing.assert_allclose(grid, g["grid"], rtol=0, atol=1e-5 * np.abs(g["grid"]).max())


def test_testpy_line_test():
    """test.py:12-37: spline S along each axis against the exact DFT."""
    ew = E()
    x = TESTPY_CRDS @ ew.LofS(TESTPY_L)
    q = np.ones(4)
    s = ew.Sfac(TESTPY_L, np.array([12, 13, 14]), 4)
    s.sfac(q, x)
    M = s.get_S()
    mx = np.arange(12); mx[7:] -= 12
    my = np.arange(13); my[7:] -= 13
    mz = np.arange(8)
    sx = sum(qq * np.exp(-2j * np.pi * c[0] * mx) for qq, c in zip(q, TESTPY_CRDS))
    sy = sum(qq * np.exp(-2j * np.pi * c[1] * my) for qq, c in zip(q, TESTPY_CRDS))
    sz = sum(qq * np.exp(-2j * np.pi * c[2] * mz) for qq, c in zip(q, TESTPY_CRDS))
    assert np.abs(M[:, 0, 0] - sx)[:3].max() < 0.01
    assert np.abs(M[0, :, 0] - sy)[:3].max() < 0.01
    assert np.abs(M[0, 0, :] - sz)[:4].max() < 0.1


def test_testpy_potl_fixture():
    """test.py:test_potl() (test.py:39-62): phi and E = q.phi/2."""
    ew = E()
    g = np.load(os.path.join(GOLD, "testpy_ref.npz"))
    x = TESTPY_CRDS @ ew.LofS(TESTPY_L)
    qp = g["q_potl"]
    s = ew.Sfac(TESTPY_L, np.array([12, 13, 14]), 4)
    s.set_A(ew.ewald_f, 1.0)
    s.sfac(qp, x)
    e0 = s.en()
    vir = np.zeros(6)
    s.de1(vir)
    phi = np.zeros(4)
    s.potl(4, x, phi)
    assert rel_rms(phi, g["phi_potl"]) < 1e-5
    assert abs(0.5 * qp @ phi - e0) <= 2e-6 * abs(e0)


def test_testpy_gradient_and_virial_finite_differences():
    """test.py's FD checks of de2 and of the virial (via set_L, fixed
    fractional coordinates), with a step suited to an FP32 pipeline."""
    ew = E()
    x = TESTPY_CRDS @ ew.LofS(TESTPY_L)
    q = np.ones(4)
    s = ew.Sfac(TESTPY_L, np.array([12, 13, 14]), 4)
    s.set_A(ew.ewald_f, 1.0)
    h = 1e-3

    def Ex(xx):
        s.sfac(q, xx.reshape(4, 3))
        return s.en()

    flat = x.ravel().copy()
    fd = np.zeros(12)
    for i in range(12):
        a = flat.copy(); a[i] += h
        b = flat.copy(); b[i] -= h
        fd[i] = (Ex(a) - Ex(b)) / (2 * h)
    s.sfac(q, x)
    vir = np.zeros(6)
    s.de1(vir)
    dx = np.zeros((4, 3))
    s.de2(4, q, x, dx)
    assert np.abs(dx.ravel() - fd).max() < 2e-3 * np.abs(fd).max()

    def EL(LL):
        s.set_L(LL)  # wrapper re-runs set_A(f, 1.0) (ewald.py:119-122)
        return s.en()

    s.sfac(q, x)
    dEL = np.zeros(6)
    for i in range(6):
        a = TESTPY_L.copy(); a[i] += h
        b = TESTPY_L.copy(); b[i] -= h
        dEL[i] = (EL(a) - EL(b)) / (2 * h)
    V = TESTPY_L[0] * TESTPY_L[1] * TESTPY_L[2]
    Pi = ew.SofL((ew.LofS(dEL).T @ ew.LofS(TESTPY_L)).T) / (-V)
    assert np.abs(vir - Pi).max() < 2e-3 * np.abs(vir).max()


# ---------------------------------------------------------- cell sort --
def _sort_inputs():
    rng = np.random.default_rng(5)
    L = np.array([2.0, 1.9, 2.1, 0.4, -0.2, 0.3])
    out = [("random", L, (12, 13, 14), rng.uniform(-4, 6, size=(3000, 3)))]
    # exact cell boundaries, duplicates and negative zero-ish coordinates
    K = (8, 8, 8)
    Lc = np.array([2.0, 2.0, 2.0, 0.0, 0.0, 0.0])
    grid_pts = np.stack(np.meshgrid(*[np.arange(8) * 0.25] * 3, indexing="ij"), -1).reshape(-1, 3)
    edge = np.concatenate([grid_pts, grid_pts, -1e-17 * np.ones((5, 3)), np.full((4, 3), 2.0 - 1e-16),
                           grid_pts + 2.0, grid_pts - 4.0])
    out.append(("boundaries", Lc, K, edge))
    # heavy clustering: many atoms per cell
    cl = np.repeat(rng.uniform(0, 2, size=(20, 3)), 150, axis=0) + rng.normal(0, 1e-3, size=(3000, 3))
    out.append(("clustered", Lc, (16, 16, 16), cl))
    c1 = configs.cfg1_plain()
    out.append(("plain1000", c1.L, c1.K, c1.x))
    c2 = configs.cfg2_water()
    out.append(("water98304", c2.L, c2.K, c2.x))
    # cells with more atoms than the in-place fix-up takes (two large cells,
    # 2000 and 300 atoms, among scattered ones), and one cell holding every
    # atom at the same point
    big = np.concatenate([rng.uniform(0, 2, size=(700, 3)), 0.51 + rng.uniform(0, 0.1, size=(2000, 3)),
                          rng.uniform(0, 2, size=(300, 3)), 1.26 + rng.uniform(0, 0.1, size=(300, 3))])
    out.append(("large_cells", Lc, K, rng.permutation(big)))
    out.append(("one_cell", Lc, K, np.full((4097, 3), 0.7)))
    # a grid above the single-launch sort's cell limit: the multi-kernel sort
    out.append(("grid168", np.array([6.0, 5.5, 6.2, 0.8, -0.5, 0.4]), (168, 168, 168),
                rng.uniform(-2, 8, size=(20000, 3))))
    return out


@pytest.mark.parametrize("case", range(8))
def test_cell_sort_bit_exact(case):
    name, L, K, x = _sort_inputs()[case]
    ew = E()
    n = len(x)
    s = ew.Sfac(L, np.array(K), 4)
    s.sfac(np.ones(n), x)
    keys, perm = s.debug_sort(n)
    o = O.OracleSfac(L, np.array(K), 4)
    okeys, operm, _ = o.sort(x)
    np.testing.assert_array_equal(keys, okeys, err_msg=name)
    np.testing.assert_array_equal(perm, operm, err_msg=name)


# ------------------------------------------------------------- spread --
@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_spread_grid_matches_oracle(order):
    rng = np.random.default_rng(order)
    L = np.array([2.2, 2.0, 2.4, 0.3, 0.1, -0.2])
    K = (11, 16, 15)
    n = 500
    x = rng.uniform(-1, 3, size=(n, 3))
    q = rng.normal(size=n)
    ew = E()
    s = ew.Sfac(L, np.array(K), order)
    s.sfac(q, x)
    grid = s.debug_spread()
    o = O.OracleSfac(L, np.array(K), order)
    o.sfac(q, x)
    ref = o.get_spread()
    np.testing.assert_allclose(grid, ref, rtol=0, atol=2e-6 * np.abs(ref).max())


# ------------------------------------------------- full-solve parity --
def test_small_reference_fixtures():
    g = np.load(os.path.join(GOLD, "small_ref.npz"))
    names = sorted({k.split("_")[0] for k in g.files})
    for nm in names:
        r = solve("gpu", g[f"{nm}_L"], tuple(g[f"{nm}_K"]), int(g[f"{nm}_order"]), g[f"{nm}_x"],
                  g[f"{nm}_q"], float(g[f"{nm}_beta"]), float(g[f"{nm}_max_m"]))
        ref = {k: g[f"{nm}_{k}"] for k in ("en", "de1", "vir", "dx", "phi")}
        assert_parity(r, ref, nm)
        # S = F(Q) iB0 iB1 iB2: the FP32 error of F(Q) is amplified by the
        # moduli division, strongly at high order near Nyquist.
        K = tuple(g[f"{nm}_K"])
        order = int(g[f"{nm}_order"])
        ib = [O.bspline_moduli(k, order) for k in K]
        amp = np.abs(ib[0][:, None, None] * ib[1][None, :, None] * ib[2][None, None, : K[2] // 2 + 1])
        FQ = g[f"{nm}_S"] / amp
        err = np.abs(r["S"] - g[f"{nm}_S"]) / amp
        assert err.max() <= 3e-6 * np.abs(FQ).max(), (nm, err.max(), np.abs(FQ).max())


def test_plain1000_fixture():
    c = configs.cfg1_plain()
    g = np.load(os.path.join(GOLD, "plain1000_ref.npz"))
    r = solve("gpu", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    assert_parity(r, {k: g[k] for k in ("en", "de1", "vir", "dx", "phi")}, "plain1000")


def test_water_box_against_oracle():
    c = configs.cfg2_water()
    r = solve("gpu", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    o = solve("oracle", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    assert_parity(r, o, c.name)


def test_triclinic_order6_against_oracle():
    c = configs.cfg3_triclinic(n=20000, K=48)
    r = solve("gpu", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    o = solve("oracle", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    assert_parity(r, o, c.name)


def test_triclinic_1m_full_size_against_oracle():
    """The 1,048,576-charge triclinic solve (256^3 grid, order 6, beta 3.5)
    at full size against the FP64 oracle: FP32 in-cell fractions, weights,
    FFT and gather in a 20 nm box, energy within 1e-6 and forces within
    1e-5 relative RMS."""
    c = configs.cfg3_triclinic()
    r = solve("gpu", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    o = solve("oracle", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    assert_parity(r, o, c.name)


def test_device_ewald_matches_host_table():
    """sfac_set_ewald (device FP64 influence function) == set_A(ewald_f)."""
    ew = E()
    c = configs.cfg1_plain()
    a = solve("gpu", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)

    from math import exp, pi

    fac = -((pi / c.beta) ** 2)

    def f(r2, ptr, info):
        if r2 < 1e-10:
            ptr.contents.value = 0.0
            return 0.0
        v = exp(r2 * fac) / (r2 * pi)
        ptr.contents.value = (fac - 1.0 / r2) * v
        return v

    b = solve("gpu", c.L, c.K, c.order, c.x, c.q, callback=f, set_A_max_m=c.max_m)
    assert abs(a["en"] - b["en"]) <= 1e-12 * abs(b["en"])
    np.testing.assert_allclose(a["vir"], b["vir"], rtol=1e-10, atol=1e-16)
    np.testing.assert_allclose(a["dx"], b["dx"], rtol=1e-5, atol=1e-9)


# ------------------------------------------------------- edge cases --
@pytest.mark.parametrize("K,order", [((3, 3, 3), 6), ((1, 1, 1), 4), ((2, 5, 1), 4), ((13, 13, 13), 8),
                                     ((7, 1, 9), 2), ((4, 4, 4), 8)])
def test_tiny_and_odd_grids(K, order):
    rng = np.random.default_rng(sum(K) + order)
    L = np.array([1.3, 1.1, 1.7, 0.2, -0.3, 0.1])
    n = 37
    x = rng.uniform(-2, 3, size=(n, 3))
    q = rng.normal(size=n)  # not neutralised: S(0) stays O(1) on tiny grids
    r = solve("gpu", L, K, order, x, q, 2.5, 6.0)
    o = solve("oracle", L, K, order, x, q, 2.5, 6.0)
    # force scale floor |E| / L: on a 1x1x1 grid the forces vanish exactly,
    # and every atom's whole p^3 stencil folds onto one FP32 point
    assert_parity(r, o, f"K={K} p={order}", energy_rtol=1e-5, force_rrms=3e-5, pot_rrms=3e-5, vir_rtol=3e-5,
                  force_floor=abs(o["en"]) / L[:3].min())


def test_no_atoms_and_one_atom():
    L = np.array([2.0, 2.0, 2.0, 0.0, 0.0, 0.0])
    r = solve("gpu", L, (8, 8, 8), 4, np.zeros((0, 3)), np.zeros(0), 3.0, 6.0)
    assert r["en"] == 0.0 and np.all(r["vir"] == 0.0) and np.all(r["S"] == 0)
    x = np.array([[0.3, 1.1, 1.7]])
    q = np.array([1.0])
    r = solve("gpu", L, (8, 8, 8), 4, x, q, 3.0, 6.0)
    o = solve("oracle", L, (8, 8, 8), 4, x, q, 3.0, 6.0)
    assert_parity(r, o, "one atom")


def test_state_machine_errors(capfd):
    """Wrong-state calls print the reference's messages and return 0 / leave
    outputs untouched (sfac.cpp:310-317,348-355,414-417,502-505)."""
    ew = E()
    L = np.array([2.0, 2.0, 2.0, 0.0, 0.0, 0.0])
    s = ew.Sfac(L, np.array([8, 8, 8]), 4)
    assert s.en() == 0.0
    x = np.array([[0.1, 0.2, 0.3], [1.0, 1.5, 0.2]])
    q = np.array([1.0, -1.0])
    s.sfac(q, x)
    assert s.en() == 0.0  # no kernel set
    out = capfd.readouterr().out
    assert "You must call sfac before this routine" in out
    assert "No convolution kernel has been set" in out
    dx = np.full((2, 3), 7.0)
    s.de2(2, q, x, dx)
    assert np.all(dx == 7.0)
    assert "You must call de1 before this routine" in capfd.readouterr().out
    s.set_ewald(3.0, 6.0)
    vir = np.zeros(6)
    s.de1(vir)
    assert s.en() == 0.0  # state 1
    phi = np.zeros(2)
    s.potl(2, x, phi)
    assert np.any(phi != 0)


def test_gather_accepts_other_point_sets():
    """de2/potl may use points other than those given to sfac
    (sfac.cpp:401-403)."""
    rng = np.random.default_rng(9)
    L = np.array([2.0, 2.2, 2.4, 0.1, 0.2, 0.3])
    x = rng.uniform(0, 2, size=(200, 3))
    q = rng.normal(size=200)
    probes = rng.uniform(-3, 5, size=(333, 3))
    pw = rng.normal(size=333)
    out = []
    for kind in ("gpu", "oracle"):
        if kind == "gpu":
            s = E().Sfac(L, np.array([16, 15, 18]), 6)
        else:
            s = O.OracleSfac(L, np.array([16, 15, 18]), 6)
        s.set_ewald(3.0, 6.0)
        s.sfac(q, x)
        s.de1(np.zeros(6))
        dx = np.zeros((333, 3))
        phi = np.zeros(333)
        s.de2(333, pw, probes, dx)
        s.potl(333, probes, phi)
        out.append((dx, phi))
    assert rel_rms(out[0][0], out[1][0]) < 1e-5
    assert rel_rms(out[0][1], out[1][1]) < 1e-5


def test_pipelined_gather_matches_single_copy():
    """de2/potl with pinned host arrays and enough points split the copies and
    the gather into overlapping chunks; every point must come out exactly as
    in the single-copy path taken for pageable arrays."""
    import torch

    c = configs.cfg2_water()
    n = 400001  # several chunks, the last one short
    rng = np.random.default_rng(11)
    probes = rng.uniform(-1, 11, size=(n, 3))
    pw = rng.normal(size=n)
    s = E().Sfac(c.L, np.array(c.K), c.order)
    s.set_ewald(c.beta, c.max_m)
    s.sfac(c.q, c.x)
    s.de1(np.zeros(6))
    dx_pg, phi_pg = np.zeros((n, 3)), np.zeros(n)
    s.de2(n, pw, probes, dx_pg)
    s.potl(n, probes, phi_pg)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    xp, wp = pin(probes), pin(pw)
    dx_pn, phi_pn = pin(np.zeros((n, 3))), pin(np.zeros(n))
    for _ in range(2):
        dx_pn[:] = 0.0
        phi_pn[:] = 0.0
        s.de2(n, wp, xp, dx_pn)
        s.potl(n, xp, phi_pn)
        np.testing.assert_array_equal(dx_pn, dx_pg)
        np.testing.assert_array_equal(phi_pn, phi_pg)


def test_deterministic_repeat():
    c = configs.cfg1_plain()
    a = solve("gpu", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    b = solve("gpu", c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    assert a["en"] == b["en"]
    np.testing.assert_array_equal(a["S"], b["S"])
    np.testing.assert_array_equal(a["dx"], b["dx"])
    np.testing.assert_array_equal(a["phi"], b["phi"])
