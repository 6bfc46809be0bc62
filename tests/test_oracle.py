"""CPU tests of the oracle: it is pinned against the reference's own golden
vectors (test.log.ref, test.cpp's spline values), against the reference's
sfac.cpp compiled unmodified (fixtures in tests/golden/, and live when
oracle/_ref is built), and against numpy's FFT.  No GPU needed."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _built(oracle_built):
    return oracle_built


def test_bspline_known_values():
    # test.cpp prints M_4 at 0.1 steps; the analytic cubic B-spline gives
    # M_4(1) = 1/6, M_4(2) = 2/3, M_4(0.5) = 1/48, M_4(3) = 1/6.
    for x, want in [(0.5, 1 / 48), (1.0, 1 / 6), (2.0, 2 / 3), (3.0, 1 / 6), (1.5, 23 / 48)]:
        j = int(x) if x < 4 else 3
        got = O.bspl_value(4, x - j, j)
        assert abs(got - want) < 1e-15, (x, got, want)


@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_bspline_partition_of_unity_and_symmetry(order):
    for t in np.linspace(0.0, 1.0, 11)[:-1]:
        vals = [O.bspl_value(order, t, j) for j in range(order)]
        assert abs(sum(vals) - 1.0) < 1e-12  # Horner on the reference table: ~1e-14 roundoff
        # M(t + j) = M(order - t - j)
        for j in range(order):
            other = order - t - j
            jj = min(order - 1, int(math.floor(other)))
            assert abs(vals[j] - O.bspl_value(order, other - jj, jj)) < 1e-12


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 8, 12, 13, 14, 30, 97, 128, 210])
def test_fft_shim_matches_numpy(n):
    rng = np.random.default_rng(n)
    z = rng.normal(size=n) + 1j * rng.normal(size=n)
    np.testing.assert_allclose(O.fft1d(z, -1), np.fft.fft(z), rtol=0, atol=1e-12 * n)
    np.testing.assert_allclose(O.fft1d(z, +1), np.fft.ifft(z) * n, rtol=0, atol=1e-12 * n)


def _testpy_system():
    L = np.array([9.0, 10.0, 11.0, 2.0, -0.1, 1.0])
    crds = np.array([[0.1, 0.5, 0.1], [0.9, 0.4, 0.1], [0.1, 0.4, 0.9], [0.9, 0.5, 0.9]])
    return L, crds, crds @ O.LofS(L)


def test_oracle_reproduces_test_log_ref():
    """test.py:test() on the oracle reproduces every number of test.log.ref."""
    log = json.load(open(os.path.join(GOLD, "test_log_ref.json")))
    L, crds, atoms = _testpy_system()
    q = np.ones(4)
    s = O.OracleSfac(L, np.array([12, 13, 14]), 4)
    s.set_A_callback(O.ewald_f(0.5), 1.0)
    s.sfac(q, atoms)
    S = s.get_S()
    np.testing.assert_allclose(S[0, 0].real, log["spl_S00"], atol=1e-8)
    e0 = s.en()
    vir = np.zeros(6)
    e1 = s.de1(vir)
    assert abs(e0 - log["E"]) < 1e-14 and abs(e1 - log["E1"]) < 1e-14
    dx = np.zeros((4, 3))
    s.de2(4, q, atoms, dx)
    np.testing.assert_allclose(dx.ravel(), log["spl_dx"], atol=6e-9)
    np.testing.assert_allclose(vir, log["spl_vir"], rtol=6e-8)


def test_oracle_test_py_checks():
    """The asserts of test.py:test() (test.py:64-132) hold for the oracle."""
    L, crds, atoms = _testpy_system()
    q = np.ones(4)
    K = np.array([12, 13, 14])
    s = O.OracleSfac(L, K, 4)
    f = O.ewald_f(0.5)
    s.set_A_callback(f, 1.0)
    s.sfac(q, atoms)
    M = s.get_S()
    # line test (test.py:12-37)
    mx = np.arange(12); mx[12 // 2 + 1:] -= 12
    my = np.arange(13); my[13 // 2 + 1:] -= 13
    mz = np.arange(8)
    sx = sum(qq * np.exp(-2j * np.pi * c[0] * mx) for qq, c in zip(q, crds))
    sy = sum(qq * np.exp(-2j * np.pi * c[1] * my) for qq, c in zip(q, crds))
    sz = sum(qq * np.exp(-2j * np.pi * c[2] * mz) for qq, c in zip(q, crds))
    assert np.abs(M[:, 0, 0] - sx)[:3].max() < 0.01
    assert np.abs(M[0, :, 0] - sy)[:3].max() < 0.01
    assert np.abs(M[0, 0, :] - sz)[:4].max() < 0.1

    def E(x):
        s.sfac(q, x.reshape(4, 3))
        return s.en()

    h = 1e-7
    dx0 = np.zeros(12)
    flat = atoms.ravel().copy()
    for i in range(12):
        xp = flat.copy(); xp[i] += h
        xm = flat.copy(); xm[i] -= h
        dx0[i] = (E(xp) - E(xm)) / (2 * h)
    s.sfac(q, atoms)
    en0 = s.en()
    vir = np.zeros(6)
    en1 = s.de1(vir)
    assert abs(en1 - en0) < 1e-14
    dx = np.zeros((4, 3))
    s.de2(4, q, atoms, dx)
    assert np.abs(dx.ravel() - dx0).max() < 1e-7

    # virial vs FD of E(L) at fixed fractional coordinates (test.py:107-116)
    def EL(LL):
        s.set_L(LL)
        s.set_A_callback(f, 1.0)
        return s.en()

    s.set_L(L)
    s.set_A_callback(f, 1.0)
    s.sfac(q, atoms)
    dEL = np.zeros(6)
    for i in range(6):
        Lp = L.copy(); Lp[i] += h
        Lm = L.copy(); Lm[i] -= h
        dEL[i] = (EL(Lp) - EL(Lm)) / (2 * h)
    V = L[0] * L[1] * L[2]
    Pi = O.LofS(dEL).T
    Pi = O.SofL((Pi @ O.LofS(L)).T) / (-V)
    assert np.abs(vir - Pi).max() < 1e-8


def test_oracle_potl_fixture():
    """test.py:test_potl(): potentials and 0.5 q.phi = E (test.py:39-62)."""
    g = np.load(os.path.join(GOLD, "testpy_ref.npz"))
    L, crds, atoms = _testpy_system()
    qp = g["q_potl"]
    s = O.OracleSfac(L, np.array([12, 13, 14]), 4)
    s.set_A_callback(O.ewald_f(0.5), 1.0)
    s.sfac(qp, atoms)
    e0 = s.en()
    vir = np.zeros(6)
    s.de1(vir)
    phi = np.zeros(4)
    s.potl(4, atoms, phi)
    np.testing.assert_allclose(phi, [0.42564717, 0.527872, 0.45544654, 0.54449008], atol=5e-9)
    np.testing.assert_allclose(phi, g["phi_potl"], rtol=1e-13)
    assert abs(0.5 * qp @ phi - e0) < 1e-13


def _run(cls, L, K, order, x, q, beta, max_m):
    s = cls(L, np.array(K), order)
    s.set_ewald(beta, max_m)
    s.sfac(q, x)
    S = s.get_S()
    e0 = s.en()
    vir = np.zeros(6)
    e1 = s.de1(vir)
    n = len(q)
    dx = np.zeros((n, 3))
    phi = np.zeros(n)
    s.de2(n, q, x, dx)
    s.potl(n, x, phi)
    return dict(S=S, en=e0, de1=e1, vir=vir, dx=dx, phi=phi, grid=s.get_grid())


def _small_cases():
    g = np.load(os.path.join(GOLD, "small_ref.npz"))
    names = sorted({k.split("_")[0] for k in g.files})
    return g, names


def test_oracle_matches_reference_fixtures_small():
    g, names = _small_cases()
    for nm in names:
        r = _run(O.OracleSfac, g[f"{nm}_L"], tuple(g[f"{nm}_K"]), int(g[f"{nm}_order"]), g[f"{nm}_x"],
                 g[f"{nm}_q"], float(g[f"{nm}_beta"]), float(g[f"{nm}_max_m"]))
        scale = np.abs(g[f"{nm}_S"]).max()
        np.testing.assert_allclose(r["S"], g[f"{nm}_S"], rtol=0, atol=1e-12 * scale, err_msg=nm)
        assert abs(r["en"] - g[f"{nm}_en"]) <= 1e-12 * abs(g[f"{nm}_en"]), nm
        np.testing.assert_allclose(r["vir"], g[f"{nm}_vir"], rtol=1e-10, atol=1e-14, err_msg=nm)
        np.testing.assert_allclose(r["dx"], g[f"{nm}_dx"], rtol=1e-10, atol=1e-12, err_msg=nm)
        np.testing.assert_allclose(r["phi"], g[f"{nm}_phi"], rtol=1e-10, atol=1e-12, err_msg=nm)


def test_oracle_matches_reference_fixture_plain1000():
    from ewaldcorrel_b200 import configs

    c = configs.cfg1_plain()
    g = np.load(os.path.join(GOLD, "plain1000_ref.npz"))
    r = _run(O.OracleSfac, c.L, c.K, c.order, c.x, c.q, c.beta, c.max_m)
    assert abs(r["en"] - g["en"]) <= 1e-12 * abs(g["en"])
    np.testing.assert_allclose(r["vir"], g["vir"], rtol=1e-10)
    np.testing.assert_allclose(r["dx"], g["dx"], rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(r["phi"], g["phi"], rtol=1e-9, atol=1e-11)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_oracle_matches_live_reference_random():
    rng = np.random.default_rng(7)
    for K, order, L in [((9, 10, 11), 4, [2.0, 2.1, 2.2, 0.3, -0.2, 0.1]), ((16, 12, 10), 6, [3, 2, 2, 0, 0, 0])]:
        L = np.array(L, dtype=float)
        n = 50
        x = rng.uniform(-3, 6, size=(n, 3))
        q = rng.normal(size=n)
        a = _run(O.OracleSfac, L, K, order, x, q, 3.0, 6.0)
        b = _run(O.RefSfac, L, K, order, x, q, 3.0, 6.0)
        assert abs(a["en"] - b["en"]) <= 1e-12 * abs(b["en"])
        np.testing.assert_allclose(a["dx"], b["dx"], rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(a["phi"], b["phi"], rtol=1e-10, atol=1e-12)


def test_oracle_forward_path_matches_numpy_rfftn():
    """Spread grid -> numpy rfftn -> moduli division equals the oracle's S."""
    rng = np.random.default_rng(3)
    L = np.array([2.0, 2.5, 3.0, 0.2, 0.1, -0.3])
    K = (10, 12, 15)
    x = rng.uniform(0, 3, size=(40, 3))
    q = rng.normal(size=40)
    s = O.OracleSfac(L, np.array(K), 6)
    s.sfac(q, x)
    Q = s.get_spread()
    iB = [O.bspline_moduli(k, 6) for k in K]
    ref = np.fft.rfftn(Q) * iB[0][:, None, None] * iB[1][None, :, None] * iB[2][None, None, : K[2] // 2 + 1]
    np.testing.assert_allclose(s.get_S(), ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_oracle_sort_is_stable_cell_order():
    rng = np.random.default_rng(11)
    L = np.array([2.0, 2.0, 2.0, 0.5, 0.0, 0.3])
    K = (5, 6, 7)
    s = O.OracleSfac(L, np.array(K), 4)
    # many atoms per cell, exact duplicates and periodic images
    base = rng.uniform(0, 2, size=(30, 3))
    x = np.concatenate([base, base, base + 2.0 * np.array([1, 0, 0]) @ O.LofS(L) / 2.0, base[:5]])
    keys, perm, frac = s.sort(x)
    assert np.all(np.diff(keys) >= 0)
    same = np.diff(keys) == 0
    assert np.all(np.diff(perm)[same] > 0)  # ties keep input order
    assert sorted(perm.tolist()) == list(range(len(x)))
    assert np.all((frac >= 0) & (frac < 1))


def _ewald_tables_per_mode(L, K, beta, max_m):
    """Independent numpy evaluation of set_A's folded sums, per stored mode:
    A = w * sum_{m = n mod K} f, dA = 2 w sum f' m m, w = 1/2 on the kz = 0
    and even-K2 Nyquist planes, 1 elsewhere.  This is the formula the device
    Ewald path evaluates.  m = iL n with iL the inverse of the lower-triangular
    box (Cell, sfac.hpp:37-52)."""
    iL = np.linalg.inv(O.LofS(L))
    K0, K1, K2 = K
    ldim = K2 // 2 + 1
    fac = -((np.pi / beta) ** 2)
    r = 40
    g = np.arange(-r, r + 1)
    n = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    m = n @ iL.T
    m2 = (m * m).sum(1)
    keep = (m2 < max_m ** 2) & (m2 >= 1e-10) & (n[:, 2] % K2 < ldim)
    n, m, m2 = n[keep], m[keep], m2[keep]
    f = np.exp(m2 * fac) / (m2 * np.pi)
    fp = (fac - 1 / m2) * f
    idx = ((n[:, 0] % K0) * K1 + n[:, 1] % K1) * ldim + n[:, 2] % K2
    A = np.bincount(idx, weights=f, minlength=K0 * K1 * ldim)
    prods = np.stack([m[:, 0] ** 2, m[:, 1] ** 2, m[:, 2] ** 2, m[:, 1] * m[:, 0], m[:, 2] * m[:, 0],
                      m[:, 2] * m[:, 1]], 1)
    dA = np.stack([np.bincount(idx, weights=fp * prods[:, c], minlength=K0 * K1 * ldim) for c in range(6)], 1)
    A = A.reshape(K0, K1, ldim)
    dA = dA.reshape(K0, K1, ldim, 6)
    w = np.ones(ldim)
    w[0] = 0.5
    if K2 % 2 == 0:
        w[-1] = 0.5
    return A * w[None, None, :], dA * (2 * w)[None, None, :, None]


def test_per_mode_ewald_formula_matches_set_A_fold():
    """The per-mode image sum used by the device Ewald path equals the
    oracle's set_A fold (sfac.cpp:240-289), including aliases."""
    L = np.array([1.1, 1.0, 1.2, 0.3, -0.1, 0.2])
    K = (6, 5, 8)
    beta, max_m = 2.0, 5.5  # max_m beyond Nyquist: aliases are folded
    s = O.OracleSfac(L, np.array(K), 4)
    s.set_ewald(beta, max_m)
    A, dA = s.get_A()
    A2, dA2 = _ewald_tables_per_mode(L, K, beta, max_m)
    np.testing.assert_allclose(A, A2, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(dA, dA2, rtol=1e-12, atol=1e-15)
