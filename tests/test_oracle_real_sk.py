"""CPU pins of the oracle's real-space term and radial binning, the checkers
of the device's sfac_real_space and sfac_sk_radial: gradient and virial
against central finite differences, the full Ewald energy of rock salt
against its Madelung constant, and the binning against a direct loop and
against the reference's own plot.py (fixture tests/golden/plot_radial_ref.npz,
made by tests/golden/make_plot_golden.py)."""
import math

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module", autouse=True)
def _built(oracle_built):
    return oracle_built


def _system(seed, n=60):
    rng = np.random.default_rng(seed)
    L = np.array([3.1, 2.9, 3.3, 0.6, -0.4, 0.3])
    x = rng.uniform(0, 1, size=(n, 3)) @ O.LofS(L)
    q = rng.normal(size=n)  # not neutral
    return L, x, q


def test_real_space_gradient_matches_finite_differences():
    L, x, q = _system(3)
    eta, rc = 3.3, 1.4  # erfc(eta rc) ~ 1e-10: nothing jumps at the cutoff
    _, _, _, _, dx = O.real_space(L, x, q, eta, rc)
    h = 1e-6
    rng = np.random.default_rng(4)
    for i in rng.choice(len(q), 6, replace=False):
        for a in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, a] += h
            xm[i, a] -= h
            fd = (O.real_space(L, xp, q, eta, rc)[0] - O.real_space(L, xm, q, eta, rc)[0]) / (2 * h)
            assert abs(fd - dx[i, a]) <= 1e-6 * max(1.0, abs(dx[i, a])), (i, a, fd, dx[i, a])


@pytest.mark.parametrize("ab", [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)])
def test_real_space_virial_matches_strain_derivative(ab):
    """Under the strain r -> (I + e) r (e upper triangular, so the box stays
    lower triangular) dE/de_ab = W_ab, with vir = -W/V in de1's order
    [xx, yy, zz, yx, zx, zy]; E_real + E_net both move."""
    L, x, q = _system(5)
    eta, rc = 3.3, 1.4
    _, _, _, vir, _ = O.real_space(L, x, q, eta, rc)
    V = L[0] * L[1] * L[2]
    a, b = ab
    comp = {(0, 0): 0, (1, 1): 1, (2, 2): 2, (0, 1): 3, (0, 2): 4, (1, 2): 5}[ab]
    h = 1e-6

    def energy(t):
        F = np.eye(3)
        F[a, b] += t
        Lm = O.LofS(L) @ F.T
        r = O.real_space(O.SofL(Lm), x @ F.T, q, eta, rc)
        return r[0] + r[2]

    fd = (energy(h) - energy(-h)) / (2 * h)
    assert abs(fd - (-V * vir[comp])) <= 1e-6 * max(1.0, abs(fd)), (ab, fd, -V * vir[comp])


def test_ewald_energy_of_rock_salt_is_the_madelung_energy():
    """The oracle's reciprocal sum (set_A with ewald_f) plus the real-space
    and self terms is the Coulomb energy of the periodic crystal: for rock
    salt of unit charges and nearest-neighbour distance r0, -M N / (2 r0)
    with M = 1.747564594633 (N ions); independent of eta."""
    a = 1.0
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) * a
    pts, q = [], []
    for i in range(2):
        for j in range(2):
            for k in range(2):
                off = np.array([i, j, k]) * a
                for p in base:
                    pts.append(p + off)
                    q.append(1.0)
                    pts.append(p + off + np.array([0.5, 0, 0]) * a)
                    q.append(-1.0)
    x, q = np.array(pts), np.array(q)
    L = np.array([2 * a, 2 * a, 2 * a, 0, 0, 0])
    want = -1.747564594633 * len(q) / (2 * 0.5 * a)
    for eta in (3.7, 4.2):
        s = O.OracleSfac(L, np.array([48, 48, 48]), 8)
        s.set_ewald(eta, eta * math.sqrt(math.log(1e16)) / math.pi)
        s.sfac(q, x)
        e_rec = s.en()
        e_real, e_self, e_net, _, _ = O.real_space(L, x, q, eta, 0.999 * a)
        assert e_net == 0.0
        tot = e_rec + e_real + e_self
        assert abs(tot - want) <= 2e-6 * abs(want), (eta, tot, want)


def test_sk_radial_matches_direct_loop():
    rng = np.random.default_rng(9)
    L = np.array([4.0, 3.5, 4.4, 0.7, -0.5, 0.9])
    K = (10, 9, 12)
    ldim = K[2] // 2 + 1
    acc = rng.uniform(0, 2, size=(K[0], K[1], ldim))
    nbins, kmax = 17, 30.0
    sums, counts = O.sk_radial(L, K, acc, nbins, kmax)
    iL = np.linalg.inv(O.LofS(L))
    ws, wc = np.zeros(nbins), np.zeros(nbins)
    for i in range(K[0]):
        for j in range(K[1]):
            for k in range(ldim):
                n = np.array([i - K[0] if i > K[0] // 2 else i, j - K[1] if j > K[1] // 2 else j, k], float)
                m = iL @ n  # m . x = n . s for s = inv(box) x
                kk = 2 * math.pi * math.sqrt(m @ m)
                b = int(math.floor(kk / (kmax / nbins)))
                if 0 <= b < nbins:
                    ws[b] += acc[i, j, k]
                    wc[b] += 1
    np.testing.assert_array_equal(counts, wc)
    np.testing.assert_allclose(sums, ws, rtol=1e-13, atol=0)


def test_sk_radial_matches_reference_plot_py():
    """Per-bin sums of the reference's plot.py (plot.py:9-32), run unmodified
    on a seeded |S|^2 array that is zero on the modes where its z fold and
    overflow bin differ from the oracle's binning (fixture and generator in
    tests/golden/)."""
    import os
    import sys

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    try:
        import make_plot_golden as G
    finally:
        sys.path.remove(here)
    z = np.load(os.path.join(here, "plot_radial_ref.npz"))
    K, L, nbins, kmax = tuple(int(k) for k in z["K"]), float(z["L"]), int(z["nbins"]), float(z["kmax"])
    f, kmax_gen = G.seeded_array(K, int(z["seed"]), L)
    assert kmax_gen == kmax
    sums, counts = O.sk_radial(np.array([L, L, L, 0, 0, 0]), K, f, nbins, kmax)
    bins, ref = z["bins"], z["sums"]
    inside = bins < nbins  # plot.py also prints its overflow bin (|k| >= kmax: zero here)
    assert np.all(ref[~inside] == 0.0)
    np.testing.assert_allclose(sums[bins[inside]], ref[inside], rtol=1e-12, atol=0)
    rest = np.ones(nbins, bool)
    rest[bins[inside]] = False
    rest[0] = False  # plot.py does not print bin 0 (the k = 0 mode)
    assert not np.any(sums[rest])
