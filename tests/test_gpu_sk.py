"""Structure-factor analysis on the device against the FP64 oracle: the sum
of |S|^2 over frames (sfac_sk_*, run.py:27-47), its radial binning
(plot.py:9-32), and the cross-correlations of several densities (sfac_xc_*,
gmx_ewald.py:76-95)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# neutron scattering lengths of run.py:7-11 (H, C, O)
BFAC = np.array([-3.7390, 6.6460, 5.803])


@pytest.fixture(scope="module", autouse=True)
def _libs(libsfac_path, oracle_built):
    return libsfac_path


def E():
    from ewaldcorrel_b200 import ewald

    return ewald


@pytest.mark.parametrize("box", ["cubic", "triclinic"])
def test_sk_accumulate_and_radial_match_oracle(box):
    rng = np.random.default_rng(7 if box == "cubic" else 8)
    if box == "cubic":
        L = np.array([5.84, 5.84, 5.84, 0.0, 0.0, 0.0])
        K = (48, 48, 48)
    else:
        L = np.array([5.0, 4.6, 5.3, 1.1, -0.6, 0.8])
        K = (40, 36, 45)
    n = 1500
    w = BFAC[rng.integers(0, 3, size=n)]
    g = E().Sfac(L, np.array(K), 4)
    o = O.OracleSfac(L, np.array(K), 4)
    g.sk_reset()
    ref = 0.0
    frames = 3
    for _ in range(frames):
        x = rng.uniform(-1, 7, size=(n, 3))
        g.sfac(w, x)
        g.sk_accumulate()
        o.sfac(w, x)
        ref = ref + np.abs(np.array(o.get_S())) ** 2
    acc, nf = g.sk_get()
    assert nf == frames
    assert acc.shape == ref.shape
    assert np.abs(acc - ref).max() <= 2e-5 * np.abs(ref).max()
    kmax, nbins = 37.1234, 1500  # two binning passes of the device kernel
    sums, counts = g.sk_radial(nbins, kmax)
    osums, ocounts = O.sk_radial(L, K, ref, nbins, kmax)
    np.testing.assert_array_equal(counts, ocounts)
    assert np.abs(sums - osums).max() <= 2e-5 * np.abs(osums).max()
    # repeated binning of the same sums gives the same bits
    s2, c2 = g.sk_radial(nbins, kmax)
    np.testing.assert_array_equal(s2, sums)


def test_sk_needs_sfac_first():
    g = E().Sfac(np.array([3.0, 3.0, 3.0, 0, 0, 0]), np.array([16, 16, 16]), 4)
    with pytest.raises(RuntimeError):
        g.sk_accumulate()


def test_cross_correlations_match_oracle():
    """gmx_ewald.py:76-95: per frame, S of each of D densities (own points and
    weights), then C[k] += Q[i] conj(Q[j]) for i <= j."""
    rng = np.random.default_rng(12)
    L = np.array([4.2, 4.0, 4.4, 0.5, -0.3, 0.2])
    K = (32, 30, 36)
    D = 3
    g = E().Sfac(L, np.array(K), 4)
    o = O.OracleSfac(L, np.array(K), 4)
    g.xc_reset(D)
    npair = D * (D + 1) // 2
    ref = np.zeros((npair,) + g.get_S().shape, np.complex128)
    for _ in range(2):
        Q = []
        for i in range(D):
            n = 300 + 100 * i
            x = rng.uniform(-2, 6, size=(n, 3))
            w = rng.normal(size=n)
            g.sfac(w, x)
            g.xc_store(i)
            o.sfac(w, x)
            Q.append(np.array(o.get_S()))
        g.xc_accumulate()
        k = 0
        for i in range(D):
            for j in range(i, D):
                ref[k] += Q[i] * np.conj(Q[j])
                k += 1
    C, nf = g.xc_get()
    assert nf == 2
    assert np.abs(C - ref).max() <= 2e-5 * np.abs(ref).max()
