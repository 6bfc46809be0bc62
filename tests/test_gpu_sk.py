"""Structure-factor analysis on the device (sfac_sk_*): the sum of |S|^2 over
frames (run.py:27-47) and its radial binning (plot.py:9-32) against the FP64
oracle."""
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
