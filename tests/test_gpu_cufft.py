"""Cross-check of the hand-written forward FFT against cuFFT (through
torch.fft, test-only): S = F(Q) * iB0 iB1 iB2 (sfac.cpp:125-138) from this
library must match cuFFT's FP32 r2c of the same spread grid Q, times the
B-spline moduli, within FP32 round-off.  Also checks the spread grid itself
on grids that take each of the spread's halo paths (z extent a multiple of
the 32-cell bucket or not, several orders) against the FP64 oracle."""
import numpy as np
import pytest

from ewaldcorrel_b200 import configs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _libs(libsfac_path, oracle_built):
    return libsfac_path


def _forward_vs_cufft(c):
    import torch

    from ewaldcorrel_b200 import ewald

    s = ewald.Sfac(np.asarray(c.L, dtype=np.float64), np.array(c.K), c.order)
    s.sfac(c.q, c.x)
    grid = s.debug_spread()
    S = s.get_S()
    F = torch.fft.rfftn(torch.from_numpy(grid).cuda()).cpu().numpy().astype(np.complex128)
    K0, K1, K2 = c.K
    iB = (O.bspline_moduli(K0, c.order)[:, None, None] * O.bspline_moduli(K1, c.order)[None, :, None] *
          O.bspline_moduli(K2, c.order)[None, None, : K2 // 2 + 1])
    ref = F * iB
    return S, ref, iB


@pytest.mark.parametrize("which", ["water", "triclinic"])
def test_forward_fft_matches_cufft(which):
    """Compared before the moduli: F = S / (iB0 iB1 iB2) against cuFFT's F
    (the order-6 moduli reach large values at high frequencies, where they
    would scale up the FP32 round-off of both transforms alike)."""
    c = configs.cfg2_water() if which == "water" else configs.cfg3_triclinic(n=200000, K=128)
    S, ref, iB = _forward_vs_cufft(c)
    ours, theirs = S / iB, ref / iB
    scale = np.abs(theirs).max()
    err = np.abs(ours - theirs).max() / scale
    rms = np.sqrt(np.mean(np.abs(ours - theirs) ** 2) / np.mean(np.abs(theirs) ** 2))
    # FP32 transforms of 2^21 points: each is within ~log2(N) eps of exact
    assert err < 5e-6, f"{which}: max |F - cuFFT| / max |F| = {err:.2e}"
    assert rms < 2e-6, f"{which}: relative RMS {rms:.2e}"


@pytest.mark.parametrize("K,order", [((40, 36, 64), 6), ((24, 24, 48), 8), ((33, 17, 96), 4), ((20, 22, 70), 2)])
def test_spread_grid_bucket_paths(K, order):
    """Grids whose z extent is or is not a multiple of the spread's 32-cell
    buckets: every halo cut (bucket boundary, head/tail counts, key search,
    periodic wrap) against the oracle's spread grid."""
    rng = np.random.default_rng(sum(K) + order)
    L = np.array([3.1, 2.9, 4.4, 0.3, -0.2, 0.4])
    n = 6000
    x = rng.uniform(-1, 5, size=(n, 3))
    q = rng.normal(size=n)
    from ewaldcorrel_b200 import ewald

    s = ewald.Sfac(L, np.array(K), order)
    s.sfac(q, x)
    grid = s.debug_spread()
    o = O.OracleSfac(L, np.array(K), order)
    o.sfac(q, x)
    ref = o.get_spread()
    np.testing.assert_allclose(grid, ref, rtol=0, atol=2e-6 * np.abs(ref).max())
