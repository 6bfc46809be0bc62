"""Regenerates tests/golden/plot_radial_ref.npz: the radial binning of the
reference's own plot.py (plot.py:9-32), run unmodified on a seeded |S|^2
array, as the pin of the oracle's restatement (oracle.oracle.sk_radial).

    python tests/golden/make_plot_golden.py [--reference PATH]
        (default: $EWALDCORREL_REFERENCE, else /root/reference)

plot.py's main() loads the array from a .npy file, bins |k| (cubic box of side
L = 11.680933 * 5, kmax = 0.25 K0 pi / L, 5000 bins) and prints one line
"k mean count" per non-empty bin other than the first and the overflow bin;
each bin's sum is mean * count.  It folds the stored z index as if that axis
had ldim points and clips |k| >= kmax into an extra bin, where the oracle and
the device take the stored z index as it is and drop |k| >= kmax; the seeded
array is therefore zero on every mode where those two choices differ (stored
z index >= ldim // 2, or |k| >= kmax), so the per-bin sums must agree.  The
fixture keeps the seed, the grid and the printed bins with their sums; the
array is regenerated from the seed at test time.
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os
import runpy
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

L_PLOT = 11.680933 * 5  # plot.py's box side
K = (56, 56, 56)  # k / dk = 714.29 |n|: no mode sits exactly on a bin edge (where rounding could
                  # put it on either side), unlike K0 = 64 (625 |n|, integer for integer |n|)
SEED = 21


def seeded_array(K=K, seed=SEED, L=L_PLOT):
    """|S|^2-like positive array over the stored modes (K0, K1, K2 // 2 + 1),
    zero where plot.py's z fold or overflow clip would differ from the
    oracle's binning."""
    K0, K1, K2 = K
    ldim = K2 // 2 + 1
    rng = np.random.default_rng(seed)
    f = rng.uniform(0.5, 2.0, size=(K0, K1, ldim))
    kmax = 0.25 * K0 * np.pi / L
    n0 = np.arange(K0); n0 = np.where(n0 >= K0 // 2, n0 - K0, n0)
    n1 = np.arange(K1); n1 = np.where(n1 >= K1 // 2, n1 - K1, n1)
    n2 = np.arange(ldim)
    k = 2 * np.pi / L * np.sqrt(n0[:, None, None] ** 2 + n1[None, :, None] ** 2 + n2[None, None, :] ** 2)
    f[:, :, ldim // 2:] = 0.0
    f[k >= kmax * (1 - 1e-12)] = 0.0
    return f, kmax


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("EWALDCORREL_REFERENCE", "/root/reference"))
    a = ap.parse_args(argv)
    f, kmax = seeded_array()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "sk.npy")
        np.save(path, f)
        ns = runpy.run_path(os.path.join(a.reference, "plot.py"))  # defines kvec, main (no side effects)
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            ns["main"](["plot.py", path])
    rows = np.array([[float(t) for t in line.split()] for line in buf.getvalue().splitlines() if line.strip()])
    dk = kmax / 5000
    bins = np.rint(rows[:, 0] / dk).astype(np.int64)
    sums = rows[:, 1] * rows[:, 2]
    out = os.path.join(HERE, "plot_radial_ref.npz")
    np.savez(out, K=np.array(K), seed=SEED, L=L_PLOT, kmax=kmax, nbins=5000, bins=bins, sums=sums,
             counts=rows[:, 2])
    print(out, len(bins), "bins")


if __name__ == "__main__":
    sys.exit(main())
