"""Regenerates the golden fixtures in tests/golden/ (run in a container that
has the reference sources; the fixtures are committed, this script is not
needed at test time).

    make -C oracle all ref
    python tests/golden/make_golden.py [--reference PATH]   (default: $EWALDCORREL_REFERENCE, else /root/reference)

Sources of truth:
  * test_log_ref.json  -- the numbers recorded in the reference's own
    test.log.ref (output of test.py's test(), test.py:64-132), parsed from the
    file as text.
  * *.npz              -- outputs of the reference's own sfac.cpp, compiled
    unmodified against the project FFTW-API shim (oracle/_ref/libsfac_ref.so),
    on seeded inputs.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ewaldcorrel_b200 import configs  # noqa: E402
from oracle.oracle import RefSfac, LofS, ewald_f, ref_available  # noqa: E402


def _floats(text):
    return [float(t) for t in re.findall(r"[-+]?\d+\.\d*(?:e[-+]?\d+)?", text)]


def parse_test_log(path):
    txt = open(path).read()

    def block(start, end=None):
        i = txt.index(start) + len(start)
        j = txt.index(end, i) if end else len(txt)
        return txt[i:j]

    out = {
        "spl_S00": _floats(block("spl S[0,0]:", "ref S[0,0]:")),
        "ref_S00": _floats(block("ref S[0,0]:", "Line errors:")),
        "line_errors": _floats(block("Line errors:", "E:")),
        "E": float(block("E:", "E1:").strip()),
        "E1": float(block("E1:", "spl dx:").strip()),
        "spl_dx": _floats(block("spl dx:", "ref dx:")),
        "ref_dx": _floats(block("ref dx:", "spl vir:")),
        "spl_vir": _floats(block("spl vir:", "ref vir:")),
        "ref_vir": _floats(block("ref vir:")),
    }
    return out


TESTPY_L = np.array([9.0, 10.0, 11.0, 2.0, -0.1, 1.0])
TESTPY_CRDS = np.array([[0.1, 0.5, 0.1], [0.9, 0.4, 0.1], [0.1, 0.4, 0.9], [0.9, 0.5, 0.9]])


def run_ref(L, K, order, x, q, eta, max_m, callback=False):
    s = RefSfac(L, np.array(K), order)
    if callback:
        s.set_A_callback(ewald_f(eta), max_m)
    else:
        s.set_ewald(eta, max_m)
    s.sfac(q, x)
    S = s.get_S()
    e0 = s.en()
    vir = np.zeros(6)
    e1 = s.de1(vir)
    grid = s.get_grid()
    n = len(q)
    dx = np.zeros((n, 3))
    phi = np.zeros(n)
    s.de2(n, q, x, dx)
    s.potl(n, x, phi)
    s.close()
    return dict(S=S, en=e0, de1=e1, vir=vir, grid=grid, dx=dx, phi=phi)


def small_systems():
    """Seeded small systems covering odd/prime/even grids, every order and
    triclinic boxes."""
    rng = np.random.default_rng(2024)
    cases = [
        ((12, 13, 14), 4, [9.0, 10.0, 11.0, 2.0, -0.1, 1.0]),
        ((16, 16, 16), 2, [2.5, 2.5, 2.5, 0.0, 0.0, 0.0]),
        ((15, 9, 20), 6, [3.0, 2.0, 4.0, 0.5, 0.3, -0.4]),
        ((7, 11, 13), 4, [1.7, 2.3, 2.9, -0.3, 0.2, 0.6]),
        ((20, 18, 24), 8, [2.0, 1.8, 2.4, 0.0, 0.0, 0.0]),
        ((10, 10, 9), 6, [2.0, 2.0, 2.0, 1.0, 0.0, 0.0]),
    ]
    out = []
    for i, (K, order, L) in enumerate(cases):
        L = np.array(L)
        n = int(rng.integers(3, 200))
        s = rng.uniform(0.0, 1.0, size=(n, 3))
        x = s @ LofS(L) + rng.integers(-2, 3, size=(n, 3)) @ LofS(L)  # periodic images too
        q = rng.uniform(-1.0, 1.0, size=n)
        q -= q.mean()
        beta = float(rng.uniform(2.0, 4.0))
        max_m = configs.MAX_M_FACTOR * beta
        out.append((f"small{i}", L, K, order, x, q, beta, max_m))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("EWALDCORREL_REFERENCE", "/root/reference"))
    a = ap.parse_args(argv)
    if not ref_available():
        raise SystemExit("oracle/_ref/libsfac_ref.so is not built: make -C oracle ref")

    log = parse_test_log(os.path.join(a.reference, "test.log.ref"))
    with open(os.path.join(HERE, "test_log_ref.json"), "w") as f:
        json.dump(log, f, indent=1)

    # test.py's fixture (test.py:65-85): unit charges, eta = 0.5, max_m = 1.0
    x = TESTPY_CRDS @ LofS(TESTPY_L)
    r = run_ref(TESTPY_L, (12, 13, 14), 4, x, np.ones(4), 0.5, 1.0, callback=True)
    qp = (np.arange(4) % 2) * 0.5 + 0.5  # test_potl's charges (test.py:39-62)
    rp = run_ref(TESTPY_L, (12, 13, 14), 4, x, qp, 0.5, 1.0, callback=True)
    np.savez_compressed(os.path.join(HERE, "testpy_ref.npz"), L=TESTPY_L, x=x, q=np.ones(4),
                        K=np.array([12, 13, 14]), order=4, eta=0.5, max_m=1.0,
                        q_potl=qp, phi_potl=rp["phi"], en_potl=rp["en"], **r)

    # plain 1000-charge system (32^3, order 4, beta 3.47): per-atom outputs
    c1 = configs.cfg1_plain()
    r1 = run_ref(c1.L, c1.K, c1.order, c1.x, c1.q, c1.beta, c1.max_m)
    np.savez_compressed(os.path.join(HERE, "plain1000_ref.npz"), en=r1["en"], de1=r1["de1"],
                        vir=r1["vir"], dx=r1["dx"], phi=r1["phi"],
                        S_abs2_sum=np.sum(np.abs(r1["S"]) ** 2),
                        S_corner=r1["S"][:4, :4, :4])

    # small systems
    rec = {}
    for name, L, K, order, x, q, beta, max_m in small_systems():
        r = run_ref(L, K, order, x, q, beta, max_m)
        for k in ("en", "de1", "vir", "dx", "phi", "S", "grid"):
            rec[f"{name}_{k}"] = r[k]
        rec[f"{name}_x"] = x
        rec[f"{name}_q"] = q
        rec[f"{name}_L"] = L
        rec[f"{name}_K"] = np.array(K)
        rec[f"{name}_order"] = order
        rec[f"{name}_beta"] = beta
        rec[f"{name}_max_m"] = max_m
    np.savez_compressed(os.path.join(HERE, "small_ref.npz"), **rec)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
