"""Helpers shared by the GPU parity tests: run one full solve through the
B200 library's C ABI (via the ewald.py-compatible wrapper) and through the
FP64 CPU oracle, and compare by relative RMS force error and relative energy error."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

# Accuracy bar of the FP32 B200 path against the FP64 oracle.
ENERGY_RTOL = 1e-6  # relative energy error
FORCE_RRMS = 1e-5  # relative RMS force (dE/dx) error
POT_RRMS = 1e-5  # relative RMS potential error
VIRIAL_RTOL = 1e-5  # |dvir| / max|vir|


def rel_rms(a, b, floor=0.0):
    """RMS(a - b) / max(RMS(b), floor)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(float(np.sqrt(np.mean(b * b))), floor)
    return float(np.sqrt(np.mean((a - b) ** 2)) / den) if den > 0 else float(np.abs(a - b).max())


def solve(cls, L, K, order, x, q, beta=None, max_m=None, callback=None, set_A_max_m=None):
    """Full reciprocal solve: sfac -> en -> de1 -> de2 -> potl -> grid."""
    from ewaldcorrel_b200 import ewald as E

    L = np.ascontiguousarray(L, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    if cls == "gpu":
        s = E.Sfac(L, np.asarray(K), order)
        if callback is not None:
            s.set_A(callback, set_A_max_m)
        else:
            s.set_ewald(beta, max_m)
    else:
        s = O.OracleSfac(L, np.asarray(K), order)
        if callback is not None:
            s.set_A_callback(callback, set_A_max_m)
        else:
            s.set_ewald(beta, max_m)
    n = len(q)
    s.sfac(q, x)
    S = np.array(s.get_S())
    e0 = s.en()
    vir = np.zeros(6)
    e1 = s.de1(vir)
    grid = s.get_grid()
    dx = np.zeros((n, 3))
    phi = np.zeros(n)
    if n:
        s.de2(n, q, x, dx)
        s.potl(n, x, phi)
    return dict(S=S, en=e0, de1=e1, vir=vir, grid=grid, dx=dx, phi=phi, handle=s)


def assert_parity(g, o, name="", energy_rtol=ENERGY_RTOL, force_rrms=FORCE_RRMS, pot_rrms=POT_RRMS,
                  vir_rtol=VIRIAL_RTOL, force_floor=0.0):
    """force_floor: lower bound of the force scale, for systems whose forces
    vanish by symmetry (e.g. a 1x1x1 grid), where a relative error of
    round-off is meaningless."""
    e_err = abs(g["en"] - o["en"]) / max(abs(o["en"]), 1e-300)
    assert e_err <= energy_rtol, f"{name}: energy rel err {e_err:.3e} (gpu {g['en']!r} oracle {o['en']!r})"
    assert g["en"] == g["de1"], f"{name}: en() and de1() energies differ"
    if np.any(o["dx"]):
        f_err = rel_rms(g["dx"], o["dx"], force_floor)
        assert f_err <= force_rrms, f"{name}: force rel-RMS err {f_err:.3e}"
    if np.any(o["phi"]):
        p_err = rel_rms(g["phi"], o["phi"])
        assert p_err <= pot_rrms, f"{name}: potential rel-RMS err {p_err:.3e}"
    vmax = np.abs(o["vir"]).max()
    if vmax > 0:
        v_err = np.abs(g["vir"] - o["vir"]).max() / vmax
        assert v_err <= vir_rtol, f"{name}: virial err {v_err:.3e}"
