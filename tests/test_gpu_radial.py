"""A radial influence function evaluated on the device (sfac_set_radial)
against the reference's mechanism for the same function: set_A with a host
callback (sfac.cpp:213-292, ewald.py:111-117), on the GPU and in the FP64
oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.spme_testlib import assert_parity, rel_rms

pytestmark = pytest.mark.gpu

A_SCR, KAPPA2 = 0.05, 0.7  # f(z) = exp(-a z) / (z + kappa^2): screened, finite at m = 0


def f_np(z):
    return np.exp(-A_SCR * z) / (z + KAPPA2)


def df_np(z):
    return -A_SCR * f_np(z) - f_np(z) / (z + KAPPA2)


def f_cb(r2, ptr, info):
    f = float(np.exp(-A_SCR * r2) / (r2 + KAPPA2))
    ptr.contents.value = -A_SCR * f - f / (r2 + KAPPA2)
    return f


@pytest.fixture(scope="module", autouse=True)
def _libs(libsfac_path, oracle_built):
    return libsfac_path


def _run(s, q, x):
    n = len(q)
    s.sfac(q, x)
    e0 = s.en()
    vir = np.zeros(6)
    e1 = s.de1(vir)
    dx = np.zeros((n, 3))
    phi = np.zeros(n)
    s.de2(n, q, x, dx)
    s.potl(n, x, phi)
    return dict(en=e0, de1=e1, vir=vir, dx=dx, phi=phi)


def test_device_radial_matches_host_callback():
    from ewaldcorrel_b200 import ewald as E

    rng = np.random.default_rng(31)
    L = np.array([3.1, 2.9, 3.3, 0.4, -0.5, 0.3])
    K = (24, 20, 27)
    n = 400
    x = rng.uniform(0, 3, size=(n, 3))
    q = rng.normal(size=n)
    max_m = 4.3
    dev = E.Sfac(L, np.array(K), 4)
    dev.set_radial(f_np, df_np, max_m)
    host = E.Sfac(L, np.array(K), 4)
    host.set_A(f_cb, max_m)
    orc = O.OracleSfac(L, np.array(K), 4)
    orc.set_A_callback(f_cb, max_m)
    g, h, o = _run(dev, q, x), _run(host, q, x), _run(orc, q, x)
    # the same images and weights: device tables agree with the host tables
    # to the interpolation error
    assert abs(g["en"] - h["en"]) <= 1e-9 * abs(h["en"])
    assert np.abs(g["vir"] - h["vir"]).max() <= 1e-8 * np.abs(h["vir"]).max()
    assert rel_rms(g["dx"], h["dx"]) <= 1e-6
    assert rel_rms(g["phi"], h["phi"]) <= 1e-6
    assert_parity(g, o, "radial vs oracle")
