"""Real-space Ewald term (sfac_real_space): parity with the FP64 oracle and
the physical check that the full Ewald energy does not depend on the
splitting parameter eta (notes.tex:68-79)."""
import numpy as np
import pytest

from ewaldcorrel_b200 import configs
from oracle import oracle as O
from tests.spme_testlib import rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _libs(libsfac_path, oracle_built):
    return libsfac_path


def E():
    from ewaldcorrel_b200 import ewald

    return ewald


def _check(g, o, name, scale=0.0):
    """Energy within 1e-6 of E_real, or within 2e-7 of `scale` (the sum of
    |pair energies|) when that is larger: with charges of random sign E_real
    is a small residue of cancelling terms, each computed in FP32."""
    e, es, en, vir, dx = g
    oe, oes, oen, ovir, odx = o
    assert abs(e - oe) <= max(1e-6 * abs(oe), 2e-7 * scale), f"{name}: E_real {e!r} vs {oe!r} (scale {scale!r})"
    assert abs(es - oes) <= 1e-12 * abs(oes), f"{name}: E_self"
    assert abs(en - oen) <= 1e-12 * max(abs(oen), 1e-300) + 1e-12, f"{name}: E_net"
    assert np.abs(vir - ovir).max() <= 1e-5 * np.abs(ovir).max(), f"{name}: virial"
    assert rel_rms(dx, odx) <= 1e-5, f"{name}: dE/dx"


def test_real_space_matches_oracle_cubic():
    c = configs.cfg1_plain()
    s = E().Sfac(c.L, np.array(c.K), c.order)
    g = s.real_space(c.q, c.x, c.beta, 1.45)
    o = O.real_space(c.L, c.x, c.q, c.beta, 1.45)
    _check(g, o, "cfg1")


def test_real_space_matches_oracle_triclinic_charged():
    rng = np.random.default_rng(21)
    L = np.array([4.0, 3.6, 3.8, 0.9, -0.7, 0.5])
    n = 700
    x = rng.uniform(0, 1, size=(n, 3)) @ O.LofS(L) + rng.normal(0, 2.0, size=(n, 3))  # unwrapped positions
    q = rng.normal(size=n)  # not neutral: exercises the background term
    s = E().Sfac(L, np.array([24, 24, 24]), 4)
    g = s.real_space(q, x, 2.9, 1.7)
    o = O.real_space(L, x, q, 2.9, 1.7)
    _check(g, o, "triclinic")


def test_real_space_matches_oracle_water_close_pairs():
    """Rigid 3-site water at liquid density (O-H 0.0957 nm): large opposing
    intramolecular terms in every gradient, a 6^3 coarse grid whose
    neighbour runs wrap around the box."""
    rng = np.random.default_rng(23)
    nmol, side = 1000, 3.1
    centers = rng.uniform(0, side, size=(nmol, 3))
    u = rng.normal(size=(nmol, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    v = np.cross(u, rng.normal(size=(nmol, 3)))
    v /= np.linalg.norm(v, axis=1)[:, None]
    d, th = 0.09572, np.radians(104.52)
    x = np.empty((nmol, 3, 3))
    x[:, 0] = centers
    x[:, 1] = centers + d * (np.cos(th / 2) * u + np.sin(th / 2) * v)
    x[:, 2] = centers + d * (np.cos(th / 2) * u - np.sin(th / 2) * v)
    x = x.reshape(-1, 3)
    q = np.tile([-0.834, 0.417, 0.417], nmol)
    L = np.array([side, side, side, 0.0, 0.0, 0.0])
    s = E().Sfac(L, np.array([32, 32, 32]), 4)
    g = s.real_space(q, x, 3.12, 1.0)
    o = O.real_space(L, x, q, 3.12, 1.0)
    _check(g, o, "water")


@pytest.mark.parametrize("case", ["sparse_rows", "mixed_axes", "clustered"])
def test_real_space_traversal_cases(case):
    """The warp walk's paths: sparse rows (a warp's 32 points span several
    rows; z runs that cover whole rows), axes with fewer than five coarse
    cells next to axes with more (image reduction on some passes only), and
    coarse cells holding more points than the sort's in-place fix-up takes."""
    rng = np.random.default_rng({"sparse_rows": 31, "mixed_axes": 32, "clustered": 33}[case])
    if case == "sparse_rows":
        L, n, rc = np.array([6.0, 5.5, 7.0, 1.0, -1.2, 0.8]), 300, 1.0
        x = rng.uniform(-3, 9, size=(n, 3))
    elif case == "mixed_axes":
        L, n, rc = np.array([3.0, 6.0, 12.0, 0.0, 0.0, 0.0]), 1500, 1.2
        x = rng.uniform(-3, 9, size=(n, 3))
    else:
        L, rc = np.array([5.0, 5.0, 5.0, 0.0, 0.0, 0.0]), 1.0
        centres = rng.uniform(0, 5, size=(6, 3))
        x = np.repeat(centres, 400, axis=0) + rng.normal(0, 0.08, size=(2400, 3))
        x = np.concatenate([x, rng.uniform(0, 5, size=(600, 3))])
        n = len(x)
    q = rng.normal(size=n)
    s = E().Sfac(L, np.array([24, 24, 24]), 4)
    g = s.real_space(q, x, 3.0, rc)
    o = O.real_space(L, x, q, 3.0, rc)
    _check(g, o, case, O.real_space_scale(L, x, q, 3.0, rc))


def test_real_space_is_deterministic():
    """Warps take their groups from a counter, so which warp evaluates which
    group changes from call to call; the sums must not."""
    c = configs.cfg1_plain()
    s = E().Sfac(c.L, np.array(c.K), c.order)
    a = s.real_space(c.q, c.x, c.beta, 1.45)
    for _ in range(3):
        b = s.real_space(c.q, c.x, c.beta, 1.45)
        assert a[0] == b[0] and a[1] == b[1] and a[2] == b[2]
        np.testing.assert_array_equal(a[3], b[3])
        np.testing.assert_array_equal(a[4], b[4])


def test_real_space_rejects_long_cutoff():
    c = configs.cfg1_plain()
    s = E().Sfac(c.L, np.array(c.K), c.order)
    with pytest.raises(RuntimeError):
        s.real_space(c.q, c.x, c.beta, 1.6)  # more than half the 3 nm box


def _total(L, K, order, x, q, eta, rcut):
    s = E().Sfac(L, np.array(K), order)
    s.set_ewald(eta, eta * np.sqrt(np.log(1e16)) / np.pi)
    s.sfac(q, x)
    vir = np.zeros(6)
    e_rec = s.de1(vir)
    n = len(q)
    dx = np.zeros((n, 3))
    s.de2(n, q, x, dx)
    e_real, e_self, e_net, vir_real, dx_real = s.real_space(q, x, eta, rcut)
    return e_rec + e_real + e_self + e_net, dx + dx_real, vir + vir_real, (e_rec, e_real, e_self)


def test_total_ewald_energy_independent_of_eta():
    """E_recip + E_real + E_self: each term moves by O(1) between the two
    splittings, their sum (the Coulomb energy of the periodic system) not."""
    c = configs.cfg1_plain()
    K, order, rcut = (64, 64, 64), 8, 1.45
    ea, fa, va, parts_a = _total(c.L, K, order, c.x, c.q, 3.9, rcut)
    eb, fb, vb, parts_b = _total(c.L, K, order, c.x, c.q, 4.6, rcut)
    assert abs(parts_a[0] - parts_b[0]) > 1e-2 * abs(ea)  # the split really moved
    assert abs(ea - eb) <= 2e-6 * abs(ea), (ea, eb, parts_a, parts_b)
    assert rel_rms(fa, fb) <= 2e-5
    assert np.abs(va - vb).max() <= 2e-5 * np.abs(va).max()


def test_real_space_device_entry_matches_host():
    import torch

    c = configs.cfg1_plain()
    s = E().Sfac(c.L, np.array(c.K), c.order)
    host = s.real_space(c.q, c.x, c.beta, 1.45)
    lib = s._libsfac
    import ctypes

    lib.sfac_real_space_device.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 2 + \
        [ctypes.c_double, ctypes.c_double] + [ctypes.c_void_p] * 2
    lib.sfac_real_space_device.restype = ctypes.c_int
    dev = torch.device("cuda", lib.sfac_device(s._data))
    x = torch.from_numpy(c.x).to(dev)
    q = torch.from_numpy(c.q).to(dev)
    out = torch.zeros(10, dtype=torch.float64, device=dev)
    dx = torch.zeros((c.n, 3), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    assert lib.sfac_real_space_device(s._data, c.n, x.data_ptr(), q.data_ptr(), c.beta, 1.45, out.data_ptr(),
                                      dx.data_ptr()) == 0
    torch.cuda.synchronize(dev)
    o = out.cpu().numpy()
    assert o[0] == host[0] and o[1] == host[1]
    np.testing.assert_array_equal(dx.cpu().numpy(), host[4])
