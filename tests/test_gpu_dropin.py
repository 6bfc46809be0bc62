"""Drop-in test: libsfac.so bound through the reference's OWN ctypes wrapper.

`make -C oracle ref` copies the reference's ewald.py byte for byte into
oracle/_ref/ (a git-ignored build output, like the reference's compiled
sfac.cpp beside it).  Here it is placed, unmodified (its SHA-256 is checked),
in a fresh directory next to this library's libsfac.so -- ewald.py loads the
library from its own directory (ewald.py:52-53) -- imported, and put through
the checks of the reference's test.py (test.py:12-37 line test, 64-132 test(),
39-62 test_potl()) and the numbers of test.log.ref.  The finite-difference
steps suit an FP32 pipeline (test.py's h = 1e-7 with 1e-7/1e-8 bounds assumes
FP64 throughout)."""
import hashlib
import importlib.util
import json
import os
import shutil

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
REF_WRAPPER = os.path.join(ROOT, "oracle", "_ref", "ewald.py")
# SHA-256 of the reference's ewald.py (frobnitzem/EwaldCorrel), the file the
# test must load unchanged.
REF_EWALD_SHA256 = "f70256aa7f4de7a6f2e6d104ac3b9b1f0ca4f1c0b06832d631c71ceb1d2bd571"

TESTPY_L = np.array([9.0, 10.0, 11.0, 2.0, -0.1, 1.0])
TESTPY_CRDS = np.array([[0.1, 0.5, 0.1], [0.9, 0.4, 0.1], [0.1, 0.4, 0.9], [0.9, 0.5, 0.9]])


def _sha256(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def test_pinned_wrapper_hash_is_the_references():
    """Where the reference checkout is present, the pinned hash is that of its
    ewald.py, and the copy `make -C oracle ref` made is identical."""
    ref = os.path.join(os.environ.get("EWALDCORREL_REFERENCE", "/root/reference"), "ewald.py")
    if not os.path.exists(ref):
        pytest.skip("reference checkout not present")
    assert _sha256(ref) == REF_EWALD_SHA256
    if os.path.exists(REF_WRAPPER):
        assert _sha256(REF_WRAPPER) == REF_EWALD_SHA256


@pytest.fixture(scope="module")
def ref_ewald(libsfac_path, tmp_path_factory):
    """The reference's ewald.py, unmodified, loaded beside libsfac.so."""
    if not os.path.exists(REF_WRAPPER):
        pytest.skip("oracle/_ref/ewald.py not built (make -C oracle ref needs the reference checkout)")
    assert _sha256(REF_WRAPPER) == REF_EWALD_SHA256, "oracle/_ref/ewald.py differs from the reference's"
    d = tmp_path_factory.mktemp("dropin")
    shutil.copyfile(REF_WRAPPER, d / "ewald.py")
    os.symlink(libsfac_path, d / "libsfac.so")
    assert _sha256(d / "ewald.py") == REF_EWALD_SHA256
    spec = importlib.util.spec_from_file_location("reference_ewald_dropin", str(d / "ewald.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _num_diff(f, x, h):
    """Central differences of f at x (test.py's num_diff with step h)."""
    x = np.asarray(x, dtype=np.float64)
    flat = x.ravel()
    out = np.zeros(flat.size)
    for i in range(flat.size):
        a = flat.copy()
        b = flat.copy()
        a[i] += h
        b[i] -= h
        out[i] = (f(a.reshape(x.shape)) - f(b.reshape(x.shape))) / (2 * h)
    return out.reshape(x.shape)


@pytest.mark.gpu
def test_reference_wrapper_test_py(ref_ewald):
    """test.py:test() through the unmodified wrapper: line test, en == de1,
    FD gradient, FD virial through set_L (which re-runs set_A(f, 1.0)), and
    test.log.ref's energy, gradient and virial."""
    ew = ref_ewald
    log = json.load(open(os.path.join(GOLD, "test_log_ref.json")))
    L = TESTPY_L.copy()
    V = L[0] * L[1] * L[2]
    N = 4
    atoms = np.dot(TESTPY_CRDS, ew.LofS(L))
    q = np.ones(N)
    s = ew.Sfac(L, np.array([12, 13, 14], dtype=int), 4)
    s.set_A(ew.ewald_f, 1.0)
    s.sfac(q, atoms)

    # test.py:12-37: spline S along each axis against the exact DFT
    M = s.get_S()
    mx = np.arange(12); mx[7:] -= 12
    my = np.arange(13); my[7:] -= 13
    mz = np.arange(8)
    sx = sum(qq * np.exp(-2j * np.pi * c[0] * mx) for qq, c in zip(q, TESTPY_CRDS))
    sy = sum(qq * np.exp(-2j * np.pi * c[1] * my) for qq, c in zip(q, TESTPY_CRDS))
    sz = sum(qq * np.exp(-2j * np.pi * c[2] * mz) for qq, c in zip(q, TESTPY_CRDS))
    assert np.abs(M[:, 0, 0] - sx)[:3].max() < 0.01
    assert np.abs(M[0, :, 0] - sy)[:3].max() < 0.01
    assert np.abs(M[0, 0, :] - sz)[:4].max() < 0.1
    np.testing.assert_allclose(M[0, 0].real, log["spl_S00"], atol=2e-6)

    def Ex(x):
        s.sfac(q, np.ascontiguousarray(x.reshape((N, 3))))
        return s.en()

    dx0 = _num_diff(Ex, atoms, 1e-3)
    s.sfac(q, atoms)
    en0 = s.en()
    vir = np.zeros(6)
    en1 = s.de1(vir)
    assert np.abs(en1 - en0) < 1e-14  # test.py:100
    assert abs(en0 - log["E"]) <= 1e-6 * log["E"]
    dx = np.zeros((N, 3))
    s.de2(N, q, atoms, dx)
    assert np.abs(dx - dx0).max() < 2e-3 * np.abs(dx0).max()
    np.testing.assert_allclose(dx.ravel(), log["spl_dx"], atol=2e-6)
    np.testing.assert_allclose(vir, log["spl_vir"], rtol=0, atol=1e-5 * np.abs(log["spl_vir"]).max())

    def EL(LL):
        s.set_L(np.ascontiguousarray(LL))
        return s.en()

    s.sfac(q, atoms)
    Pi = ew.LofS(_num_diff(EL, L, 1e-3)).transpose()
    Pi = ew.SofL(np.dot(Pi, ew.LofS(L)).transpose()) / (-V)
    assert np.abs(vir - Pi).max() < 2e-3 * np.abs(vir).max()


@pytest.mark.gpu
def test_reference_wrapper_test_potl(ref_ewald):
    """test.py:test_potl() through the unmodified wrapper: phi against the
    compiled reference's values, and E = q . phi / 2."""
    ew = ref_ewald
    g = np.load(os.path.join(GOLD, "testpy_ref.npz"))
    N = 4
    atoms = np.dot(TESTPY_CRDS, ew.LofS(TESTPY_L))
    q = (np.arange(N) % 2) * 0.5 + 0.5
    s = ew.Sfac(TESTPY_L.copy(), np.array([12, 13, 14], dtype=int), 4)
    s.set_A(ew.ewald_f, 1.0)
    s.sfac(q, atoms)
    en0 = s.en()
    vir = np.zeros(6)
    en1 = s.de1(vir)
    assert en0 == en1
    pot = np.zeros(N)
    s.potl(N, atoms, pot)
    np.testing.assert_allclose(q, g["q_potl"])
    err = np.sqrt(np.mean((pot - g["phi_potl"]) ** 2) / np.mean(g["phi_potl"] ** 2))
    assert err < 1e-5
    assert abs(0.5 * np.dot(q, pot) - en0) <= 2e-6 * abs(en0)


@pytest.mark.gpu
def test_reference_wrapper_constructor_error(ref_ewald):
    """A bad order makes sfac_ctor return NULL, so the unmodified wrapper
    raises its own error (ewald.py:80-81) instead of crashing."""
    with pytest.raises(RuntimeError, match="intializing"):
        ref_ewald.Sfac(TESTPY_L.copy(), np.array([12, 13, 14], dtype=int), 3)
