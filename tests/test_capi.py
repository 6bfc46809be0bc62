"""CPU tests of the C ABI boundary: libsfac.so builds for sm_100a, loads, and
exports every symbol include/sfac.h declares; the ctypes wrapper offers the
reference wrapper's names; with no GPU the constructor fails cleanly
(NULL -> RuntimeError) instead of crashing.  No kernels are launched."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sfac.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = "\n".join(l for l in txt.splitlines() if not l.lstrip().startswith(("typedef", "#")))
    names = re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", txt, flags=re.M)
    return sorted(set(n for n in names if n not in ("rad_fn",)))


def test_header_declares_reference_interface():
    names = declared_functions()
    for ref_name in ["sfac_ctor", "sfac_dtor", "sfac", "get_S", "set_L", "set_A", "en", "de1", "de2",
                     "potl"]:
        assert ref_name in names


def test_library_exports_every_declared_symbol(libsfac_path):
    lib = ctypes.CDLL(libsfac_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_built_for_sm100a(libsfac_path):
    import subprocess

    out = subprocess.run(["cuobjdump", "--list-elf", libsfac_path], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_wrapper_has_reference_names():
    from ewaldcorrel_b200 import ewald

    for name in ["describe_sfac", "Sfac", "eta", "ewald_f", "LofS", "SofL"]:
        assert hasattr(ewald, name)
    for meth in ["get_S", "sfac", "set_A", "set_L"]:
        assert callable(getattr(ewald.Sfac, meth))
    assert ewald.eta == 0.5
    L = np.array([9.0, 10.0, 11.0, 2.0, -0.1, 1.0])
    np.testing.assert_array_equal(ewald.SofL(ewald.LofS(L)), L)


def test_ewald_f_matches_reference_formula():
    from math import exp, pi

    from ewaldcorrel_b200 import ewald

    class P:
        class contents:
            value = 0.0

    for r2 in [0.0, 1e-11, 0.3, 2.0]:
        v = ewald.ewald_f(r2, P, None)
        if r2 < 1e-10:
            assert v == 0.0 and P.contents.value == 0.0
        else:
            fac = -(pi / 0.5) ** 2
            assert v == exp(r2 * fac) / (r2 * pi)
            assert P.contents.value == (fac - 1.0 / r2) * v


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_only_the_checking_build_checks(libsfac_path):
    """sfac_check_enabled makes no CUDA call: 0 in the product library, 1 in
    the index-checking one (-DSPME_CHECK), which exports the same symbols."""
    import ctypes

    from ewaldcorrel_b200 import build

    assert ctypes.CDLL(libsfac_path).sfac_check_enabled() == 0
    if not os.path.exists(build.LIB_CHECK):
        pytest.skip("libsfac_check.so not built")
    chk = ctypes.CDLL(build.LIB_CHECK)
    assert chk.sfac_check_enabled() == 1
    for name in declared_functions():
        assert hasattr(chk, name), name


def test_ctor_without_gpu_returns_null(libsfac_path):
    from ewaldcorrel_b200 import ewald

    with pytest.raises(RuntimeError):
        ewald.Sfac(np.array([1.0, 1, 1, 0, 0, 0]), np.array([8, 8, 8]), 4)


def test_ctor_rejects_bad_arguments(libsfac_path):
    """Bad order / K return NULL before touching the device (sfac.cpp:41-51
    threw exceptions through extern "C"; here they are NULL returns)."""
    from ewaldcorrel_b200 import ewald

    for K, order in [((8, 8, 8), 3), ((8, 8, 8), 10), ((0, 8, 8), 4), ((8, -1, 8), 4)]:
        with pytest.raises(RuntimeError):
            ewald.Sfac(np.array([1.0, 1, 1, 0, 0, 0]), np.array(K), order)


def test_null_handle_calls_are_safe(libsfac_path):
    lib = ctypes.CDLL(libsfac_path)
    lib.en.restype = ctypes.c_double
    lib.en.argtypes = [ctypes.c_void_p]
    assert lib.en(None) == 0.0
    lib.sfac_dtor.argtypes = [ctypes.c_void_p]
    lib.sfac_dtor(None)
