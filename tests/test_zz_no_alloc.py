"""GPU test of sfac_cell_sort_noalloc, the cell sort that allocates no device
memory (for host programs whose device memory is already held by their own
pool, or whose loops must not pay cudaMalloc's device-wide synchronisation).

It is called through the C ABI on device arrays and must give exactly the
keys and order of the existing entry point (sfac() + sfac_debug_sort), on two
different systems in a row: the shared scratch array keeps the first call's
contents, which must not leak into the second.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib(libsfac_path):
    from ewaldcorrel_b200 import ewald

    _, _, lib = ewald.describe_sfac()
    f = lib.sfac_cell_sort_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [np.ctypeslib.ndpointer(np.float64, shape=(6,), flags="C_CONTIGUOUS"),
                  np.ctypeslib.ndpointer(np.int32, shape=(3,), flags="C_CONTIGUOUS"), ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return f


def _noalloc_sort(f, L, K, x):
    import torch

    n = len(x)
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
    keys = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    perm = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = f(np.asarray(L, dtype=np.float64), np.asarray(K, dtype=np.int32), n, xd.data_ptr(), keys.data_ptr(),
           perm.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, keys.cpu().numpy()[:n], perm.cpu().numpy()[:n]


def _existing_sort(L, K, x):
    from ewaldcorrel_b200 import ewald

    n = len(x)
    s = ewald.Sfac(np.asarray(L, dtype=np.float64), np.asarray(K), 4)
    s.sfac(np.ones(n), np.ascontiguousarray(x, dtype=np.float64))
    return s.debug_sort(n)


def test_noalloc_sort_matches_existing_entry_point(libsfac_path):
    f = _lib(libsfac_path)
    rng = np.random.default_rng(77)
    systems = [
        (np.array([2.0, 1.9, 2.1, 0.4, -0.2, 0.3]), (12, 13, 14), rng.uniform(-4, 6, size=(20000, 3))),
        (np.array([10.0, 10.0, 10.0, 0.0, 0.0, 0.0]), (96, 96, 96), rng.uniform(0, 10, size=(65536, 3))),
    ]
    for L, K, x in systems:  # two calls in a row on the shared scratch
        rc, keys, perm = _noalloc_sort(f, L, K, x)
        assert rc == 0
        k0, p0 = _existing_sort(L, K, x)
        np.testing.assert_array_equal(keys, k0)
        np.testing.assert_array_equal(perm, p0)


def test_noalloc_sort_rejects_more_than_capacity(libsfac_path):
    f = _lib(libsfac_path)
    x = np.zeros((65537, 3))
    rc, _, _ = _noalloc_sort(f, np.array([1.0, 1, 1, 0, 0, 0]), (8, 8, 8), x)
    assert rc == 1
