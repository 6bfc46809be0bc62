"""ctypes wrapper of libsfac.so with the interface of the reference's ewald.py.

Same names, argument types and behaviour as frobnitzem/EwaldCorrel's
ewald.py (ewald.py:15-140): ``describe_sfac``, ``Sfac``, ``eta``,
``ewald_f``, ``LofS``, ``SofL``.  The library is loaded from this file's own
directory (as ewald.py:52-53 does), so code written against the reference's
wrapper runs unchanged on the B200 library.

Additions (no counterpart in the reference): ``Sfac.set_ewald`` selects the
on-device FP64 Ewald influence function, ``Sfac.get_grid`` returns the real
potential grid, and ``Sfac.last_error``/``Sfac.launches`` expose the
handle's diagnostics.
"""
from __future__ import annotations

import os
from ctypes import CDLL, POINTER, PYFUNCTYPE, byref, c_char_p, c_double, c_int, c_longlong, c_void_p, cast
from math import exp, pi

import numpy as np
import numpy.ctypeslib as ct

array = np.array

_LIB = None


def _load():
    """Loads libsfac.so from this directory (or the library file that
    EWALDCORREL_LIBSFAC names, e.g. the index-checking libsfac_check.so);
    fails loudly if it is not built."""
    global _LIB
    if _LIB is None:
        here = os.path.dirname(os.path.abspath(__file__))
        path = os.environ.get("EWALDCORREL_LIBSFAC") or os.path.join(here, "libsfac.so")
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is not built: run `python -m ewaldcorrel_b200.build` (needs nvcc)")
        _LIB = CDLL(path)
    return _LIB


def describe_sfac():
    """Declares argument types of the C interface (ewald.py:15-68)."""
    nparr = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    dblarr = POINTER(c_double)

    def nparr_t(*shape):
        return np.ctypeslib.ndpointer(dtype=np.float64, shape=shape, flags="C_CONTIGUOUS")

    def np_intarr_t(*shape):
        return np.ctypeslib.ndpointer(dtype=np.int32, shape=shape, flags="C_CONTIGUOUS")

    def decl(f, res, *args):
        f.argtypes = list(args)
        f.restype = res

    sfac_p = c_void_p
    rad_fn = PYFUNCTYPE(c_double, c_double, POINTER(c_double), c_void_p)
    lib = _load()
    decl(lib.sfac_ctor, sfac_p, nparr_t(6), np_intarr_t(3), c_int)
    decl(lib.sfac_dtor, None, sfac_p)
    decl(lib.sfac, None, sfac_p, c_int, nparr, nparr)
    decl(lib.get_S, dblarr, sfac_p)
    decl(lib.set_L, None, sfac_p, nparr_t(6))
    decl(lib.set_A, c_int, sfac_p, rad_fn, c_double, c_void_p)
    decl(lib.en, c_double, sfac_p)
    decl(lib.de1, c_double, sfac_p, nparr_t(6))
    decl(lib.de2, None, sfac_p, c_int, nparr, nparr, nparr)
    decl(lib.potl, None, sfac_p, c_int, nparr, nparr)
    # additions
    decl(lib.sfac_set_ewald, c_int, sfac_p, c_double, c_double)
    decl(lib.sfac_set_radial, c_int, sfac_p, c_int, nparr, nparr, c_double, c_double)
    decl(lib.sfac_last_error, c_int, sfac_p)
    decl(lib.sfac_error_string, c_char_p, sfac_p)
    decl(lib.sfac_device, c_int, sfac_p)
    decl(lib.sfac_kernel_launches, c_longlong, sfac_p)
    decl(lib.sfac_real_space, c_int, sfac_p, c_int, nparr, nparr, c_double, c_double, nparr_t(10), c_void_p)
    decl(lib.sfac_sk_reset, c_int, sfac_p)
    decl(lib.sfac_sk_accumulate, c_int, sfac_p)
    decl(lib.sfac_sk_get, c_int, sfac_p, nparr, POINTER(c_longlong))
    decl(lib.sfac_sk_radial, c_int, sfac_p, c_int, c_double, nparr, nparr)
    decl(lib.sfac_xc_reset, c_int, sfac_p, c_int)
    decl(lib.sfac_xc_store, c_int, sfac_p, c_int)
    decl(lib.sfac_xc_accumulate, c_int, sfac_p)
    decl(lib.sfac_xc_get, c_int, sfac_p, c_int, nparr, POINTER(c_longlong))
    intarr = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    decl(lib.sfac_debug_sort, c_int, sfac_p, c_int, intarr, intarr)
    decl(lib.sfac_debug_spread, c_int, sfac_p,
         np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS"))
    return sfac_p, rad_fn, lib


class Sfac:
    """One SPME reciprocal-space solver (ewald.py:70-122)."""

    def __init__(self, L, K, order=4):
        sfac_p, rad_fn, libsfac = describe_sfac()
        self._libsfac = libsfac
        self.rad_fn = rad_fn
        K = np.asarray(K)
        self.K = tuple(int(k) for k in K.tolist())
        self.ldim = self.K[2] // 2 + 1
        self._data = libsfac.sfac_ctor(np.asarray(L).astype(np.float64),
                                       K.astype(np.int32), int(order))
        if not self._data:
            raise RuntimeError("Error intializing Sfac.")

    def __getattr__(self, name):
        """Passes the handle as the first argument of these C functions."""
        names = ["sfac_dtor", "en", "de1", "de2", "potl"]
        if name not in names:
            raise AttributeError(name)
        try:
            f = getattr(self._libsfac, name)
        except AttributeError:
            return None
        return lambda *args, **kws: f(self._data, *args, **kws)

    def get_S(self):
        """Structure factor (after sfac) as a complex (K0, K1, ldim) array."""
        Q = self._libsfac.get_S(self._data)
        shape = (self.K[0], self.K[1], self.ldim, 2)
        s = ct.as_array(Q, shape=shape)
        return s[:, :, :, 0] + 1j * s[:, :, :, 1]

    def get_grid(self):
        """Real potential grid (after de1) as a (K0, K1, K2) array (copy)."""
        Q = self._libsfac.get_S(self._data)
        s = ct.as_array(Q, shape=(self.K[0], self.K[1], 2 * self.ldim))
        return s[:, :, : self.K[2]].copy()

    def sfac(self, w, x):
        assert len(w.shape) == 1
        assert x.shape == (len(w), 3)
        self._libsfac.sfac(self._data, len(w), w, x)

    def __del__(self):
        if getattr(self, "_data", None):
            self._libsfac.sfac_dtor(self._data)
            self._data = None

    def set_A(self, f, max_m):
        self.f = f
        self._cb = self.rad_fn(f)  # keep the callback alive
        n = self._libsfac.set_A(self._data, self._cb, max_m, cast(0, c_void_p))
        if n != 0:
            raise RuntimeError("Error (%d) setting A-array." % n)

    def set_ewald(self, beta, max_m):
        """On-device Ewald influence function (same image set as
        set_A(ewald_f, max_m) with eta = beta)."""
        self._ewald = (float(beta), float(max_m))
        self.__dict__.pop("f", None)
        n = self._libsfac.sfac_set_ewald(self._data, float(beta), float(max_m))
        if n != 0:
            raise RuntimeError("Error (%d) setting the Ewald kernel." % n)

    def set_radial(self, f, df, max_m, m2max=None, samples=200001):
        """A radial influence function evaluated on the device (an addition:
        set_A calls a host function once per lattice vector).  f, df:
        vectorised callables giving f(m^2) and f'(m^2), sampled at `samples`
        points of [0, m2max] (default max_m^2)."""
        m2max = float(max_m) ** 2 if m2max is None else float(m2max)
        z = np.linspace(0.0, m2max, int(samples))
        fv = np.ascontiguousarray(f(z), dtype=np.float64)
        dv = np.ascontiguousarray(df(z), dtype=np.float64)
        self.__dict__.pop("f", None)
        self.__dict__.pop("_ewald", None)
        self._radial = (f, df, float(max_m), m2max, int(samples))
        n = self._libsfac.sfac_set_radial(self._data, len(z), fv, dv, m2max, float(max_m))
        if n != 0:
            raise RuntimeError("Error (%d) setting the radial kernel." % n)

    def set_L(self, L):
        """Replaces the box.  Like the reference wrapper (ewald.py:119-122),
        a host influence function is re-tabulated with max_m = 1.0; an
        on-device Ewald kernel is re-set with its own max_m."""
        self._libsfac.set_L(self._data, L)
        if hasattr(self, "f"):
            self.set_A(self.f, 1.0)
        elif hasattr(self, "_ewald"):
            self.set_ewald(*self._ewald)
        elif hasattr(self, "_radial"):
            f, df, max_m, m2max, samples = self._radial
            self.set_radial(f, df, max_m, m2max, samples)

    def real_space(self, w, x, eta, rcut, grad=True):
        """Real-space Ewald term beside this solver's reciprocal sum (an
        addition: the reference's notes give only the self correction,
        notes.tex:73-77).  Returns (E_real, E_self, E_net, vir[6], dx): with
        the Ewald influence function of the same eta, en() + E_real +
        E_self + E_net is the full Ewald energy; vir is E_real's virial in
        de1's convention plus the net-charge term on its diagonal; dx is
        dE_real/dx (n x 3) or None."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = len(w)
        out = np.zeros(10)
        dx = np.zeros((n, 3)) if grad else None
        rc = self._libsfac.sfac_real_space(self._data, n, w, x, float(eta), float(rcut), out,
                                           dx.ctypes.data if grad else None)
        if rc != 0:
            raise RuntimeError("sfac_real_space failed (%d)" % rc)
        vir = out[3:9].copy()
        vir[:3] += out[9]
        return out[0], out[1], out[2], vir, dx

    # structure-factor analysis (additions; run.py:27-47, plot.py:9-32)
    def sk_reset(self):
        if self._libsfac.sfac_sk_reset(self._data) != 0:
            raise RuntimeError("sfac_sk_reset failed")

    def sk_accumulate(self):
        """Adds |S|^2 of the last sfac() to the running sum."""
        if self._libsfac.sfac_sk_accumulate(self._data) != 0:
            raise RuntimeError("sfac_sk_accumulate failed (call sfac first)")

    def sk_get(self):
        """(sum of |S|^2 as a (K0, K1, ldim) array, number of frames)."""
        out = np.zeros((self.K[0], self.K[1], self.ldim))
        frames = c_longlong(0)
        if self._libsfac.sfac_sk_get(self._data, out, byref(frames)) != 0:
            raise RuntimeError("sfac_sk_get failed")
        return out, int(frames.value)

    def sk_radial(self, nbins, kmax):
        """(bin sums, bin counts) of the accumulated |S|^2 over |k| = 2 pi |m|
        in nbins bins of width kmax / nbins."""
        sums, counts = np.zeros(int(nbins)), np.zeros(int(nbins))
        if self._libsfac.sfac_sk_radial(self._data, int(nbins), float(kmax), sums, counts) != 0:
            raise RuntimeError("sfac_sk_radial failed")
        return sums, counts

    # cross-correlations of several densities (additions; gmx_ewald.py:76-95)
    def xc_reset(self, D):
        if self._libsfac.sfac_xc_reset(self._data, int(D)) != 0:
            raise RuntimeError("sfac_xc_reset failed")
        self._xc_D = int(D)

    def xc_store(self, i):
        """Keeps the structure factor of the last sfac() as density i."""
        if self._libsfac.sfac_xc_store(self._data, int(i)) != 0:
            raise RuntimeError("sfac_xc_store failed (call xc_reset, then sfac)")

    def xc_accumulate(self):
        """C[k] += Q[i] conj(Q[j]) for i <= j over the stored densities."""
        if self._libsfac.sfac_xc_accumulate(self._data) != 0:
            raise RuntimeError("sfac_xc_accumulate failed")

    def xc_get(self):
        """(C as a (D(D+1)/2, K0, K1, ldim) complex array, number of frames)."""
        D = self._xc_D
        C = np.zeros((D * (D + 1) // 2, self.K[0], self.K[1], self.ldim), np.complex128)
        frames = c_longlong(0)
        for k in range(C.shape[0]):
            buf = np.zeros(2 * C[k].size)
            if self._libsfac.sfac_xc_get(self._data, k, buf, byref(frames)) != 0:
                raise RuntimeError("sfac_xc_get failed")
            C[k] = (buf[0::2] + 1j * buf[1::2]).reshape(C[k].shape)
        return C, int(frames.value)

    # diagnostics (additions)
    def last_error(self):
        return self._libsfac.sfac_last_error(self._data), \
            (self._libsfac.sfac_error_string(self._data) or b"").decode()

    def launches(self):
        return int(self._libsfac.sfac_kernel_launches(self._data))

    def debug_sort(self, n):
        keys = np.zeros(max(n, 1), np.int32)
        perm = np.zeros(max(n, 1), np.int32)
        if self._libsfac.sfac_debug_sort(self._data, n, keys, perm) != 0:
            raise RuntimeError("debug_sort failed")
        return keys[:n], perm[:n]

    def debug_spread(self):
        g = np.zeros(self.K, np.float32)
        if self._libsfac.sfac_debug_spread(self._data, g) != 0:
            raise RuntimeError("debug_spread failed (needs state 0)")
        return g


eta = 0.5
_fac = -(pi / eta) ** 2


def ewald_f(r2, ptr, info):
    """Ewald influence function f(r2) and f'(r2) (ewald.py:124-132)."""
    if r2 < 1e-10:
        ptr.contents.value = 0.0
        return 0.0
    f = exp(r2 * _fac) / (r2 * pi)
    ptr.contents.value = (_fac - 1.0 / r2) * f
    return f


def LofS(L):
    return np.array([[L[0], 0.0, 0.0],
                     [L[3], L[1], 0.0],
                     [L[4], L[5], L[2]]])


def SofL(L):
    return np.array([L[0, 0], L[1, 1], L[2, 2], L[1, 0], L[2, 0], L[2, 1]])
