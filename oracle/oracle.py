"""CPU oracle loader -- TEST INFRASTRUCTURE ONLY.

Loads, through ctypes, the two CPU implementations of the SPME
reciprocal-space path that the tests and the benchmark's CPU-baseline leg
check the CUDA path against:

* ``OracleSfac``: the project's FP64 C restatement (``oracle/liborc.so``,
  built from ``spme_oracle.c``); always available.
* ``RefSfac``: the reference's own ``sfac.cpp`` compiled unmodified against
  the project FFTW-API shim (``oracle/_ref/libsfac_ref.so``); present where
  the reference sources were available at build time.

Both mirror the method names of the reference's ``ewald.Sfac``
(ewald.py:70-122).  Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_LIB = os.path.join(HERE, "liborc.so")
REF_LIB = os.path.join(HERE, "_ref", "libsfac_ref.so")

RAD_FN = ctypes.CFUNCTYPE(c_double, c_double, POINTER(c_double), c_void_p)

_dbl = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_int = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

_libs: dict = {}


def _load(path: str, prefix: str):
    key = (path, prefix)
    if key in _libs:
        return _libs[key]
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run `make -C oracle all ref`)")
    lib = ctypes.CDLL(path)

    def fn(name, res, *args):
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = list(args)
        return f

    api = {
        "ctor": fn("ctor" if prefix else "sfac_ctor", c_void_p, _dbl, _int, c_int),
        "dtor": fn("dtor" if prefix else "sfac_dtor", None, c_void_p),
        "sfac": fn("sfac_run" if prefix else "sfac", None, c_void_p, c_int, _dbl, _dbl),
        "get_S": fn("get_S", POINTER(c_double), c_void_p),
        "set_L": fn("set_L", None, c_void_p, _dbl),
        "set_A": fn("set_A", c_int, c_void_p, c_void_p, c_double, c_void_p),
        "en": fn("en", c_double, c_void_p),
        "de1": fn("de1", c_double, c_void_p, _dbl),
        "de2": fn("de2", None, c_void_p, c_int, _dbl, _dbl, _dbl),
        "potl": fn("potl", None, c_void_p, c_int, _dbl, _dbl),
    }
    if prefix:
        api["sort"] = fn("sort", c_int, c_void_p, c_int, _dbl, _int, _int, _dbl)
        api["get_spread"] = fn("get_spread", POINTER(c_double), c_void_p)
        api["get_A"] = fn("get_A", POINTER(c_double), c_void_p)
        api["ewald_rad"] = lib.orc_ewald_rad
        api["bspl_value"] = fn("bspl_value", c_double, c_int, c_double, c_int)
        api["bspline_table"] = fn("bspline_table", None, c_int, _dbl)
        api["bspline_moduli"] = fn("bspline_moduli", None, c_int, c_int, _dbl)
        api["cell_consts"] = fn("cell_consts", None, _dbl, _dbl, _dbl)
        api["fft1d"] = lib.shim_fft1d
        api["fft1d"].restype = None
        api["fft1d"].argtypes = [c_int, _dbl, _dbl, c_int]
    api["_lib"] = lib
    _libs[key] = api
    return api


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


class _Base:
    """Common ctypes plumbing; mirrors ewald.Sfac (ewald.py:70-122)."""

    prefix = ""
    path = ""

    def __init__(self, L, K, order=4):
        self._api = _load(self.path, self.prefix)
        self.L = np.ascontiguousarray(L, dtype=np.float64)
        self.K = tuple(int(k) for k in np.asarray(K).tolist())
        self.order = int(order)
        self.ldim = self.K[2] // 2 + 1
        h = self._api["ctor"](self.L, np.ascontiguousarray(self.K, dtype=np.int32), self.order)
        if not h:
            raise RuntimeError("Error intializing Sfac.")
        self._h = h
        self._keep = []

    def close(self):
        if getattr(self, "_h", None):
            self._api["dtor"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sfac(self, w, x):
        w = np.ascontiguousarray(w, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert x.shape == (len(w), 3)
        self._api["sfac"](self._h, len(w), w, x)

    def get_S(self):
        """Structure factor (state 0) as complex (K0, K1, ldim), copied."""
        ptr = self._api["get_S"](self._h)
        s = np.ctypeslib.as_array(ptr, shape=(self.K[0], self.K[1], self.ldim, 2))
        return (s[..., 0] + 1j * s[..., 1]).copy()

    def get_grid(self):
        """Real potential grid (state 1) as (K0, K1, K2), copied."""
        ptr = self._api["get_S"](self._h)
        s = np.ctypeslib.as_array(ptr, shape=(self.K[0], self.K[1], 2 * self.ldim))
        return s[:, :, : self.K[2]].copy()

    def set_L(self, L):
        self.L = np.ascontiguousarray(L, dtype=np.float64)
        self._api["set_L"](self._h, self.L)

    def set_A_callback(self, f, max_m, info=None):
        cb = RAD_FN(f)
        self._keep.append(cb)
        rc = self._api["set_A"](self._h, ctypes.cast(cb, c_void_p), float(max_m), info)
        if rc != 0:
            raise RuntimeError("Error (%d) setting A-array." % rc)

    def set_ewald(self, eta, max_m):
        """set_A with the C twin of ewald.ewald_f (oracle/spme_oracle.c)."""
        orc = _load(ORC_LIB, "orc_")
        box = ctypes.c_double(float(eta))
        self._keep.append(box)
        fptr = ctypes.cast(orc["ewald_rad"], c_void_p)
        rc = self._api["set_A"](self._h, fptr, float(max_m), ctypes.cast(ctypes.byref(box), c_void_p))
        if rc != 0:
            raise RuntimeError("Error (%d) setting A-array." % rc)

    def en(self):
        return self._api["en"](self._h)

    def de1(self, vir):
        return self._api["de1"](self._h, vir)

    def de2(self, n, w, x, dx):
        self._api["de2"](self._h, int(n), np.ascontiguousarray(w, dtype=np.float64),
                         np.ascontiguousarray(x, dtype=np.float64), dx)

    def potl(self, n, x, phi):
        self._api["potl"](self._h, int(n), np.ascontiguousarray(x, dtype=np.float64), phi)


class OracleSfac(_Base):
    """The project's FP64 C restatement (spme_oracle.c)."""

    prefix = "orc_"
    path = ORC_LIB

    def sort(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.shape[0]
        keys = np.zeros(max(n, 1), np.int32)
        perm = np.zeros(max(n, 1), np.int32)
        frac = np.zeros((max(n, 1), 3), np.float64)
        self._api["sort"](self._h, n, x, keys, perm, frac)
        return keys[:n], perm[:n], frac[:n]

    def get_spread(self):
        ptr = self._api["get_spread"](self._h)
        return np.ctypeslib.as_array(ptr, shape=self.K).copy()

    def get_A(self):
        n = self.K[0] * self.K[1] * self.ldim
        ptr = self._api["get_A"](self._h)
        a = np.ctypeslib.as_array(ptr, shape=(7 * n,)).copy()
        return a[:n].reshape(self.K[0], self.K[1], self.ldim), a[n:].reshape(self.K[0], self.K[1], self.ldim, 6)


class RefSfac(_Base):
    """The reference's sfac.cpp compiled unmodified (oracle/_ref)."""

    prefix = ""
    path = REF_LIB


def bspline_table(order):
    api = _load(ORC_LIB, "orc_")
    M = np.zeros(order * order)
    api["bspline_table"](order, M)
    return M.reshape(order, order)


def bspline_moduli(n, order):
    api = _load(ORC_LIB, "orc_")
    out = np.zeros(n)
    api["bspline_moduli"](n, order, out)
    return out


def bspl_value(order, x, j):
    return _load(ORC_LIB, "orc_")["bspl_value"](order, x, j)


def fft1d(z, sign=-1):
    api = _load(ORC_LIB, "orc_")
    z = np.ascontiguousarray(z, dtype=np.complex128)
    inp = z.view(np.float64).copy()
    out = np.zeros_like(inp)
    api["fft1d"](len(z), inp, out, sign)
    return out.view(np.complex128)


def ewald_f(eta):
    """Python twin of ewald.ewald_f (ewald.py:124-132) for a given eta."""
    from math import exp, pi

    fac = -((pi / eta) ** 2)

    def f(r2, ptr, info):
        if r2 < 1e-10:
            ptr[0] = 0.0
            return 0.0
        v = exp(r2 * fac) / (r2 * pi)
        ptr[0] = (fac - 1.0 / r2) * v
        return v

    return f


def LofS(L):
    """Lower-triangular box matrix from the 6-vector (ewald.py:134-138)."""
    return np.array([[L[0], 0.0, 0.0], [L[3], L[1], 0.0], [L[4], L[5], L[2]]])


def SofL(L):
    """6-vector from the box matrix (ewald.py:139-140)."""
    return np.array([L[0, 0], L[1, 1], L[2, 2], L[1, 0], L[2, 0], L[2, 1]])


def real_space(L, x, q, eta, rcut):
    """FP64 restatement of the real-space Ewald term and its corrections, all
    pairs (O(N^2), small systems only), minimum image.  With the reference's
    influence function f(z) = exp(-z pi^2/eta^2)/(pi z) (ewald.py:124-132)
    the reciprocal sum is the erfc-split long-range part of the CGS Coulomb
    energy, so (notes.tex:68-79, E_self being the "correction energy" there):
      E_real = 1/2 sum_{i != j, r < rcut} q_i q_j erfc(eta r)/r,
      E_self = -eta/sqrt(pi) sum q^2,
      E_net  = -pi (sum q)^2 / (2 V eta^2)  (the "further corrections ... if
               sum q != 0" the notes mention: a neutralising background).
    Returns (E_real, E_self, E_net, vir[6], dx) with vir = -W/V,
    W = sum_pairs q q phi'(r)/r r r^T, in de1's [xx, yy, zz, yx, zx, zy]
    order plus the background's -pi Q^2/(2 eta^2 V^2) on the diagonal, and dx
    = dE_real/dx."""
    from scipy.special import erfc

    Lm = LofS(L)
    V = L[0] * L[1] * L[2]
    iLt = np.linalg.inv(Lm)  # s = x @ iLt
    x = np.asarray(x, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    s = x @ iLt
    n = len(q)
    e = 0.0
    W = np.zeros((3, 3))
    dx = np.zeros((n, 3))
    for i in range(n):
        ds = s - s[i]
        ds -= np.rint(ds)
        d = ds @ Lm  # r_j - r_i
        r2 = np.einsum("ij,ij->i", d, d)
        mask = (r2 < rcut * rcut) & (np.arange(n) != i)
        if not mask.any():
            continue
        r = np.sqrt(r2[mask])
        dd = d[mask]
        qq = q[i] * q[mask]
        phi = erfc(eta * r) / r
        dphi = -(2.0 * eta / np.sqrt(np.pi) * np.exp(-(eta * r) ** 2) + phi) / r
        e += 0.5 * np.sum(qq * phi)
        t = qq * dphi / r
        dx[i] = -np.sum(t[:, None] * dd, axis=0)
        W += 0.5 * np.einsum("k,ka,kb->ab", t, dd, dd)
    Q = q.sum()
    e_self = -eta / np.sqrt(np.pi) * np.sum(q * q)
    e_net = -np.pi * Q * Q / (2.0 * V * eta * eta)
    vir = SofL(W) / -V
    vir[:3] += -np.pi * Q * Q / (2.0 * eta * eta * V * V)
    return e, e_self, e_net, vir, dx


def real_space_scale(L, x, q, eta, rcut):
    """Sum of |pair energies| of real_space's E_real, 1/2 sum |q_i q_j| erfc(eta r)/r
    over the same pairs: the magnitude against which the rounding of a sum of
    terms of both signs is measured."""
    from scipy.special import erfc

    Lm = LofS(L)
    s = np.asarray(x, dtype=np.float64) @ np.linalg.inv(Lm)
    q = np.asarray(q, dtype=np.float64)
    n = len(q)
    tot = 0.0
    for i in range(n):
        ds = s - s[i]
        ds -= np.rint(ds)
        d = ds @ Lm
        r2 = np.einsum("ij,ij->i", d, d)
        mask = (r2 < rcut * rcut) & (np.arange(n) != i)
        r = np.sqrt(r2[mask])
        tot += 0.5 * np.sum(np.abs(q[i] * q[mask]) * erfc(eta * r) / r)
    return tot


def sk_radial(L, K, acc, nbins, kmax):
    """FP64 restatement of the radial binning of a sum of |S|^2 over the
    stored half-space modes (the reference's plot.py:9-32, on the general
    box): |k| = 2 pi |m|, m = inv(box) n with n the signed x/y frequency indices
    and the stored z index; bin floor(|k| / dk), dk = kmax / nbins; returns
    per-bin (sums, counts).  plot.py folds the stored z index as if that axis
    had ldim points (index >= ldim/2 taken as negative); this restatement, like
    the device code, uses the stored z index as it is."""
    K0, K1, K2 = K
    ldim = K2 // 2 + 1
    n0 = np.arange(K0)
    n0 = np.where(n0 > K0 // 2, n0 - K0, n0).astype(np.float64)
    n1 = np.arange(K1)
    n1 = np.where(n1 > K1 // 2, n1 - K1, n1).astype(np.float64)
    n2 = np.arange(ldim).astype(np.float64)
    N0, N1, N2 = np.meshgrid(n0, n1, n2, indexing="ij")
    # m . x = n . s with s = x @ inv(box), box rows a, b, c: m = inv(box) n
    # (set_A's mx, my, mz, sfac.cpp:240-262)
    iL = np.linalg.inv(LofS(L))
    M = np.stack([N0, N1, N2], axis=-1) @ iL.T
    k = 2.0 * np.pi * np.sqrt(np.sum(M * M, axis=-1))
    b = np.floor(k / (kmax / nbins)).astype(np.int64).ravel()
    v = np.asarray(acc, dtype=np.float64).ravel()
    keep = (b >= 0) & (b < nbins)
    sums = np.bincount(b[keep], weights=v[keep], minlength=nbins)
    counts = np.bincount(b[keep], minlength=nbins).astype(np.float64)
    return sums, counts
