"""Device-tensor interface to libsfac.so (torch tensors, no host copies).

``SpmeSolver`` owns one C handle and runs full solves on CUDA tensors that
stay resident in HBM: cell sort -> spread -> forward FFT -> convolution
(energy, virial) -> inverse FFT -> gather (dE/dx, phi).  The handle's work is
enqueued on a torch stream, so torch events and ops order with it.

This is plumbing around the C ABI (include/sfac.h); all computation runs in
the library's sm_100a kernels.
"""
from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int, c_void_p

import numpy as np

from . import ewald as _ew

STAGES = ("cell_sort", "spread", "fft_forward", "convolution", "fft_inverse", "gather")


def _lib():
    _, _, lib = _ew.describe_sfac()
    if not getattr(lib, "_device_declared", False):
        lib.sfac_set_stream.argtypes = [c_void_p, c_void_p]
        lib.sfac_set_stream.restype = c_int
        lib.sfac_get_stream.argtypes = [c_void_p]
        lib.sfac_get_stream.restype = c_void_p
        lib.sfac_solve_device.argtypes = [c_void_p, c_int] + [c_void_p] * 5
        lib.sfac_solve_device.restype = c_int
        lib.sfac_solve_device_timed.argtypes = [c_void_p, c_int] + [c_void_p] * 5 + [ctypes.POINTER(c_float)]
        lib.sfac_solve_device_timed.restype = c_int
        lib.sfac_set_graphs.argtypes = [c_void_p, c_int]
        lib.sfac_set_graphs.restype = c_int
        lib.sfac_real_space_device.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_double, c_double, c_void_p,
                                               c_void_p]
        lib.sfac_real_space_device.restype = c_int
        lib._device_declared = True
    return lib


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class SpmeSolver:
    """One SPME reciprocal-space solver bound to a CUDA device and stream."""

    def __init__(self, L, K, order, beta, max_m, device=None, stream=None):
        import torch

        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        with torch.cuda.device(self.device):
            self.sf = _ew.Sfac(np.asarray(L, dtype=np.float64), np.asarray(K), int(order))
            self.sf.set_ewald(float(beta), float(max_m))
            self.lib = _lib()
            self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
            rc = self.lib.sfac_set_stream(self.sf._data, ctypes.c_void_p(self.stream.cuda_stream))
            if rc != 0:
                raise RuntimeError("sfac_set_stream failed")
        self.K = tuple(int(k) for k in K)
        self.order = int(order)

    @property
    def handle(self):
        return self.sf._data

    def launches(self) -> int:
        return self.sf.launches()

    def _check(self, x, q, dx, phi, ev):
        t = self.torch
        n = q.shape[0]
        assert x.dtype == t.float64 and q.dtype == t.float64 and x.is_cuda and q.is_cuda
        assert x.shape == (n, 3) and x.is_contiguous() and q.is_contiguous()
        for a, shape in ((dx, (n, 3)), (phi, (n,)), (ev, (7,))):
            if a is not None:
                assert a.dtype == t.float64 and a.shape == shape and a.is_contiguous()
        return n

    def solve(self, x, q, dx=None, phi=None, ev=None):
        """Enqueues one solve; returns ev (E, 6 virial components) on device."""
        t = self.torch
        n = q.shape[0]
        if ev is None:
            ev = t.empty(7, dtype=t.float64, device=self.device)
        self._check(x, q, dx, phi, ev)
        rc = self.lib.sfac_solve_device(self.handle, n, _ptr(x), _ptr(q), _ptr(dx), _ptr(phi), _ptr(ev))
        if rc != 0:
            raise RuntimeError(f"sfac_solve_device failed ({rc}): {self.sf.last_error()}")
        return ev

    def solve_timed(self, x, q, dx=None, phi=None, ev=None):
        """Solve with per-stage CUDA-event times (ms), synchronising."""
        t = self.torch
        n = q.shape[0]
        if ev is None:
            ev = t.empty(7, dtype=t.float64, device=self.device)
        self._check(x, q, dx, phi, ev)
        ms = (c_float * 6)()
        rc = self.lib.sfac_solve_device_timed(self.handle, n, _ptr(x), _ptr(q), _ptr(dx), _ptr(phi), _ptr(ev), ms)
        if rc != 0:
            raise RuntimeError(f"sfac_solve_device_timed failed ({rc}): {self.sf.last_error()}")
        return dict(zip(STAGES, [float(v) for v in ms]))

    def real_space(self, x, q, eta, rcut, out=None, dx=None):
        """Enqueues the real-space Ewald term (sfac_real_space_device): out
        (10 doubles on device) = [E_real, E_self, E_net, virial[6], net-charge
        virial diagonal]; dx (n x 3, may be None) = dE_real/dx."""
        t = self.torch
        n = q.shape[0]
        if out is None:
            out = t.empty(10, dtype=t.float64, device=self.device)
        self._check(x, q, dx, None, None)
        rc = self.lib.sfac_real_space_device(self.handle, n, _ptr(x), _ptr(q), float(eta), float(rcut), _ptr(out),
                                             _ptr(dx))
        if rc != 0:
            raise RuntimeError(f"sfac_real_space_device failed ({rc}): {self.sf.last_error()}")
        return out
