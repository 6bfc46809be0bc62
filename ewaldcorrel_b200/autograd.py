"""Differentiable SPME reciprocal energy for PyTorch.

``spme_energy(x, q, L)`` returns the reciprocal-space Ewald energy of one
periodic system (the reference's ``de1`` energy, sfac.cpp:339-396) as a 0-d
FP64 tensor whose backward gives dE/dx (the ``de2`` gradient,
sfac.cpp:409-483), dE/dq (the ``potl`` potential, sfac.cpp:497-545) and
dE/dL at fixed Cartesian positions, L = [ax, by, cz, bx, cx, cy].  All of
them come out of one device solve (the gather kernel's adjoint); backward
only scales them by the incoming gradient.

``SpmeBatch`` evaluates many independent systems (different sizes, boxes and
grids) in one call: every system keeps a plan with fixed device buffers, so
its solve replays as a CUDA graph, and the solves run concurrently on the
plans' own streams.
"""
from __future__ import annotations

from ctypes import c_int, c_void_p

import numpy as np
import torch

from . import ewald as _ew
from .configs import MAX_M_FACTOR


def _lib():
    _, _, lib = _ew.describe_sfac()
    if not getattr(lib, "_autograd_declared", False):
        lib.sfac_solve_device_cell.argtypes = [c_void_p, c_int] + [c_void_p] * 6
        lib.sfac_solve_device_cell.restype = c_int
        lib.sfac_get_stream.argtypes = [c_void_p]
        lib.sfac_get_stream.restype = c_void_p
        lib._autograd_declared = True
    return lib


class SpmePlan:
    """One system shape (atom count, grid, order) with fixed device buffers.

    The box may change between calls (the influence function is re-set on
    the device); inputs are copied into the plan's buffers so that the
    solve's CUDA graph keeps valid pointers."""

    def __init__(self, n, K, order=4, beta=3.47, max_m=None, L=None, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.n, self.K, self.order = int(n), tuple(int(k) for k in K), int(order)
        self.beta = float(beta)
        self.max_m = float(MAX_M_FACTOR * beta if max_m is None else max_m)
        L = np.asarray([1.0, 1.0, 1.0, 0.0, 0.0, 0.0] if L is None else L, dtype=np.float64)
        with torch.cuda.device(self.device):
            self.sf = _ew.Sfac(L.copy(), np.asarray(self.K), self.order)
            self.sf.set_ewald(self.beta, self.max_m)
            self.L = L.copy()
            self.lib = _lib()
            self.stream = torch.cuda.ExternalStream(self.lib.sfac_get_stream(self.sf._data), device=self.device)
            dev = self.device
            self.x = torch.zeros((max(self.n, 1), 3), dtype=torch.float64, device=dev)
            self.q = torch.zeros(max(self.n, 1), dtype=torch.float64, device=dev)
            self.dx = torch.zeros((max(self.n, 1), 3), dtype=torch.float64, device=dev)
            self.phi = torch.zeros(max(self.n, 1), dtype=torch.float64, device=dev)
            self.ev = torch.zeros(7, dtype=torch.float64, device=dev)
            self.dEdL = torch.zeros(6, dtype=torch.float64, device=dev)
        self.done = torch.cuda.Event()

    def set_box(self, L):
        L = np.asarray(L, dtype=np.float64).reshape(6)
        if not np.array_equal(L, self.L):
            self.sf._libsfac.set_L(self.sf._data, L.copy())
            self.sf.set_ewald(self.beta, self.max_m)  # influence function of the new box
            self.L = L.copy()

    def launch(self, x, q, ready):
        """Copies the inputs in and enqueues the solve on the plan's stream
        after `ready` (an event on the caller's stream)."""
        self.stream.wait_event(ready)
        with torch.cuda.stream(self.stream):
            self.x[: self.n].copy_(x)
            self.q[: self.n].copy_(q)
            rc = self.lib.sfac_solve_device_cell(self.sf._data, self.n, self.x.data_ptr(), self.q.data_ptr(),
                                                 self.dx.data_ptr(), self.phi.data_ptr(), self.ev.data_ptr(),
                                                 self.dEdL.data_ptr())
            if rc != 0:
                raise RuntimeError(f"sfac_solve_device_cell failed ({rc}): {self.sf.last_error()}")
            self.done.record(self.stream)


def _box_numpy(L):
    if torch.is_tensor(L):
        return L.detach().to("cpu", torch.float64).numpy().reshape(-1)
    return np.asarray(L, np.float64).reshape(-1)


class _SpmeBatchFn(torch.autograd.Function):
    """Energies of a batch of systems; the gradients are computed in the
    forward solve and scaled by the incoming gradient in backward."""

    @staticmethod
    def forward(ctx, x, q, L, batch):
        offs = batch.offsets
        cur = torch.cuda.current_stream(batch.device)
        xd, qd = x.detach().to(batch.device, torch.float64), q.detach().to(batch.device, torch.float64)
        ready = torch.cuda.Event()
        ready.record(cur)
        boxes = _box_numpy(L).reshape(-1, 6)
        for i, p in enumerate(batch.plans):
            p.set_box(boxes[i])
            p.launch(xd[offs[i]:offs[i + 1]], qd[offs[i]:offs[i + 1]], ready)
        B = len(batch.plans)
        E = torch.empty(B, dtype=torch.float64, device=batch.device)
        dx = torch.empty_like(xd)
        phi = torch.empty_like(qd)
        dL = torch.empty((B, 6), dtype=torch.float64, device=batch.device)
        for i, p in enumerate(batch.plans):
            cur.wait_event(p.done)
            E[i : i + 1].copy_(p.ev[:1])
            dx[offs[i]:offs[i + 1]].copy_(p.dx[: p.n])
            phi[offs[i]:offs[i + 1]].copy_(p.phi[: p.n])
            dL[i].copy_(p.dEdL)
        ctx.save_for_backward(dx, phi, dL)
        ctx.sysid = batch.sysid
        ctx.L_meta = (L.shape, L.device, L.dtype)
        ctx.x_meta = (x.device, x.dtype)
        ctx.q_meta = (q.device, q.dtype)
        return E

    @staticmethod
    def backward(ctx, gE):
        dx, phi, dL = ctx.saved_tensors
        g_atom = gE[ctx.sysid]
        shape, ldev, ldt = ctx.L_meta
        gx = (g_atom[:, None] * dx).to(*ctx.x_meta)
        gq = (g_atom * phi).to(*ctx.q_meta)
        gL = (gE[:, None] * dL).reshape(shape).to(ldev, ldt)
        return gx, gq, gL, None


class SpmeBatch:
    """Independent periodic systems evaluated together.

    systems: list of (n_atoms, K, order[, beta[, max_m]]) tuples;
    calling it with the concatenated positions (sum n, 3), charges (sum n)
    and boxes (B, 6) returns the B energies; autograd gives dE/dx, dE/dq
    and dE/dL of every system."""

    def __init__(self, systems, beta=3.47, max_m=None, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.plans = []
        counts = []
        for s in systems:
            n, K, order = s[0], s[1], s[2]
            b = s[3] if len(s) > 3 else beta
            mm = s[4] if len(s) > 4 else max_m
            self.plans.append(SpmePlan(n, K, order, b, mm, device=self.device.index))
            counts.append(int(n))
        self.offsets = [int(v) for v in np.concatenate([[0], np.cumsum(counts)])]
        self.sysid = torch.repeat_interleave(torch.arange(len(counts), device=self.device),
                                             torch.tensor(counts, device=self.device))

    def __call__(self, x, q, L):
        return _SpmeBatchFn.apply(x, q, L, self)


_PLANS: dict = {}


def spme_energy(x, q, L, K, order=4, beta=3.47, max_m=None):
    """Reciprocal SPME energy of one system (0-d FP64 tensor), differentiable
    in x (N, 3), q (N) and L (6)."""
    n = int(q.shape[0])
    dev = x.device
    key = (dev.index, n, tuple(int(k) for k in K), int(order), float(beta), max_m)
    batch = _PLANS.get(key)
    if batch is None:
        batch = SpmeBatch([(n, K, order, beta, max_m)], device=dev.index)
        _PLANS[key] = batch
    L2 = L.reshape(1, 6) if torch.is_tensor(L) else torch.as_tensor(np.asarray(L, np.float64).reshape(1, 6))
    return batch(x, q, L2)[0]
