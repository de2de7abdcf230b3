"""Reverse-mode derivatives of a rollout (ss_adjoint_* of libsmokesim.so).

`Rollout` drives the C ABI: forward pass with checkpoints, reverse pass from
the adjoint of the final state, derivatives of the initial state and of the
per-step emitter forces.  `rollout_fn` wraps it in a torch.autograd.Function
(a thin test binding: the arithmetic is in the library's CUDA kernels).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .sim import Sim, _check


class Rollout:
    """nsteps steps of `sim` from its current state, checkpointed every
    `checkpoint_every` steps.  deterministic=True makes the reverse pass's
    scatter-adds owner-computes (bitwise-repeatable gradients) instead of
    atomic."""

    def __init__(self, sim: Sim, nsteps: int, checkpoint_every: int = 0, deterministic: bool = False,
                 store_pressure: bool = False):
        self.sim = sim
        self.L = sim.L
        self.nsteps = nsteps
        h = C.c_void_p()
        _check(self.L.ss_adjoint_create(sim.h, nsteps, checkpoint_every, C.byref(h)), "ss_adjoint_create")
        self.h = h
        if deterministic:
            self.set_deterministic(True)
        if store_pressure:
            self.set_pressure_store(True)

    def set_deterministic(self, on: bool = True):
        _check(self.L.ss_adjoint_set_deterministic(self.h, int(bool(on))), "ss_adjoint_set_deterministic")

    def set_pressure_store(self, on: bool = True):
        """Keep every step's solved pressure in the forward pass, so the reverse
        pass recomputes segments without solving again (same gradients)."""
        _check(self.L.ss_adjoint_set_pressure_store(self.h, int(bool(on))), "ss_adjoint_set_pressure_store")

    def close(self):
        if getattr(self, "h", None):
            self.L.ss_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, params, forces=None, stream=None):
        fp = None
        if forces is not None:
            f = np.ascontiguousarray(forces, dtype=np.float32).reshape(self.nsteps * 3)
            self._forces = f
            fp = f.ctypes.data_as(C.POINTER(C.c_float))
        _check(self.L.ss_adjoint_forward(self.h, C.byref(params), fp, C.c_void_p(stream)), "ss_adjoint_forward")

    def backward(self, params, grad_density=None, grad_temperature=None, grad_velocity=None, stream=None):
        """Gradients of the final state as device pointers (ints) or None.
        Returns dL/d(force) per step, (nsteps, 3) float32."""
        gv = (C.c_void_p * 3)()
        if grad_velocity is not None:
            for d, ptr in enumerate(grad_velocity):
                gv[d] = ptr
        gf = np.zeros(self.nsteps * 3, np.float32)
        _check(self.L.ss_adjoint_backward(self.h, C.byref(params), C.c_void_p(grad_density),
                                          C.c_void_p(grad_temperature), C.byref(gv),
                                          gf.ctypes.data_as(C.POINTER(C.c_float)), C.c_void_p(stream)),
               "ss_adjoint_backward")
        return gf.reshape(self.nsteps, 3)

    def grad(self, field):
        """dL/d(initial field) on the host (after backward)."""
        n = abi.field_count(self.sim.dim, self.sim.n, field, self.sim.nch)
        out = np.empty(n, np.float32)
        _check(self.L.ss_adjoint_get_field(self.h, field, out.ctypes.data, n, 0, None), "ss_adjoint_get_field")
        return out

    def grad_to_device(self, field, dst_ptr, stream=None):
        n = abi.field_count(self.sim.dim, self.sim.n, field, self.sim.nch)
        _check(self.L.ss_adjoint_get_field(self.h, field, C.c_void_p(dst_ptr), n, 1, C.c_void_p(stream)),
               "ss_adjoint_get_field")

    def force_field_grad(self, n):
        """dL/d(coarse force field) of the last backward pass, shape (3, n, n, n)."""
        out = np.empty((3, n, n, n), np.float32)
        _check(self.L.ss_adjoint_force_field_grad(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size),
               "ss_adjoint_force_field_grad")
        return out

    def info(self):
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(self.L.ss_adjoint_info(self.h, C.byref(a), C.byref(b), C.byref(c)), "ss_adjoint_info")
        return {"kernel_launches": a.value, "checkpoint_bytes": b.value, "workspace_bytes": c.value}


def _vel_fields(dim):
    return [abi.FIELD_VX, abi.FIELD_VY] + ([abi.FIELD_VZ] if dim == 3 else [])


def rollout_fn(rollout: Rollout, params):
    """torch.autograd.Function mapping (initial velocities..., forces) to the
    final density of the rollout; gradients come from the library's adjoint."""
    import torch

    sim = rollout.sim
    dim = sim.dim

    class RolloutFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, forces, *vel):
            stream = torch.cuda.current_stream().cuda_stream
            for f, t in zip(_vel_fields(dim), vel):
                t = t.detach().contiguous()
                _check(sim.L.ss_set_field_device(sim.h, f, C.c_void_p(t.data_ptr()), t.numel(), C.c_void_p(stream)),
                       "ss_set_field_device")
            rollout.forward(params, forces.detach().cpu().numpy(), stream=stream)
            n = abi.field_count(dim, sim.n, abi.FIELD_DENSITY, sim.nch)
            out = torch.empty(n, dtype=torch.float32, device=vel[0].device)
            _check(sim.L.ss_get_field_device(sim.h, abi.FIELD_DENSITY, C.c_void_p(out.data_ptr()), n, C.c_void_p(stream)),
                   "ss_get_field_device")
            return out

        @staticmethod
        def backward(ctx, grad_out):
            stream = torch.cuda.current_stream().cuda_stream
            g = grad_out.detach().contiguous().float()
            gf = rollout.backward(params, grad_density=g.data_ptr(), stream=stream)
            grads = []
            for f in _vel_fields(dim):
                n = abi.field_count(dim, sim.n, f, sim.nch)
                t = torch.empty(n, dtype=torch.float32, device=g.device)
                rollout.grad_to_device(f, t.data_ptr(), stream=stream)
                grads.append(t)
            return (torch.from_numpy(gf).to(g.device), *grads)

    return RolloutFn.apply
