"""Gray-level lattice and its discrete adjoint over the C ABI (no counterpart
in the reference, which has no adjoint).

`GrayLattice` is a D3Q19 BGK lattice whose design-box cells carry a solid
fraction gamma in [0, 1] (Brinkman drag: a cell removes alpha * gamma of its
momentum each step); `backward()` returns an objective (the mean force or
moment on the gray body over a window of steps) and its gradient with respect
to every design cell's gamma, from the hand-written adjoint of
include/simlab_lbm.h (lbm_backward).  `GrayObjective` wraps the pair in a
torch.autograd.Function; it exists for the gradient-check harness only.
Every call goes to libsimlab_lbm.so; there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from .lbm import LbmError, Storage, _global_error, _v3, library


class _GraySetup(C.Structure):
    _fields_ = [
        ("dims", C.c_uint32 * 3),
        ("box_lo", C.c_uint32 * 3),
        ("box_n", C.c_uint32 * 3),
        ("storage", C.c_int32),
        ("nu", C.c_double),
        ("u_in", C.c_double * 3),
        ("alpha", C.c_double),
        ("center", C.c_double * 3),
    ]


class _AdjointSpec(C.Structure):
    _fields_ = [
        ("steps", C.c_uint64),
        ("t0", C.c_uint64),
        ("t1", C.c_uint64),
        ("checkpoint_every", C.c_uint32),
        ("objective", C.c_int32),
        ("dir", C.c_double * 3),
        ("recompute", C.c_int32),
        ("_pad", C.c_int32),
    ]


@dataclass
class GraySetup:
    dims: Sequence[int]
    box_lo: Sequence[int]
    box_n: Sequence[int]
    nu: float
    u_in: Sequence[float] = (0.04, 0.0, 0.0)
    alpha: float = 1.0
    center: Sequence[float] = (0.0, 0.0, 0.0)
    storage: Storage = Storage.FP32

    def nbox(self) -> int:
        return int(np.prod([int(v) for v in self.box_n]))

    def cells(self) -> int:
        return int(np.prod([int(v) for v in self.dims]))

    def to_c(self) -> _GraySetup:
        s = _GraySetup()
        s.dims[:] = [int(v) for v in self.dims]
        s.box_lo[:] = [int(v) for v in self.box_lo]
        s.box_n[:] = [int(v) for v in self.box_n]
        s.storage = int(self.storage)
        s.nu = float(self.nu)
        s.u_in[:] = _v3(self.u_in)
        s.alpha = float(self.alpha)
        s.center[:] = _v3(self.center)
        return s


@dataclass
class AdjointSpec:
    """The objective J = mean over steps t0..t1 (1-based, inclusive) of
    dir . F_t (objective 0) or dir . M_t (objective 1)."""

    steps: int
    t0: int
    t1: int
    checkpoint_every: int = 50
    objective: int = 0
    dir: Sequence[float] = (1.0, 0.0, 0.0)
    recompute: bool = True

    def to_c(self) -> _AdjointSpec:
        s = _AdjointSpec()
        s.steps, s.t0, s.t1 = int(self.steps), int(self.t0), int(self.t1)
        s.checkpoint_every = int(self.checkpoint_every)
        s.objective = int(self.objective)
        s.dir[:] = _v3(self.dir)
        s.recompute = int(bool(self.recompute))
        return s

    def value(self, forces: np.ndarray) -> float:
        """The objective from per-step forces (6 per step) of a forward run."""
        f = np.asarray(forces)[int(self.t0) - 1:int(self.t1)]
        col = f[:, 3:6] if self.objective == 1 else f[:, 0:3]
        return float((col @ np.asarray(self.dir, dtype=np.float64)).mean())


_bound = False


def _lib() -> C.CDLL:
    global _bound
    L = library()
    if not _bound:
        vp, u64, dp = C.c_void_p, C.c_uint64, C.POINTER(C.c_double)
        L.lbm_gray_create.argtypes = [C.POINTER(_GraySetup), C.POINTER(vp)]
        L.lbm_gray_destroy.argtypes = [vp]
        L.lbm_gray_destroy.restype = None
        L.lbm_gray_last_error.argtypes = [vp, C.c_char_p, u64]
        L.lbm_gray_set_field.argtypes = [vp, dp]
        L.lbm_gray_reset.argtypes = [vp]
        L.lbm_gray_run.argtypes = [vp, u64, dp]
        L.lbm_backward.argtypes = [vp, C.POINTER(_AdjointSpec), dp, dp]
        L.lbm_gray_backward_times.argtypes = [vp, dp, dp, dp]
        L.lbm_gray_stream.argtypes = [vp, C.POINTER(vp)]
        _bound = True
    return L


class GrayLattice:
    def __init__(self, setup: GraySetup, gamma: np.ndarray | None = None):
        L = _lib()
        self._L = L
        self.setup = setup
        cs = setup.to_c()
        h = C.c_void_p()
        rc = L.lbm_gray_create(C.byref(cs), C.byref(h))
        if rc != 0:
            raise _global_error(rc)
        self._h = h
        if gamma is not None:
            self.set_field(gamma)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.lbm_gray_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != 0:
            buf = C.create_string_buffer(1024)
            self._L.lbm_gray_last_error(self._h, buf, 1024)
            raise LbmError(rc, buf.value.decode(errors="replace"))

    def set_field(self, gamma) -> None:
        g = np.ascontiguousarray(np.asarray(gamma, dtype=np.float64).reshape(-1))
        if g.size != self.setup.nbox():
            raise ValueError(f"gamma needs {self.setup.nbox()} values (the design box)")
        self._check(self._L.lbm_gray_set_field(self._h, g.ctypes.data_as(C.POINTER(C.c_double))))

    def reset(self) -> None:
        self._check(self._L.lbm_gray_reset(self._h))

    def run(self, n: int) -> np.ndarray:
        out = np.zeros((int(n), 6), dtype=np.float64)
        self._check(self._L.lbm_gray_run(self._h, int(n), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def objective(self, spec: AdjointSpec) -> float:
        """J from a forward run from the initial state (no adjoint)."""
        self.reset()
        return spec.value(self.run(spec.steps))

    def backward(self, spec: AdjointSpec) -> tuple[float, np.ndarray]:
        """(J, dJ/dgamma) with dJ/dgamma in design-box order (x fastest)."""
        J = C.c_double()
        grad = np.zeros(self.setup.nbox(), dtype=np.float64)
        cs = spec.to_c()
        self._check(self._L.lbm_backward(self._h, C.byref(cs), C.byref(J), grad.ctypes.data_as(C.POINTER(C.c_double))))
        return J.value, grad

    def backward_times(self) -> dict:
        f, r, b = C.c_double(), C.c_double(), C.c_double()
        self._check(self._L.lbm_gray_backward_times(self._h, C.byref(f), C.byref(r), C.byref(b)))
        return {"forward_ms": f.value, "recompute_ms": r.value, "reverse_ms": b.value}

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self._L.lbm_gray_stream(self._h, C.byref(s)))
        return int(s.value or 0)


def gray_objective_function():
    """A torch.autograd.Function over (GrayLattice, AdjointSpec, gamma) -> J,
    whose backward is lbm_backward; for the gradient-check harness only."""
    import torch

    class GrayObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, gamma, lat, spec):
            lat.set_field(gamma.detach().cpu().double().numpy())
            J, grad = lat.backward(spec)
            ctx.save_for_backward(torch.from_numpy(grad).to(gamma.dtype))
            return gamma.new_tensor(J)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad, None, None

    return GrayObjective
