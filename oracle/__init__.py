"""TEST INFRASTRUCTURE -- the CPU oracle of the D3Q19 time step.

A C++ restatement of SimLab's WGSL update (crates/cfd/src/shader.rs) and its
driver (crates/cfd/src/lattice.rs), see d3q19_oracle.hpp.  Imported only by
the tests, the smoke check and the bench's CPU baseline; never by the engine.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .build import LIB, build_oracle

_lib = None


def library() -> C.CDLL:
    global _lib
    if _lib is None:
        build_oracle()
        L = C.CDLL(str(LIB))
        vp, u64 = C.c_void_p, C.c_ulonglong
        L.orc_create.argtypes = [vp, vp, C.c_int]
        L.orc_create.restype = vp
        L.orc_destroy.argtypes = [vp]
        L.orc_destroy.restype = None
        L.orc_run.argtypes = [vp, vp, u64, vp]
        L.orc_macros.argtypes = [vp, vp]
        L.orc_step_slab.argtypes = [vp, C.c_uint, C.c_uint]
        L.orc_nrec.argtypes = [vp]
        L.orc_nrec.restype = u64
        L.orc_nface.argtypes = [vp]
        L.orc_nface.restype = u64
        L.orc_records.argtypes = [vp, vp]
        L.orc_flags.argtypes = [vp, vp]
        L.orc_faces.argtypes = [vp, vp]
        L.orc_raw.argtypes = [vp, vp]
        L.orc_steps_done.argtypes = [vp]
        L.orc_steps_done.restype = u64
        L.orc_last_error.argtypes = [C.c_char_p, u64]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_f32_to_f16.argtypes = [C.c_float]
        L.orc_f32_to_f16.restype = C.c_uint16
        L.orc_f16_to_f32.argtypes = [C.c_uint16]
        L.orc_f16_to_f32.restype = C.c_float
        L.orc_f16_bits_ref.argtypes = [C.c_float]
        L.orc_f16_bits_ref.restype = C.c_uint16
        L.orc_f32_to_bf16.argtypes = [C.c_float]
        L.orc_f32_to_bf16.restype = C.c_uint16
        L.orc_sround16.argtypes = [C.c_float, C.c_uint32, C.c_uint32]
        L.orc_sround16.restype = C.c_float
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return library().orc_set_threads(int(n))


class OracleLattice:
    """The oracle with the same constructor and readback as simlab_b200.Lattice.

    real64=False: the reference's FP32 update; real64=True: the FP64 oracle
    (use Storage.FP64 in the setup for FP64 storage)."""

    def __init__(self, setup, geometry=None, real64: bool = False, _frozen=None):
        L = library()
        self._L = L
        self.setup = setup
        cs = setup.to_c()
        if _frozen is not None:  # a fixture's geometry (oracle.abi), no engine import
            g, keep = _frozen
        else:
            from simlab_b200.lbm import geometry_struct  # the C-ABI structs are shared

            g, keep = geometry_struct(geometry)
        h = L.orc_create(C.addressof(cs), C.addressof(g), int(real64))
        del keep
        if not h:
            buf = C.create_string_buffer(1024)
            L.orc_last_error(buf, 1024)
            raise RuntimeError(buf.value.decode())
        self._h = h

    @classmethod
    def from_fixture(cls, path, real64: bool = False) -> "OracleLattice":
        """The oracle on a frozen case (oracle/fixtures, written by
        oracle/make_arm_fixture.py): setup and geometry come from the file,
        nothing of the engine is imported or loaded."""
        from .abi import load_case

        setup, g, keep = load_case(Path(path))
        return cls(setup, real64=real64, _frozen=(g, keep))

    def close(self):
        if getattr(self, "_h", None):
            self._L.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def steps_done(self) -> int:
        return int(self._L.orc_steps_done(self._h))

    @property
    def nrec(self) -> int:
        return int(self._L.orc_nrec(self._h))

    @property
    def nface(self) -> int:
        return int(self._L.orc_nface(self._h))

    def run(self, steps) -> np.ndarray:
        from simlab_b200.lbm import STEP_DTYPE, steps_array

        a = steps if isinstance(steps, np.ndarray) and steps.dtype == STEP_DTYPE else steps_array(steps)
        a = np.ascontiguousarray(a)
        out = np.zeros((len(a), 6), dtype=np.float64)
        self._L.orc_run(self._h, a.ctypes.data, len(a), out.ctypes.data)
        return out

    def step_slab(self, z0: int, z1: int) -> None:
        """CPU-baseline timing: one step's collide-stream over z-planes [z0, z1)."""
        self._L.orc_step_slab(self._h, int(z0), int(z1))

    def macros(self) -> np.ndarray:
        out = np.empty((self.setup.cells(), 4), dtype=np.float64)
        self._L.orc_macros(self._h, out.ctypes.data)
        return out

    def records(self) -> np.ndarray:
        out = np.zeros(max(self.nrec, 1) * 40, dtype=np.uint32)
        self._L.orc_records(self._h, out.ctypes.data)
        return out

    def flags(self) -> np.ndarray:
        out = np.zeros(self.setup.cells(), dtype=np.uint32)
        self._L.orc_flags(self._h, out.ctypes.data)
        return out

    def faces(self) -> np.ndarray:
        out = np.zeros(self.nface, dtype=np.uint32)
        self._L.orc_faces(self._h, out.ctypes.data)
        return out

    def raw(self) -> np.ndarray:
        out = np.zeros(19 * self.setup.cells(), dtype=np.float64)
        self._L.orc_raw(self._h, out.ctypes.data)
        return out.reshape(19, -1)


class OracleMulti:
    """The multi-level D3Q27 oracle with the readback of simlab_b200.MultiLattice.

    real64=False: the reference's FP32 update; real64=True: the FP64 oracle."""

    def __init__(self, setup, geometry=None, real64: bool = False, probes=None):
        from simlab_b200.lbm import geometry_struct, probes_struct

        L = library()
        vp, u64 = C.c_void_p, C.c_ulonglong
        L.m27_create_probes.argtypes = [vp, vp, vp, C.c_int]
        L.m27_create_probes.restype = vp
        L.m27_reset_samples.argtypes = [vp]
        L.m27_vertex_means.argtypes = [vp, vp]
        L.m27_slice_means.argtypes = [vp, vp]
        L.m27_nvert.argtypes = [vp]
        L.m27_nvert.restype = C.c_uint
        L.m27_npix.argtypes = [vp]
        L.m27_npix.restype = C.c_uint
        L.m27_destroy.argtypes = [vp]
        L.m27_destroy.restype = None
        L.m27_run.argtypes = [vp, vp, u64, vp]
        L.m27_levels.argtypes = [vp]
        L.m27_levels.restype = C.c_uint
        L.m27_dims.argtypes = [vp, vp]
        L.m27_macros.argtypes = [vp, C.c_uint, vp]
        L.m27_nrec.argtypes = [vp]
        L.m27_nrec.restype = u64
        L.m27_records.argtypes = [vp, vp]
        L.m27_flags.argtypes = [vp, C.c_uint, vp]
        L.m27_fine_steps.argtypes = [vp]
        L.m27_fine_steps.restype = u64
        self._L = L
        self.setup = setup
        cs, keep = setup.to_c()
        g, keep2 = geometry_struct(geometry)
        pr, keep3 = probes_struct(probes)
        h = L.m27_create_probes(C.addressof(cs), C.addressof(g), C.addressof(pr) if pr is not None else None, int(real64))
        del keep, keep2, keep3
        if not h:
            buf = C.create_string_buffer(1024)
            L.orc_last_error(buf, 1024)
            raise RuntimeError(buf.value.decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.m27_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def levels(self) -> int:
        return int(self._L.m27_levels(self._h))

    def level_dims(self) -> list:
        n = self.levels()
        out = np.zeros(3 * n, dtype=np.uint32)
        self._L.m27_dims(self._h, out.ctypes.data)
        return [tuple(int(v) for v in out[3 * l:3 * l + 3]) for l in range(n)]

    def sub_steps(self) -> int:
        return 1 << (self.levels() - 1)

    @property
    def nrec(self) -> int:
        return int(self._L.m27_nrec(self._h))

    @property
    def fine_steps(self) -> int:
        return int(self._L.m27_fine_steps(self._h))

    def run(self, fine) -> np.ndarray:
        from simlab_b200.lbm import STEP_DTYPE, steps_array

        a = fine if isinstance(fine, np.ndarray) and fine.dtype == STEP_DTYPE else steps_array(fine)
        a = np.ascontiguousarray(a)
        out = np.zeros((len(a), 6), dtype=np.float64)
        if self._L.m27_run(self._h, a.ctypes.data, len(a), out.ctypes.data) != 0:
            buf = C.create_string_buffer(1024)
            self._L.orc_last_error(buf, 1024)
            raise RuntimeError(buf.value.decode())
        return out

    def macros(self, level: int) -> np.ndarray:
        d = self.level_dims()[level]
        out = np.empty((d[0] * d[1] * d[2], 4), dtype=np.float32)
        self._L.m27_macros(self._h, int(level), out.ctypes.data)
        return out

    def records(self) -> np.ndarray:
        out = np.zeros(max(self.nrec, 1) * 24, dtype=np.uint32)
        self._L.m27_records(self._h, out.ctypes.data)
        return out

    def flags(self, level: int) -> np.ndarray:
        d = self.level_dims()[level]
        out = np.zeros(d[0] * d[1] * d[2], dtype=np.uint32)
        self._L.m27_flags(self._h, int(level), out.ctypes.data)
        return out

    def reset_samples(self) -> None:
        self._L.m27_reset_samples(self._h)

    def vertex_means(self) -> np.ndarray:
        n = int(self._L.m27_nvert(self._h))
        out = np.empty(max(n, 1), dtype=np.float32)
        self._L.m27_vertex_means(self._h, out.ctypes.data)
        return out[:n]

    def slice_means(self) -> np.ndarray:
        n = int(self._L.m27_npix(self._h))
        out = np.empty((max(n, 1), 4), dtype=np.float32)
        self._L.m27_slice_means(self._h, out.ctypes.data)
        return out[:n]


class OracleGray:
    """The gray-level oracle (forward model and dense-Jacobian adjoint) with
    the methods of simlab_b200.gray.GrayLattice."""

    def __init__(self, setup, gamma=None, real64: bool = True):
        L = library()
        vp, u64 = C.c_void_p, C.c_ulonglong
        L.gray_create.argtypes = [vp, C.c_int]
        L.gray_create.restype = vp
        L.gray_destroy.argtypes = [vp]
        L.gray_destroy.restype = None
        L.gray_set_field.argtypes = [vp, vp]
        L.gray_reset.argtypes = [vp]
        L.gray_run.argtypes = [vp, u64, vp]
        L.gray_backward.argtypes = [vp, vp, vp, vp]
        self._L = L
        self.setup = setup
        cs = setup.to_c()
        h = L.gray_create(C.addressof(cs), int(real64))
        if not h:
            buf = C.create_string_buffer(1024)
            L.orc_last_error(buf, 1024)
            raise RuntimeError(buf.value.decode())
        self._h = h
        if gamma is not None:
            self.set_field(gamma)

    def close(self):
        if getattr(self, "_h", None):
            self._L.gray_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_field(self, gamma):
        g = np.ascontiguousarray(np.asarray(gamma, dtype=np.float64).reshape(-1))
        assert g.size == self.setup.nbox()
        self._L.gray_set_field(self._h, g.ctypes.data)

    def reset(self):
        self._L.gray_reset(self._h)

    def run(self, n: int) -> np.ndarray:
        out = np.zeros((int(n), 6), dtype=np.float64)
        self._L.gray_run(self._h, int(n), out.ctypes.data)
        return out

    def objective(self, spec) -> float:
        self.reset()
        return spec.value(self.run(spec.steps))

    def backward(self, spec):
        J = C.c_double()
        grad = np.zeros(self.setup.nbox(), dtype=np.float64)
        cs = spec.to_c()
        self._L.gray_backward(self._h, C.addressof(cs), C.byref(J), grad.ctypes.data)
        return J.value, grad
