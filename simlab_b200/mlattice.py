"""Python mirror of the reference's multi-level D3Q27 lattice over the C ABI.

`MultiLattice`, `MultiSetup` and `LevelBox` follow crates/cfd/src/mlattice.rs:
same names, argument meaning and units (finest-level lattice units for forces
and the moment centre), errors raised where the reference bails.  Every call
goes to libsimlab_lbm.so (lbm_create_multi and the lbm_multi_* functions of
include/simlab_lbm.h); there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from .lbm import (STEP_DTYPE, FaceBc, LbmError, Probes, StaticVoxels, StepIn, Storage, _global_error, _Info, _v3, geometry_struct, library, probes_struct,
                  steps_array)

RS27 = 24  # u32 words per D3Q27 wall record (mshader.rs:32-36)


@dataclass
class LevelBox:
    """`LevelBox` (mlattice.rs:15-21): parent node of node 0, parent nodes spanned."""

    lo: Sequence[int]
    n: Sequence[int]


class _LevelBox(C.Structure):
    _fields_ = [("lo", C.c_int32 * 3), ("n", C.c_uint32 * 3)]


class _MultiSetup(C.Structure):
    _fields_ = [
        ("dims0", C.c_uint32 * 3),
        ("nboxes", C.c_uint32),
        ("boxes", C.POINTER(_LevelBox)),
        ("faces", C.c_int32 * 6),
        ("nu0", C.c_double),
        ("smagorinsky", C.c_double),
        ("u_inf", C.c_double * 3),
        ("u_init", C.c_double * 3),
        ("body_force0", C.c_double * 3),
        ("sponge", C.c_uint32 * 6),
        ("sponge_tau", C.c_double),
        ("sponge_sigma", C.c_double),
        ("absorb_velocity", C.c_int32),
        ("total_pressure_inlet", C.c_int32),
        ("storage", C.c_int32),
        ("debug_dump", C.c_int32),
        ("center", C.c_double * 3),
    ]


@dataclass
class MultiSetup:
    """`MultiSetup` (mlattice.rs:23-47)."""

    dims0: Sequence[int]
    boxes: list = field(default_factory=list)
    faces: Sequence[FaceBc] = (FaceBc.PERIODIC,) * 6
    nu0: float = 0.1
    smagorinsky: float = 0.0
    u_inf: Sequence[float] = (0.0, 0.0, 0.0)
    u_init: Sequence[float] = (0.0, 0.0, 0.0)
    body_force0: Sequence[float] = (0.0, 0.0, 0.0)
    sponge: Sequence[int] = (0, 0, 0, 0, 0, 0)
    sponge_tau: float = 1.0
    sponge_sigma: float = 0.0
    absorb_velocity: bool = False
    total_pressure_inlet: bool = False
    storage: Storage = Storage.FP32
    center: Sequence[float] = (0.0, 0.0, 0.0)
    debug_dump: bool = False

    def levels(self) -> int:
        return len(self.boxes) + 1

    def dims(self, level: int) -> tuple:
        """mlattice.rs:52-60: dims = 2 (n - 1) + 1 for refined levels."""
        if level == 0:
            return tuple(int(d) for d in self.dims0)
        b = self.boxes[level - 1]
        return tuple(2 * (int(v) - 1) + 1 for v in b.n)

    def cells(self) -> list:
        return [int(np.prod(self.dims(l))) for l in range(self.levels())]

    def to_c(self) -> tuple[_MultiSetup, list]:
        s = _MultiSetup()
        s.dims0[:] = [int(d) for d in self.dims0]
        boxes = (_LevelBox * max(len(self.boxes), 1))()
        for k, b in enumerate(self.boxes):
            boxes[k].lo[:] = [int(v) for v in b.lo]
            boxes[k].n[:] = [int(v) for v in b.n]
        s.nboxes = len(self.boxes)
        s.boxes = C.cast(boxes, C.POINTER(_LevelBox))
        if len(self.faces) != 6:
            raise ValueError("faces must list -x,+x,-y,+y,-z,+z")
        s.faces[:] = [int(f) for f in self.faces]
        s.nu0 = float(self.nu0)
        s.smagorinsky = float(self.smagorinsky)
        s.u_inf[:] = _v3(self.u_inf)
        s.u_init[:] = _v3(self.u_init)
        s.body_force0[:] = _v3(self.body_force0)
        s.sponge[:] = [int(v) for v in self.sponge]
        s.sponge_tau = float(self.sponge_tau)
        s.sponge_sigma = float(self.sponge_sigma)
        s.absorb_velocity = int(bool(self.absorb_velocity))
        s.total_pressure_inlet = int(bool(self.total_pressure_inlet))
        s.storage = int(self.storage)
        s.debug_dump = int(bool(self.debug_dump))
        s.center[:] = _v3(self.center)
        return s, [boxes]


_bound = False


def _lib() -> C.CDLL:
    global _bound
    L = library()
    if not _bound:
        vp, u64, u32, dp = C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)
        L.lbm_create_multi.argtypes = [C.POINTER(_MultiSetup), vp, vp, C.POINTER(vp)]
        L.lbm_multi_destroy.argtypes = [vp]
        L.lbm_multi_destroy.restype = None
        L.lbm_multi_last_error.argtypes = [vp, C.c_char_p, u64]
        L.lbm_multi_levels.argtypes = [vp, C.POINTER(u32)]
        L.lbm_multi_sub_steps.argtypes = [vp, C.POINTER(u32)]
        L.lbm_multi_level_dims.argtypes = [vp, C.POINTER(u32)]
        L.lbm_multi_level_cells.argtypes = [vp, C.POINTER(u64)]
        L.lbm_multi_run.argtypes = [vp, vp, u64, dp]
        L.lbm_multi_advance.argtypes = [vp, u64]
        L.lbm_multi_stream.argtypes = [vp, C.POINTER(vp)]
        L.lbm_multi_synchronize.argtypes = [vp]
        L.lbm_multi_set_timeout.argtypes = [vp, C.c_double]
        L.lbm_multi_macros.argtypes = [vp, u32, C.POINTER(C.c_float)]
        L.lbm_multi_records.argtypes = [vp, C.POINTER(u32), u64]
        L.lbm_multi_get_info.argtypes = [vp, C.POINTER(_Info)]
        L.lbm_multi_mass.argtypes = [vp, u32, dp, C.POINTER(u64)]
        L.lbm_multi_reset_samples.argtypes = [vp]
        L.lbm_multi_vertex_means.argtypes = [vp, C.POINTER(C.c_float)]
        L.lbm_multi_slice_means.argtypes = [vp, C.POINTER(C.c_float)]
        _bound = True
    return L


class MultiLattice:
    """`MultiLattice` (mlattice.rs:134-906) on one B200.

    MultiLattice(setup, geometry, probes): geometry is None (`MGeometry::None`)
    or a `StaticVoxels` made with voxelize_static(..., lattice=27) on the finest
    level (`MGeometry::Static`); probes (`MProbes`, mlattice.rs:79-84) a
    `Probes` of surface vertices relative to the centre and slices in
    finest-level cells, or None."""

    def __init__(self, setup: MultiSetup, geometry: StaticVoxels | None = None, probes: Probes | None = None):
        L = _lib()
        self._L = L
        self.setup = setup
        cs, keep = setup.to_c()
        g, keep2 = geometry_struct(geometry)
        pr, keep3 = probes_struct(probes)
        h = C.c_void_p()
        rc = L.lbm_create_multi(C.byref(cs), C.byref(g), C.byref(pr) if pr is not None else None, C.byref(h))
        del keep, keep2, keep3
        if rc != 0:
            raise _global_error(rc)
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.lbm_multi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int) -> None:
        if rc != 0:
            buf = C.create_string_buffer(1024)
            self._L.lbm_multi_last_error(self._h, buf, 1024)
            raise LbmError(rc, buf.value.decode(errors="replace"))

    def info(self) -> _Info:
        i = _Info()
        self._check(self._L.lbm_multi_get_info(self._h, C.byref(i)))
        return i

    @property
    def fine_steps(self) -> int:
        return int(self.info().steps_done)

    @property
    def nrec(self) -> int:
        return int(self.info().nrec)

    @property
    def memory_bytes(self) -> int:
        return int(self.info().memory_bytes)

    def levels(self) -> int:
        v = C.c_uint32()
        self._check(self._L.lbm_multi_levels(self._h, C.byref(v)))
        return int(v.value)

    def sub_steps(self) -> int:
        """Finest steps per coarsest step (mlattice.rs:705-708)."""
        v = C.c_uint32()
        self._check(self._L.lbm_multi_sub_steps(self._h, C.byref(v)))
        return int(v.value)

    def level_dims(self) -> list:
        n = self.levels()
        out = np.zeros(3 * n, dtype=np.uint32)
        self._check(self._L.lbm_multi_level_dims(self._h, out.ctypes.data_as(C.POINTER(C.c_uint32))))
        return [tuple(int(v) for v in out[3 * l:3 * l + 3]) for l in range(n)]

    def level_cells(self) -> list:
        n = self.levels()
        out = np.zeros(n, dtype=np.uint64)
        self._check(self._L.lbm_multi_level_cells(self._h, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return [int(v) for v in out]

    def run(self, fine: Iterable[StepIn] | int | np.ndarray) -> np.ndarray:
        """MultiLattice::run: force and moment per finest step (6 each)."""
        a = fine if isinstance(fine, np.ndarray) and fine.dtype == STEP_DTYPE else steps_array(fine)
        a = np.ascontiguousarray(a)
        out = np.zeros((len(a), 6), dtype=np.float64)
        self._check(self._L.lbm_multi_run(self._h, a.ctypes.data, len(a), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def advance(self, n_fine: int) -> None:
        self._check(self._L.lbm_multi_advance(self._h, int(n_fine)))

    def synchronize(self) -> None:
        self._check(self._L.lbm_multi_synchronize(self._h))

    def set_timeout(self, seconds: float) -> None:
        self._check(self._L.lbm_multi_set_timeout(self._h, float(seconds)))

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self._L.lbm_multi_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def macros(self, level: int) -> np.ndarray:
        """(rho, ux, uy, uz) per cell of a level (mlattice.rs:883-901)."""
        n = self.level_cells()[level]
        out = np.empty((n, 4), dtype=np.float32)
        self._check(self._L.lbm_multi_macros(self._h, int(level), out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def records(self) -> np.ndarray:
        n = max(self.nrec, 1) * RS27
        out = np.zeros(n, dtype=np.uint32)
        self._check(self._L.lbm_multi_records(self._h, out.ctypes.data_as(C.POINTER(C.c_uint32)), n))
        return out

    def mass(self, level: int) -> tuple[float, int]:
        m = C.c_double()
        bad = C.c_uint64()
        self._check(self._L.lbm_multi_mass(self._h, int(level), C.byref(m), C.byref(bad)))
        return m.value, int(bad.value)

    @property
    def nvert(self) -> int:
        return int(self.info().nvert)

    @property
    def npix(self) -> int:
        return int(self.info().npix)

    def reset_samples(self) -> None:
        """MultiLattice::reset_samples (mlattice.rs:844-858)."""
        self._check(self._L.lbm_multi_reset_samples(self._h))

    def vertex_means(self) -> np.ndarray:
        """Mean density at each surface vertex over the sampled finest steps
        (mlattice.rs:860-867); NaN where nothing was sampled."""
        out = np.empty(max(self.nvert, 1), dtype=np.float32)
        self._check(self._L.lbm_multi_vertex_means(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out[:self.nvert]

    def slice_means(self) -> np.ndarray:
        """Mean (rho, ux, uy, uz) per slice pixel (mlattice.rs:869-881)."""
        out = np.empty((max(self.npix, 1), 4), dtype=np.float32)
        self._check(self._L.lbm_multi_slice_means(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out[:self.npix]
