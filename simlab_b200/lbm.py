"""Python mirror of the reference's lattice API over the C ABI.

`Lattice`, `LatticeSetup`, `StepIn`, `Storage`, `FaceBc`, `Probes`,
`SliceDef`, `StaticVoxels`, `voxelize_static` and `inside_grid` follow
crates/cfd/src/lattice.rs and crates/cfd/src/voxel.rs: same names, same
argument meaning, same units (lattice units), and errors raised where the
reference bails.  Every call goes to libsimlab_lbm.so (include/simlab_lbm.h);
there is no Python or CPU fallback: if the library is missing, importing a
lattice raises.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from pathlib import Path
from typing import Iterable, Sequence

import numpy as np

_PKG = Path(__file__).resolve().parent
_LIB_PATH = _PKG / "libsimlab_lbm.so"


class LbmError(RuntimeError):
    """A failed engine call (the reference's anyhow::Error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


class Storage(enum.IntEnum):
    """`Storage` (lattice.rs:11-32) plus BF16 and FP64."""

    FP32 = 0
    FP16 = 1
    BF16 = 2
    FP64 = 3

    def pop_bytes(self) -> int:
        return {0: 4, 1: 2, 2: 2, 3: 8}[int(self)]

    def bytes_per_cell(self) -> int:
        """19 populations + one u32 flag word (lattice.rs:28-31)."""
        return 19 * self.pop_bytes() + 4


class FaceBc(enum.IntEnum):
    """`FaceBc` (lattice.rs:34-43) plus FREE_SLIP."""

    VELOCITY = 0
    OPEN = 1
    PERIODIC = 2
    FREE_SLIP = 3


class Collision(enum.IntEnum):
    REGULARIZED = 0
    BGK = 1


# ------------------------------------------------------------------ C structs
class _Setup(C.Structure):
    _fields_ = [
        ("dims", C.c_uint32 * 3),
        ("faces", C.c_int32 * 6),
        ("nu", C.c_double),
        ("smagorinsky", C.c_double),
        ("u_inf", C.c_double * 3),
        ("u_init", C.c_double * 3),
        ("body_force", C.c_double * 3),
        ("sponge", C.c_uint32 * 6),
        ("sponge_tau", C.c_double),
        ("sponge_sigma", C.c_double),
        ("absorb_velocity", C.c_int32),
        ("total_pressure_inlet", C.c_int32),
        ("storage", C.c_int32),
        ("collision", C.c_int32),
        ("center", C.c_double * 3),
        ("debug_dump", C.c_int32),
        ("wall_model", C.c_int32),
    ]


WALL_DTYPE = np.dtype([("cell", "<u4"), ("mask", "<u4"), ("q", "<f4", (27,))])


class _Geometry(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("_pad", C.c_int32),
        ("solid", C.POINTER(C.c_uint32)),
        ("nsolid", C.c_uint64),
        ("walls", C.c_void_p),
        ("nwalls", C.c_uint64),
        ("occ_bits", C.POINTER(C.c_uint32)),
        ("occ_lo", C.c_double * 3),
        ("occ_h", C.c_double),
        ("occ_dims", C.c_uint32 * 3),
        ("_pad2", C.c_uint32),
        ("tris", C.POINTER(C.c_float)),
        ("ntri", C.c_uint64),
        ("box_lo", C.c_int32 * 3),
        ("box_n", C.c_uint32 * 3),
    ]


class _SpinInfo(C.Structure):
    _fields_ = [
        ("occ_lo", C.c_double * 3),
        ("occ_h", C.c_double),
        ("occ_dims", C.c_uint32 * 3),
        ("_pad", C.c_uint32),
        ("occ_words", C.c_uint64),
        ("ntri", C.c_uint64),
        ("radius", C.c_double),
        ("axial", C.c_double * 2),
    ]


class _SliceDef(C.Structure):
    _fields_ = [("origin", C.c_int32 * 3), ("u", C.c_int32 * 3), ("v", C.c_int32 * 3), ("nu", C.c_uint32), ("nv", C.c_uint32)]


class _Probes(C.Structure):
    _fields_ = [
        ("verts", C.POINTER(C.c_double)),
        ("nvert", C.c_uint64),
        ("slices", C.POINTER(_SliceDef)),
        ("nslices", C.c_uint64),
        ("vertex_offset", C.c_double),
    ]


STEP_DTYPE = np.dtype([("rot", "<f8", (3, 3)), ("rot_prev", "<f8", (3, 3)), ("omega", "<f8", (3,)), ("sample", "<i4"), ("_pad", "<i4")])


class _KernelTimes(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("faces_ms", C.c_double), ("walls_ms", C.c_double), ("bulk_ms", C.c_double),
                ("launches", C.c_uint64)]


class _Info(C.Structure):
    _fields_ = [
        ("steps_done", C.c_uint64),
        ("nrec", C.c_uint32),
        ("nface", C.c_uint32),
        ("npix", C.c_uint32),
        ("nvert", C.c_uint32),
        ("memory_bytes", C.c_uint64),
        ("cells", C.c_uint64),
        ("storage", C.c_int32),
        ("collision", C.c_int32),
    ]


_lib_handle = None


def library() -> C.CDLL:
    """The engine library; raises if it has not been built (no fallback)."""
    global _lib_handle
    if _lib_handle is not None:
        return _lib_handle
    if not _LIB_PATH.exists():
        raise ImportError(f"{_LIB_PATH.name} is not built; run `python -m simlab_b200.build` (needs nvcc)")
    L = C.CDLL(str(_LIB_PATH))
    vp, u64, i32, dp = C.c_void_p, C.c_uint64, C.c_int32, C.POINTER(C.c_double)
    L.lbm_version.restype = C.c_char_p
    L.lbm_global_error.argtypes = [C.c_char_p, u64]
    L.lbm_last_error.argtypes = [vp, C.c_char_p, u64]
    L.lbm_max_cells.argtypes = [i32]
    L.lbm_max_cells.restype = u64
    L.lbm_create.argtypes = [C.POINTER(_Setup), C.POINTER(_Geometry), C.POINTER(_Probes), C.POINTER(vp)]
    L.lbm_destroy.argtypes = [vp]
    L.lbm_destroy.restype = None
    L.lbm_run.argtypes = [vp, vp, u64, dp]
    L.lbm_advance.argtypes = [vp, u64]
    L.lbm_stream.argtypes = [vp, C.POINTER(vp)]
    L.lbm_synchronize.argtypes = [vp]
    L.lbm_set_timeout.argtypes = [vp, C.c_double]
    L.lbm_selftest_copy_wait.argtypes = [u64, C.POINTER(C.c_uint32), C.POINTER(u64)]
    L.lbm_profile.argtypes = [vp, i32]
    L.lbm_get_kernel_times.argtypes = [vp, C.POINTER(_KernelTimes)]
    L.lbm_macros.argtypes = [vp, C.POINTER(C.c_float)]
    L.lbm_records.argtypes = [vp, C.POINTER(C.c_uint32), u64]
    L.lbm_reset_samples.argtypes = [vp]
    L.lbm_vertex_means.argtypes = [vp, C.POINTER(C.c_float)]
    L.lbm_slice_means.argtypes = [vp, C.POINTER(C.c_float)]
    L.lbm_get_info.argtypes = [vp, C.POINTER(_Info)]
    L.lbm_mass.argtypes = [vp, dp, C.POINTER(u64)]
    L.lbm_state_size.argtypes = [vp, C.POINTER(u64)]
    L.lbm_save_state.argtypes = [vp, vp, u64]
    L.lbm_load_state.argtypes = [vp, vp, u64]
    L.lbm_voxelize_static.argtypes = [dp, u64, C.POINTER(C.c_uint32), u64, C.POINTER(C.c_uint32), i32, C.POINTER(vp)]
    L.lbm_voxelize_static_gpu.argtypes = [dp, u64, C.POINTER(C.c_uint32), u64, C.POINTER(C.c_uint32), i32, C.POINTER(vp)]
    L.lbm_voxels_counts.argtypes = [vp, C.POINTER(u64), C.POINTER(u64)]
    L.lbm_voxels_copy.argtypes = [vp, C.POINTER(C.c_uint32), vp]
    L.lbm_voxels_free.argtypes = [vp]
    L.lbm_voxels_free.restype = None
    L.lbm_inside_grid.argtypes = [dp, u64, C.POINTER(C.c_uint32), u64, dp, C.c_double, C.POINTER(C.c_uint32), C.POINTER(C.c_uint8)]
    L.lbm_voxelize_spin.argtypes = [dp, u64, C.POINTER(C.c_uint32), u64, dp, C.c_double, C.POINTER(vp)]
    L.lbm_spin_voxels_info.argtypes = [vp, C.POINTER(_SpinInfo)]
    L.lbm_spin_voxels_copy.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_float)]
    L.lbm_spin_voxels_free.argtypes = [vp]
    L.lbm_spin_voxels_free.restype = None
    L.lbm_record_forces_noalloc.argtypes = [vp, u64, vp, vp]
    L.lbm_record_forces_noalloc_max.restype = u64
    L.lbm_noalloc_error.argtypes = [C.c_char_p, u64]
    _lib_handle = L
    return L


def _global_error(code: int) -> LbmError:
    buf = C.create_string_buffer(1024)
    library().lbm_global_error(buf, 1024)
    return LbmError(code, buf.value.decode(errors="replace"))


# ------------------------------------------------------------------ setup types
def _v3(x) -> tuple:
    t = tuple(float(v) for v in x)
    if len(t) != 3:
        raise ValueError("expected 3 components")
    return t


@dataclass
class LatticeSetup:
    """`LatticeSetup` (lattice.rs:45-76) plus `collision`."""

    dims: Sequence[int]
    faces: Sequence[FaceBc] = (FaceBc.PERIODIC,) * 6
    nu: float = 0.1
    smagorinsky: float = 0.0
    u_inf: Sequence[float] = (0.0, 0.0, 0.0)
    u_init: Sequence[float] = (0.0, 0.0, 0.0)
    body_force: Sequence[float] = (0.0, 0.0, 0.0)
    sponge: Sequence[int] = (0, 0, 0, 0, 0, 0)
    sponge_tau: float = 0.0
    sponge_sigma: float = 0.0
    absorb_velocity: bool = False
    total_pressure_inlet: bool = False
    storage: Storage = Storage.FP32
    center: Sequence[float] = (0.0, 0.0, 0.0)
    debug_dump: bool = False
    wall_model: bool = False
    collision: Collision = Collision.REGULARIZED

    def cells(self) -> int:
        return int(self.dims[0]) * int(self.dims[1]) * int(self.dims[2])

    def periodic(self) -> tuple:
        return tuple(FaceBc(self.faces[2 * a]) == FaceBc.PERIODIC for a in range(3))

    def to_c(self) -> _Setup:
        s = _Setup()
        s.dims[:] = [int(d) for d in self.dims]
        if len(self.faces) != 6:
            raise ValueError("faces must list -x,+x,-y,+y,-z,+z")
        s.faces[:] = [int(f) for f in self.faces]
        s.nu = float(self.nu)
        s.smagorinsky = float(self.smagorinsky)
        s.u_inf[:] = _v3(self.u_inf)
        s.u_init[:] = _v3(self.u_init)
        s.body_force[:] = _v3(self.body_force)
        s.sponge[:] = [int(v) for v in self.sponge]
        s.sponge_tau = float(self.sponge_tau)
        s.sponge_sigma = float(self.sponge_sigma)
        s.absorb_velocity = int(bool(self.absorb_velocity))
        s.total_pressure_inlet = int(bool(self.total_pressure_inlet))
        s.storage = int(self.storage)
        s.collision = int(self.collision)
        s.center[:] = _v3(self.center)
        s.debug_dump = int(bool(self.debug_dump))
        s.wall_model = int(bool(self.wall_model))
        return s


@dataclass
class StaticVoxels:
    """`StaticVoxels` (voxel.rs:337-344): solid cells and wall cells."""

    solid: np.ndarray
    walls: np.ndarray  # WALL_DTYPE records: cell, mask, q[27]
    lo: tuple = (0, 0, 0)
    hi: tuple = (0, 0, 0)


@dataclass
class SpinVoxels:
    """`SpinVoxels` (voxel.rs:492-505): body-frame occupancy bits on a grid of
    spacing occ_h from occ_lo, and the surface as (v0, e1, e2) triangles."""

    occ_lo: tuple
    occ_h: float
    occ_dims: tuple
    occ_bits: np.ndarray  # uint32
    tris: np.ndarray      # float32, (ntri, 12)
    radius: float
    axial: tuple


@dataclass
class SpinGeometry:
    """`Geometry::Spin` (lattice.rs:87-92): the part and the swept box of
    lattice cells that holds every cell it can reach."""

    vox: SpinVoxels
    box_lo: Sequence[int]
    box_n: Sequence[int]


@dataclass
class SliceDef:
    """`SliceDef` (shader.rs:77-84)."""

    origin: Sequence[int]
    u: Sequence[int]
    v: Sequence[int]
    nu: int
    nv: int


@dataclass
class Probes:
    """`Probes` (lattice.rs:94-102)."""

    verts: list = field(default_factory=list)  # [(p[3], n[3]), ...] body coordinates relative to centre
    slices: list = field(default_factory=list)
    vertex_offset: float = 0.0


IDENTITY = np.eye(3)


@dataclass
class StepIn:
    """`StepIn` (lattice.rs:104-121)."""

    rot: np.ndarray = field(default_factory=lambda: np.eye(3))
    rot_prev: np.ndarray = field(default_factory=lambda: np.eye(3))
    omega: Sequence[float] = (0.0, 0.0, 0.0)
    sample: bool = False

    @staticmethod
    def still(sample: bool = False) -> "StepIn":
        return StepIn(sample=sample)


def steps_array(steps: Iterable[StepIn] | int, sample: bool = False) -> np.ndarray:
    """Packs StepIn values (or n still steps) into the C layout."""
    if isinstance(steps, (int, np.integer)):
        a = np.zeros(int(steps), dtype=STEP_DTYPE)
        a["rot"] = np.eye(3)
        a["rot_prev"] = np.eye(3)
        a["sample"] = int(sample)
        return a
    steps = list(steps)
    a = np.zeros(len(steps), dtype=STEP_DTYPE)
    for k, s in enumerate(steps):
        a[k]["rot"] = np.asarray(s.rot, dtype=np.float64)
        a[k]["rot_prev"] = np.asarray(s.rot_prev, dtype=np.float64)
        a[k]["omega"] = np.asarray(s.omega, dtype=np.float64)
        a[k]["sample"] = int(bool(s.sample))
    return a


def geometry_struct(geom) -> tuple[_Geometry, list]:
    """The C struct of None, a StaticVoxels or a SpinGeometry."""
    g = _Geometry()
    keep: list = []
    if geom is None:
        g.kind = 0
        return g, keep
    if isinstance(geom, SpinGeometry):
        v = geom.vox
        occ = np.ascontiguousarray(v.occ_bits, dtype=np.uint32)
        tris = np.ascontiguousarray(v.tris, dtype=np.float32).reshape(-1, 12)
        keep += [occ, tris]
        g.kind = 2
        g.occ_bits = occ.ctypes.data_as(C.POINTER(C.c_uint32))
        g.occ_lo[:] = [float(x) for x in v.occ_lo]
        g.occ_h = float(v.occ_h)
        g.occ_dims[:] = [int(x) for x in v.occ_dims]
        g.tris = tris.ctypes.data_as(C.POINTER(C.c_float))
        g.ntri = len(tris)
        g.box_lo[:] = [int(x) for x in geom.box_lo]
        g.box_n[:] = [int(x) for x in geom.box_n]
        return g, keep
    solid = np.ascontiguousarray(geom.solid, dtype=np.uint32)
    walls = np.ascontiguousarray(geom.walls)
    if walls.dtype != WALL_DTYPE:
        raise TypeError("walls must use WALL_DTYPE")
    keep += [solid, walls]
    g.kind = 1
    g.solid = solid.ctypes.data_as(C.POINTER(C.c_uint32))
    g.nsolid = solid.size
    g.walls = walls.ctypes.data
    g.nwalls = walls.size
    return g, keep


def probes_struct(probes: Probes | None) -> tuple[_Probes | None, list]:
    if probes is None or (not probes.verts and not probes.slices):
        return None, []
    p = _Probes()
    v = np.ascontiguousarray(np.array([list(a) + list(b) for a, b in probes.verts], dtype=np.float64).reshape(-1, 6))
    sl = (_SliceDef * max(len(probes.slices), 1))()
    for k, s in enumerate(probes.slices):
        sl[k].origin[:] = [int(x) for x in s.origin]
        sl[k].u[:] = [int(x) for x in s.u]
        sl[k].v[:] = [int(x) for x in s.v]
        sl[k].nu = int(s.nu)
        sl[k].nv = int(s.nv)
    p.verts = v.ctypes.data_as(C.POINTER(C.c_double))
    p.nvert = len(probes.verts)
    p.slices = C.cast(sl, C.POINTER(_SliceDef))
    p.nslices = len(probes.slices)
    p.vertex_offset = float(probes.vertex_offset)
    return p, [v, sl]


class Lattice:
    """`Lattice` (lattice.rs:148-842) on one B200.

    Lattice(setup, geometry, probes): geometry is None (`Geometry::None`) or
    a `StaticVoxels` (`Geometry::Static`).
    """

    def __init__(self, setup: LatticeSetup, geometry: StaticVoxels | None = None, probes: Probes | None = None):
        L = library()
        self._L = L
        self.setup = setup
        cs = setup.to_c()
        g, keep = geometry_struct(geometry)
        p, keep2 = probes_struct(probes)
        h = C.c_void_p()
        rc = L.lbm_create(C.byref(cs), C.byref(g), C.byref(p) if p is not None else None, C.byref(h))
        del keep, keep2
        if rc != 0:
            raise _global_error(rc)
        self._h = h

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.lbm_destroy(self._h)
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
            self._L.lbm_last_error(self._h, buf, 1024)
            raise LbmError(rc, buf.value.decode(errors="replace"))

    # -- public fields (lattice.rs:148-170)
    def info(self) -> _Info:
        i = _Info()
        self._check(self._L.lbm_get_info(self._h, C.byref(i)))
        return i

    @property
    def steps_done(self) -> int:
        return int(self.info().steps_done)

    @property
    def nrec(self) -> int:
        return int(self.info().nrec)

    @property
    def nface(self) -> int:
        return int(self.info().nface)

    @property
    def npix(self) -> int:
        return int(self.info().npix)

    @property
    def memory_bytes(self) -> int:
        return int(self.info().memory_bytes)

    # -- stepping
    def run(self, steps: Iterable[StepIn] | int | np.ndarray) -> np.ndarray:
        """Lattice::run: force and moment (6 per step) on the geometry after each step."""
        a = steps if isinstance(steps, np.ndarray) and steps.dtype == STEP_DTYPE else steps_array(steps)
        a = np.ascontiguousarray(a)
        out = np.zeros((len(a), 6), dtype=np.float64)
        self._check(self._L.lbm_run(self._h, a.ctypes.data, len(a), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def advance(self, n: int) -> None:
        """Enqueues n still steps without waiting (forces stay on the device)."""
        self._check(self._L.lbm_advance(self._h, int(n)))

    def synchronize(self) -> None:
        self._check(self._L.lbm_synchronize(self._h))

    def set_timeout(self, seconds: float) -> None:
        self._check(self._L.lbm_set_timeout(self._h, float(seconds)))

    def profile(self, enable) -> None:
        """Starts (clearing the totals) or stops per-kernel event timing:
        True or 1 times faces, walls and bulk; 2 only the bulk kernel; False
        or 0 stops."""
        self._check(self._L.lbm_profile(self._h, int(enable)))

    def kernel_times(self) -> dict:
        """Device milliseconds per kernel summed over the profiled steps."""
        t = _KernelTimes()
        self._check(self._L.lbm_get_kernel_times(self._h, C.byref(t)))
        return {"steps": int(t.steps), "faces_ms": t.faces_ms, "walls_ms": t.walls_ms, "bulk_ms": t.bulk_ms, "launches": int(t.launches)}

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self._L.lbm_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    # -- readback
    def macros(self) -> np.ndarray:
        """(rho, ux, uy, uz) of every cell; NaN for solid and face cells."""
        n = self.setup.cells()
        out = np.empty((n, 4), dtype=np.float32)
        self._check(self._L.lbm_macros(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def records(self) -> np.ndarray:
        n = max(self.nrec, 1) * 40
        out = np.zeros(n, dtype=np.uint32)
        self._check(self._L.lbm_records(self._h, out.ctypes.data_as(C.POINTER(C.c_uint32)), n))
        return out

    def reset_samples(self) -> None:
        self._check(self._L.lbm_reset_samples(self._h))

    def vertex_means(self) -> np.ndarray:
        n = int(self.info().nvert)
        out = np.zeros(n, dtype=np.float32)
        if n:
            self._check(self._L.lbm_vertex_means(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def slice_means(self) -> np.ndarray:
        n = self.npix
        out = np.zeros((n, 4), dtype=np.float32)
        if n:
            self._check(self._L.lbm_slice_means(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def mass(self) -> tuple[float, int]:
        """FP64 sum of the density over fluid cells and the non-finite count."""
        m = C.c_double()
        bad = C.c_uint64()
        self._check(self._L.lbm_mass(self._h, C.byref(m), C.byref(bad)))
        return m.value, int(bad.value)

    # -- checkpoint
    def save_state(self) -> bytes:
        n = C.c_uint64()
        self._check(self._L.lbm_state_size(self._h, C.byref(n)))
        buf = (C.c_char * n.value)()
        self._check(self._L.lbm_save_state(self._h, buf, n.value))
        return bytes(buf)

    def load_state(self, blob: bytes) -> None:
        buf = C.create_string_buffer(blob, len(blob))
        self._check(self._L.lbm_load_state(self._h, buf, len(blob)))

    @staticmethod
    def max_cells(storage: Storage) -> int:
        return int(library().lbm_max_cells(int(storage)))


# ------------------------------------------------------------------ voxelizer
def _surface_arrays(verts, tris):
    v = np.ascontiguousarray(np.asarray(verts, dtype=np.float64).reshape(-1, 3))
    t = np.ascontiguousarray(np.asarray(tris, dtype=np.uint32).reshape(-1, 3))
    return v, t


def voxelize_static(verts, tris, dims: Sequence[int], lattice: int = 19, device: bool = False) -> StaticVoxels:
    """voxelize_static / voxelize_static27 (voxel.rs:346-359): on the host
    cores, or with device=True on the current CUDA device
    (lbm_voxelize_static_gpu, the same result bit for bit)."""
    L = library()
    v, t = _surface_arrays(verts, tris)
    d = (C.c_uint32 * 3)(*[int(x) for x in dims])
    h = C.c_void_p()
    fn = L.lbm_voxelize_static_gpu if device else L.lbm_voxelize_static
    rc = fn(v.ctypes.data_as(C.POINTER(C.c_double)), len(v), t.ctypes.data_as(C.POINTER(C.c_uint32)), len(t), d, int(lattice), C.byref(h))
    if rc != 0:
        raise _global_error(rc)
    try:
        ns, nw = C.c_uint64(), C.c_uint64()
        L.lbm_voxels_counts(h, C.byref(ns), C.byref(nw))
        solid = np.zeros(ns.value, dtype=np.uint32)
        walls = np.zeros(nw.value, dtype=WALL_DTYPE)
        L.lbm_voxels_copy(h, solid.ctypes.data_as(C.POINTER(C.c_uint32)), walls.ctypes.data)
    finally:
        L.lbm_voxels_free(h)
    return StaticVoxels(solid=solid, walls=walls)


def voxelize_spin(verts, tris, axis: Sequence[float] = (0.0, 0.0, 1.0), h: float = 0.125) -> SpinVoxels:
    """voxelize_spin (voxel.rs:507-560): the part in body coordinates (lattice
    units, origin at the spin centre)."""
    L = library()
    v, t = _surface_arrays(verts, tris)
    ax = (C.c_double * 3)(*[float(x) for x in axis])
    hnd = C.c_void_p()
    rc = L.lbm_voxelize_spin(v.ctypes.data_as(C.POINTER(C.c_double)), len(v), t.ctypes.data_as(C.POINTER(C.c_uint32)), len(t), ax, float(h),
                             C.byref(hnd))
    if rc != 0:
        raise _global_error(rc)
    try:
        info = _SpinInfo()
        L.lbm_spin_voxels_info(hnd, C.byref(info))
        occ = np.zeros(int(info.occ_words), dtype=np.uint32)
        tr = np.zeros((int(info.ntri), 12), dtype=np.float32)
        L.lbm_spin_voxels_copy(hnd, occ.ctypes.data_as(C.POINTER(C.c_uint32)), tr.ctypes.data_as(C.POINTER(C.c_float)))
    finally:
        L.lbm_spin_voxels_free(hnd)
    return SpinVoxels(occ_lo=tuple(info.occ_lo), occ_h=info.occ_h, occ_dims=tuple(info.occ_dims), occ_bits=occ, tris=tr, radius=info.radius,
                      axial=tuple(info.axial))


def inside_grid(verts, tris, origin: Sequence[float], h: float, dims: Sequence[int]) -> np.ndarray:
    """inside_grid (voxel.rs:73-95): bool per grid point origin + h (i, j, k)."""
    L = library()
    v, t = _surface_arrays(verts, tris)
    o = (C.c_double * 3)(*[float(x) for x in origin])
    d = (C.c_uint32 * 3)(*[int(x) for x in dims])
    out = np.zeros(int(dims[0]) * int(dims[1]) * int(dims[2]), dtype=np.uint8)
    rc = L.lbm_inside_grid(v.ctypes.data_as(C.POINTER(C.c_double)), len(v), t.ctypes.data_as(C.POINTER(C.c_uint32)), len(t), o,
                           float(h), d, out.ctypes.data_as(C.POINTER(C.c_uint8)))
    if rc != 0:
        raise _global_error(rc)
    return out.astype(bool)


def record_forces_noalloc(records_dev_ptr: int, nrec: int, forces_dev_ptr: int, stream: int = 0) -> None:
    """Force and moment sum over wall records already in device memory, into
    6 doubles in device memory, without allocating anything (enqueued on
    `stream`; see lbm_record_forces_noalloc in include/simlab_lbm.h)."""
    L = library()
    rc = L.lbm_record_forces_noalloc(C.c_void_p(records_dev_ptr), int(nrec), C.c_void_p(forces_dev_ptr), C.c_void_p(stream or None))
    if rc != 0:
        buf = C.create_string_buffer(512)
        L.lbm_noalloc_error(buf, 512)
        raise LbmError(rc, buf.value.decode(errors="replace"))


def selftest_copy_wait(limit_s: float = 0.005) -> tuple[bool, float]:
    """Runs the step kernel's bounded wait on a copy barrier that nothing
    completes, limited to `limit_s` seconds: returns (gave_up, seconds waited).
    The wait ends by itself; no fault and no hang."""
    gave_up = C.c_uint32(0)
    waited = C.c_uint64(0)
    rc = library().lbm_selftest_copy_wait(int(limit_s * 1e9), C.byref(gave_up), C.byref(waited))
    if rc != 0:
        raise _global_error(rc)
    return bool(gave_up.value), waited.value * 1e-6


def halfway(vox: StaticVoxels) -> StaticVoxels:
    """Same links with every wall distance set to 1/2 (halfway bounce-back)."""
    w = vox.walls.copy()
    for d in range(27):
        cut = (w["mask"] >> np.uint32(d)) & np.uint32(1)
        w["q"][:, d] = np.where(cut == 1, np.float32(0.5), w["q"][:, d])
    return StaticVoxels(solid=vox.solid.copy(), walls=w, lo=vox.lo, hi=vox.hi)
