"""TEST INFRASTRUCTURE -- ctypes mirrors of the C structs the oracle takes
(lbm_setup and lbm_geometry of include/simlab_lbm.h), so the oracle can be
driven from frozen inputs without importing the engine's package."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np


class Setup(C.Structure):
    _fields_ = [("dims", C.c_uint32 * 3), ("faces", C.c_int32 * 6), ("nu", C.c_double), ("smagorinsky", C.c_double),
                ("u_inf", C.c_double * 3), ("u_init", C.c_double * 3), ("body_force", C.c_double * 3), ("sponge", C.c_uint32 * 6),
                ("sponge_tau", C.c_double), ("sponge_sigma", C.c_double), ("absorb_velocity", C.c_int32),
                ("total_pressure_inlet", C.c_int32), ("storage", C.c_int32), ("collision", C.c_int32), ("center", C.c_double * 3),
                ("debug_dump", C.c_int32), ("wall_model", C.c_int32)]


class Geometry(C.Structure):
    _fields_ = [("kind", C.c_int32), ("_pad", C.c_int32), ("solid", C.c_void_p), ("nsolid", C.c_uint64), ("walls", C.c_void_p),
                ("nwalls", C.c_uint64), ("occ_bits", C.c_void_p), ("occ_lo", C.c_double * 3), ("occ_h", C.c_double),
                ("occ_dims", C.c_uint32 * 3), ("_pad2", C.c_uint32), ("tris", C.c_void_p), ("ntri", C.c_uint64),
                ("box_lo", C.c_int32 * 3), ("box_n", C.c_uint32 * 3)]


WALL_DTYPE = np.dtype([("cell", "<u4"), ("mask", "<u4"), ("q", "<f4", (27,))])


class FrozenSetup:
    """The setup fields of a fixture, with the two helpers the oracle's wrapper uses."""

    def __init__(self, d: dict):
        self.__dict__.update(d)

    def cells(self) -> int:
        return int(self.dims[0]) * int(self.dims[1]) * int(self.dims[2])

    def to_c(self) -> Setup:
        s = Setup()
        for name, _ in Setup._fields_:
            v = getattr(self, name)
            if isinstance(v, (list, tuple)):
                getattr(s, name)[:] = v
            else:
                setattr(s, name, v)
        return s


def load_case(path: Path):
    """(FrozenSetup, Geometry struct, arrays to keep alive) of a fixture written
    by oracle/make_arm_fixture.py."""
    z = np.load(path)
    setup = FrozenSetup(json.loads(bytes(z["setup"]).decode()))
    solid = np.ascontiguousarray(z["solid"], dtype=np.uint32)
    walls = np.ascontiguousarray(z["walls"])
    if walls.dtype != WALL_DTYPE:
        raise TypeError("fixture walls must use the lbm_wall_cell layout")
    g = Geometry()
    g.kind = 1
    g.solid = solid.ctypes.data
    g.nsolid = solid.size
    g.walls = walls.ctypes.data
    g.nwalls = walls.size
    return setup, g, [solid, walls]
