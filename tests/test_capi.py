"""The C-ABI library: loads, exports every symbol include/simlab_lbm.h
declares, struct layouts match, and host-side validation errors come back
as status codes with the reference's messages (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from simlab_b200 import lbm
from simlab_b200.lbm import FaceBc, LatticeSetup, LbmError, Storage

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "simlab_lbm.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = lbm.library()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert b"sm_100a" in L.lbm_version()


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """ctypes mirrors of the C structs have the C compiler's sizes and offsets."""
    import subprocess

    from simlab_b200 import mlattice

    structs = {"lbm_setup": lbm._Setup, "lbm_geometry": lbm._Geometry, "lbm_probes": lbm._Probes, "lbm_slice_def": lbm._SliceDef,
               "lbm_info": lbm._Info, "lbm_multi_setup": mlattice._MultiSetup, "lbm_level_box": mlattice._LevelBox}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "simlab_lbm.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append('printf("lbm_wall_cell %zu\\n", sizeof(lbm_wall_cell));')
    lines.append('printf("lbm_step_in %zu\\n", sizeof(lbm_step_in));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(out[cname]) == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)
    assert int(out["lbm_wall_cell"]) == lbm.WALL_DTYPE.itemsize
    assert int(out["lbm_step_in"]) == lbm.STEP_DTYPE.itemsize


def test_setup_validation_errors_match_reference():
    with pytest.raises(LbmError, match="at least 3 cells"):
        lbm.Lattice(LatticeSetup(dims=[2, 8, 8]))
    with pytest.raises(LbmError, match="periodic faces must come in pairs"):
        lbm.Lattice(LatticeSetup(dims=[8, 8, 8], faces=[FaceBc.PERIODIC, FaceBc.OPEN] + [FaceBc.PERIODIC] * 4))
    with pytest.raises(LbmError, match="out of range"):
        lbm.Lattice(LatticeSetup(dims=[70000, 70000, 3]))


def test_multi_setup_validation_errors_match_reference():
    """mlattice.rs:198-216: nesting and periodic checks, before any device work."""
    from simlab_b200.mlattice import LevelBox, MultiLattice, MultiSetup

    base = dict(dims0=[64, 48, 48], faces=[FaceBc.VELOCITY] + [FaceBc.OPEN] * 5, nu0=0.01)
    with pytest.raises(LbmError, match="refinement box 1 does not fit inside its parent"):
        MultiLattice(MultiSetup(boxes=[LevelBox(lo=[1, 12, 12], n=[32, 24, 24])], **base))
    with pytest.raises(LbmError, match="refinement box 1 does not fit inside its parent"):
        MultiLattice(MultiSetup(boxes=[LevelBox(lo=[16, 12, 12], n=[7, 24, 24])], **base))
    with pytest.raises(LbmError, match="refinement box 2 does not fit inside its parent"):
        MultiLattice(MultiSetup(boxes=[LevelBox(lo=[16, 12, 12], n=[32, 24, 24]), LevelBox(lo=[2, 10, 10], n=[20, 20, 20])], **base))
    with pytest.raises(LbmError, match="periodic faces only work without refinement"):
        MultiLattice(MultiSetup(dims0=[64, 48, 48], faces=[FaceBc.PERIODIC] * 6, nu0=0.01, boxes=[LevelBox(lo=[16, 12, 12], n=[32, 24, 24])]))
    with pytest.raises(LbmError, match="free-slip"):
        MultiLattice(MultiSetup(dims0=[16, 16, 16], faces=[FaceBc.FREE_SLIP] * 6, nu0=0.01))


def test_max_cells():
    assert lbm.Lattice.max_cells(Storage.FP16) == 0xFFFFFFFE
