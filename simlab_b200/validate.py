"""Accuracy of reduced-precision storage against the FP64 engine.

Runs a case with each storage format and compares the mean force over the
averaging window (the last 65 % of the run, the window rule of
crates/cfd/src/tunnel.rs:1065) with the FP64 engine's, the drag-coefficient
error the metric is quoted at (Cd = F_x / (q A) with the same q and A for all
storages, so its relative error is that of the mean F_x).

    python -m simlab_b200.validate arm [steps] [storages...]
    python -m simlab_b200.validate sphere [steps]

Prints one JSON line.
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np

from .cases import arm_les, sphere_cd, sphere_re40
from .lbm import Lattice, Storage, steps_array


def run_case(make, storage, steps: int, chunk: int = 2000):
    st, vox = make(storage)
    lat = Lattice(st, vox)
    out = []
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        n = min(chunk, steps - done)
        out.append(lat.run(steps_array(n)))
        done += n
    dt = time.perf_counter() - t0
    mass, bad = lat.mass()
    lat.close()
    return np.concatenate(out), dt, bad


def window_mean(f: np.ndarray, frac: float = 0.65) -> np.ndarray:
    k = int(len(f) * (1.0 - frac))
    return f[k:].mean(axis=0)


def compare(name: str, make, steps: int, storages):
    ref, t_ref, bad = run_case(make, Storage.FP64, steps)
    mref = window_mean(ref)
    res = {"case": name, "steps": steps, "window": "last 65 %", "fp64": {"fx": mref[0], "fz": mref[2], "seconds": round(t_ref, 2),
                                                                        "nonfinite": bad}}
    for s in storages:
        f, t, bad = run_case(make, s, steps)
        m = window_mean(f)
        res[s.name.lower()] = {"fx": m[0], "fz": m[2], "drag_rel_err": abs(m[0] / mref[0] - 1.0),
                               "lift_err_over_drag": abs(m[2] - mref[2]) / abs(mref[0]), "seconds": round(t, 2), "nonfinite": bad}
    if name == "sphere":
        res["cd_fp64"] = float(sphere_cd(mref[0]))
    return res


def main() -> None:
    which = sys.argv[1] if len(sys.argv) > 1 else "arm"
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else (20000 if which == "arm" else 2000)
    names = sys.argv[3:] or ["fp32", "fp16", "bf16"]
    storages = [Storage[n.upper()] for n in names]
    make = (lambda s: arm_les(s)) if which == "arm" else (lambda s: sphere_re40(s, debug_dump=False))
    print(json.dumps(compare(which, make, steps, storages), default=float))


if __name__ == "__main__":
    main()
