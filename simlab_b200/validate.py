"""Accuracy of reduced-precision storage against the FP64 engine.

Runs a case with each storage format and compares the mean force over the
averaging window (the last 65 % of the run, the window rule of
crates/cfd/src/tunnel.rs:1065) with the FP64 engine's, the drag-coefficient
error the metric is quoted at (Cd = F_x / (q A) with the same q and A for all
storages, so its relative error is that of the mean F_x).

    python -m simlab_b200.validate arm [steps] [storages...]
    python -m simlab_b200.validate sphere [steps]
    python -m simlab_b200.validate prop [revolutions] [storages...] [nu=<finest-level viscosity>]

The rotor case (simlab_b200.cases.prop_refined: three D3Q27 levels, a 2-blade
rotor spinning on the finest) reports thrust (force along the spin axis) and
torque (moment about it), averaged over the last revolution, per storage,
beside the device time.

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


def run_prop(storage, revs: float, chunk: int = 4096, nu_finest: float = 4e-5):
    import math

    from .cases import prop_refined, spin_schedule
    from .mlattice import MultiLattice

    s, geo, om = prop_refined(storage, nu_finest=nu_finest)
    lat = MultiLattice(s, geo)
    ss = lat.sub_steps()
    per_rev = 2.0 * math.pi / om
    n = int(round(revs * per_rev / ss)) * ss
    ramp = int(round(0.5 * per_rev))
    sched = spin_schedule(n, om, ramp)
    out = []
    t0 = time.perf_counter()
    for k in range(0, n, chunk):
        out.append(lat.run(sched[k:k + chunk]))
    dt = time.perf_counter() - t0
    f = np.concatenate(out)
    last = f[-int(round(per_rev / ss)) * ss:]
    cells = lat.level_cells()
    mlups = sum(c * 2 ** l for l, c in enumerate(cells)) / 2 ** (len(cells) - 1) * n / dt / 1e6
    lat.close()
    return {"thrust": float(last[:, 0].mean()), "torque": float(last[:, 3].mean()), "steps": n, "seconds": round(dt, 2), "mlups_wall": round(mlups, 1),
            "finite": bool(np.all(np.isfinite(f)))}


def main() -> None:
    which = sys.argv[1] if len(sys.argv) > 1 else "arm"
    if which == "prop":
        revs = float(sys.argv[2]) if len(sys.argv) > 2 else 10.0
        rest = sys.argv[3:]
        nu = 4e-5
        for a in list(rest):
            if a.startswith("nu="):
                nu = float(a[3:])
                rest.remove(a)
        names = rest or ["fp32", "fp16"]
        res = {"case": "prop", "revolutions": revs, "nu_finest": nu}
        for nm in names:
            res[nm] = run_prop(Storage[nm.upper()], revs, nu_finest=nu)
        if "fp32" in res and "fp16" in res:
            res["fp16_thrust_rel_err"] = abs(res["fp16"]["thrust"] / res["fp32"]["thrust"] - 1.0)
            res["fp16_torque_rel_err"] = abs(res["fp16"]["torque"] / res["fp32"]["torque"] - 1.0)
        print(json.dumps(res))
        return
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else (20000 if which == "arm" else 2000)
    names = sys.argv[3:] or ["fp32", "fp16", "bf16"]
    storages = [Storage[n.upper()] for n in names]
    make = (lambda s: arm_les(s)) if which == "arm" else (lambda s: sphere_re40(s, debug_dump=False))
    print(json.dumps(compare(which, make, steps, storages), default=float))


if __name__ == "__main__":
    main()
