"""Accuracy of reduced-precision storage against the FP64 engine.

Runs a case with each storage format and compares the mean force over the
averaging window (the last 65 % of the run, the window rule of
crates/cfd/src/tunnel.rs:1065) with the FP64 engine's, the drag-coefficient
error the metric is quoted at (Cd = F_x / (q A) with the same q and A for all
storages, so its relative error is that of the mean F_x).

    python -m simlab_b200.validate arm [steps] [storages...]
    python -m simlab_b200.validate sphere [steps]
    python -m simlab_b200.validate prop [revolutions] [storages...] [nu=<finest-level viscosity>] [window=<fraction>]

A storage name `fp64p` runs the FP64 engine from a perturbed initial state
(u_init plus 1e-6 of the inflow speed across the flow; `fp64p<k>` k times
that): its difference from the plain FP64 run is the noise floor of the flow
itself, the spread two runs whose roundings differ would show even with exact
storage.

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


PERTURB = 1e-6  # fraction of the inflow speed added to u_init across the flow by `fp64p`


def storage_of(name: str):
    """(Storage, perturbation multiple) of a storage name: `fp64p<k>` is FP64
    from an initial state perturbed k times PERTURB (k = 1 when omitted)."""
    nm = name.lower()
    if nm.startswith("fp64p"):
        return Storage.FP64, float(nm[5:] or 1)
    return Storage[name.upper()], 0.0


def perturb_u_init(st, k: float = 1.0) -> None:
    u = float(np.linalg.norm(st.u_inf)) or 0.01
    ui = list(st.u_init)
    ui[1] += k * PERTURB * u
    ui[2] -= 0.5 * k * PERTURB * u
    st.u_init = ui


def run_case(make, storage, steps: int, chunk: int = 2000, perturbed: float = 0.0):
    st, vox = make(storage)
    if perturbed:
        perturb_u_init(st, perturbed)
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
    for nm in storages:
        s, pert = storage_of(nm)
        f, t, bad = run_case(make, s, steps, perturbed=pert)
        m = window_mean(f)
        res[nm] = {"fx": m[0], "fz": m[2], "drag_rel_err": abs(m[0] / mref[0] - 1.0),
                               "lift_err_over_drag": abs(m[2] - mref[2]) / abs(mref[0]),
                   "lift_rel_err": abs(m[2] / mref[2] - 1.0) if mref[2] != 0 else None, "seconds": round(t, 2), "nonfinite": bad}
    if name == "sphere":
        res["cd_fp64"] = float(sphere_cd(mref[0]))
    return res


def run_prop(storage, revs: float, chunk: int = 4096, nu_finest: float = 4e-5, perturbed: float = 0.0, window: float = 0.0):
    import math

    from .cases import prop_refined, spin_schedule
    from .mlattice import MultiLattice

    s, geo, om = prop_refined(storage, nu_finest=nu_finest)
    if perturbed:
        perturb_u_init(s, perturbed)
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
    # the last revolution, or the last `window` fraction of the run
    last = f[-int(round(per_rev / ss)) * ss:] if window <= 0 else f[int(len(f) * (1.0 - window)):]
    cells = lat.level_cells()
    mlups = sum(c * 2 ** l for l, c in enumerate(cells)) / 2 ** (len(cells) - 1) * n / dt / 1e6
    lat.close()
    half = len(last) // 2
    return {"thrust": float(last[:, 0].mean()), "torque": float(last[:, 3].mean()),
            "thrust_halves": [float(last[:half, 0].mean()), float(last[half:, 0].mean())],
            "torque_halves": [float(last[:half, 3].mean()), float(last[half:, 3].mean())], "steps": n, "seconds": round(dt, 2),
            "mlups_wall": round(mlups, 1), "finite": bool(np.all(np.isfinite(f)))}


def main() -> None:
    which = sys.argv[1] if len(sys.argv) > 1 else "arm"
    if which == "prop":
        revs = float(sys.argv[2]) if len(sys.argv) > 2 else 10.0
        rest = sys.argv[3:]
        nu, window = 4e-5, 0.0
        for a in list(rest):
            if a.startswith("nu="):
                nu = float(a[3:])
                rest.remove(a)
            elif a.startswith("window="):
                window = float(a[7:])
                rest.remove(a)
        names = rest or ["fp32", "fp16"]
        res = {"case": "prop", "revolutions": revs, "nu_finest": nu, "window": f"last {window:.0%}" if window > 0 else "last revolution"}
        for nm in names:
            st, pert = storage_of(nm)
            res[nm] = run_prop(st, revs, nu_finest=nu, perturbed=pert, window=window)
        if "fp64" in res:
            ref = res["fp64"]
            for nm in names:
                if nm != "fp64":
                    res[nm]["thrust_rel_err"] = abs(res[nm]["thrust"] / ref["thrust"] - 1.0)
                    res[nm]["torque_rel_err"] = abs(res[nm]["torque"] / ref["torque"] - 1.0)
        print(json.dumps(res))
        return
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else (20000 if which == "arm" else 2000)
    storages = sys.argv[3:] or ["fp32", "fp16", "bf16"]
    make = (lambda s: arm_les(s)) if which == "arm" else (lambda s: sphere_re40(s, debug_dump=False))
    print(json.dumps(compare(which, make, steps, storages), default=float))


if __name__ == "__main__":
    main()
