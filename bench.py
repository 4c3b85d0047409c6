#!/usr/bin/env python
"""Throughput of the D3Q19 LES time step on one B200 (or N replicas).

Workload: the 512x256x256 arm case (simlab_b200.cases.arm_les): regularized
D3Q19 with Smagorinsky LES Cs=0.17, Re 1e5 on the arm width, Bouzidi walls,
wind-tunnel faces with sponges and absorbing layers.  A step is one lattice
time step over all 33.5 M cells (faces, wall cells with the fused FP64
force reduction, bulk collide-stream).

Metric: MLUPS (all lattice cells x steps / s, as crates/cfd/examples/bench.rs)
for FP16-stored populations (the headline `value`), beside the same engine's
FP32 and BF16 storage and their fraction of the measured HBM copy bandwidth.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs its own replica of
the case: the step has no data exchange across replicas ("replicas only").
On one GPU the line also carries the gray-level adjoint's time against one
forward solve (`adjoint`) and the three-level D3Q27 throughput.
--impl reference times the reference's update restated on the CPU (the
oracle; the reference itself is Rust + wgpu/Metal and cannot run here) on
bounded samples of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MLUPS (D3Q19 LES arm 512x256x256, FP16-stored populations)"
UNIT = "MLUPS"
DTYPE = "f32 arithmetic, fp16 storage"
# Arithmetic per lattice update of the two collision kernels, FP16 storage,
# from ncu's counters (profiles/opcode_mix_k_bulk_tma_k27_step_fp16.md):
# flops = FADD + FMUL + 2 FFMA thread instructions executed with the
# predicate on, per cell; instructions = executed warp instructions x 32 per
# cell (smsp__inst_executed; D3Q19 includes the copy pipeline's wait loops).  FP32 peak: 148 SMs x 128 FP32
# lanes x 2 flops x clock; issue peak: 148 SMs x 4 schedulers x 32 threads x clock.
ALU_PER_LUP = {"d3q19_bulk_fp16": {"flops": 78.93 + 40.80 + 2 * 63.71, "instr": 410.8},
               "d3q27_step_fp16": {"flops": 163.76 + 82.50 + 2 * 135.74, "instr": 1012.4}}


def alu_line(lups: dict, sm_mhz: float) -> dict:
    """FP32 throughput and issue rate of the collision kernels from their
    measured update rates (updates/s) and the per-update counts above."""
    f = sm_mhz * 1e6
    peak_fp32, peak_issue = 148 * 128 * 2 * f, 148 * 4 * 32 * f
    out = {"fp32_peak_tflops": round(peak_fp32 / 1e12, 2), "issue_peak_tinst_s": round(peak_issue / 1e12, 2), "sm_mhz": sm_mhz,
           "source": "profiles/opcode_mix_k_bulk_tma_k27_step_fp16.md"}
    for k, ups in lups.items():
        c = ALU_PER_LUP[k]
        out[k] = {"flops_per_lup": round(c["flops"], 1), "instr_per_lup": c["instr"], "glups": round(ups / 1e9, 2),
                  "fp32_tflops": round(c["flops"] * ups / 1e12, 2), "fp32_frac": round(c["flops"] * ups / peak_fp32, 3),
                  "issue_frac": round(c["instr"] * ups / peak_issue, 3)}
    return out


CONFIG = {"workload": "D3Q19 regularized + Smagorinsky LES (Cs 0.17), arm 200x12x8 + cylinder r10 h14, 512x256x256, "
                      "u 0.05, Re 1e5, Bouzidi walls, wind-tunnel faces + sponges",
          "storage": "fp16 (f - w) x 32768, stochastic rounding",
          "l2": "inputs larger than L2 (1.41 GB of populations per replica)"}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profile(storage_name: str):
    """DRAM bytes per k_bulk launch from the committed ncu summary, if any."""
    f = ROOT / "profiles" / f"k_bulk_tma_{storage_name}_arm_512x256x256.md"
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", f.read_text())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = os.environ.get("SIMLAB_BENCH_BACKEND") or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
        else:  # the host-side plumbing on CPU (tests): replicas, barrier, max over ranks
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(v: float, ws: int) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_storage(storage, steps, warmup, ws, with_profile):
    """Device time of `steps` resident time steps, CUDA events on the lattice's stream."""
    import torch

    from simlab_b200.cases import arm_les
    from simlab_b200.lbm import Lattice

    st, vox = arm_les(storage)
    lat = Lattice(st, vox)
    stream = torch.cuda.ExternalStream(lat.stream)
    lat.advance(warmup)
    lat.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if with_profile:
        lat.profile(2)  # two events around the bulk kernel per timed step
    barrier(ws)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0.record()
    lat.advance(steps)
    with torch.cuda.stream(stream):
        e1.record()
    lat.synchronize()
    torch.cuda.synchronize()
    barrier(ws)
    ms = e0.elapsed_time(e1)
    kt = lat.kernel_times() if with_profile else None
    if with_profile:
        # the face / wall / bulk split from 20 more steps with all four events
        # per step, after the timed region
        lat.profile(True)
        lat.advance(20)
        lat.synchronize()
        kt["split"] = lat.kernel_times()
        lat.profile(False)
    mass, bad = lat.mass()
    info = {"cells": st.cells(), "nrec": lat.nrec, "nface": lat.nface, "mass": mass, "nonfinite": bad}
    return lat, ms, kt, info


def e2e_time(lat, steps):
    """Through the C-ABI call a caller makes (lbm_run with host buffers), in
    the batches the reference's study loop passes to Lattice::run
    (tunnel.rs:1072: 0.25 x 2800e6 / cells steps, clamped to 16..4096): every
    step's StepIn goes host->device with its launch and every step's force and
    moment come back to the host before the call returns."""
    from simlab_b200.lbm import STEP_DTYPE, steps_array

    batch = int(min(max(0.25 * 2800e6 / lat.setup.cells(), 16), 4096))
    lat.synchronize()
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        m = min(batch, steps - done)
        f = lat.run(steps_array(m))
        done += m
    t1 = time.perf_counter()
    assert np.all(np.isfinite(f))
    return (t1 - t0) * 1e3, STEP_DTYPE.itemsize, 6 * 8, batch


ARM_FIXTURE = ROOT / "oracle" / "fixtures" / "arm_les_512x256x256.npz"
CPU_SLAB = 8  # z-planes per CPU sample step


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def cpu_oracle_sample(steps=None, warmup: int = 1, budget_s: float = 12.0):
    """The oracle (the reference's update restated in C++, OpenMP over all host
    cores) on the 512x256x256 arm case, loaded from its frozen inputs
    (oracle/fixtures, written by oracle/make_arm_fixture.py) so that nothing of
    the engine is imported or loaded.  One sample step is the collide-stream
    over a slab of CPU_SLAB z-planes of the full lattice, cycling through z;
    `steps` of them, or as many as fit in budget_s.  Both CPU figures (the
    bench line's cpu_baseline and the --impl reference arm) come from here,
    so they time the same work."""
    import oracle

    cores = oracle.set_threads(os.cpu_count() or 1)
    lat = oracle.OracleLattice.from_fixture(ARM_FIXTURE)
    nx, ny, nz = (int(d) for d in lat.setup.dims)
    slab = CPU_SLAB
    z = 0
    for _ in range(warmup):
        lat.step_slab(z, z + slab)
        z = (z + slab) % nz
    n = 0
    t0 = time.perf_counter()
    while (n < steps) if steps is not None else (time.perf_counter() - t0 < budget_s):
        lat.step_slab(z, z + slab)
        z = (z + slab) % nz
        n += 1
    dt = time.perf_counter() - t0
    lat.close()
    v = nx * ny * slab * n / dt / 1e6
    return {"value": round(v, 3), "unit": UNIT, "cores": cores, "kind": "port", "cpu": cpu_model(), "nproc": os.cpu_count(),
            "sample": f"{n} slabs of {nx}x{ny}x{slab} cells of the 512x256x256 arm lattice (FP16 storage) in {dt:.1f} s"}, n, dt


def adjoint_ratio():
    """The gray-level adjoint on its design case (simlab_b200.cases.gray_design:
    192x96x96 D3Q19 BGK, 64x48x48 design box, drag over steps 500-1000,
    checkpoint every 50, FP32): device time of one forward solve (1000 steps)
    and of lbm_backward, with every segment recomputed from its checkpoint and
    with the trailing moments kept when HBM holds them."""
    import torch

    from simlab_b200.cases import gray_design
    from simlab_b200.gray import GrayLattice
    from simlab_b200.lbm import Storage

    st, gam, spec = gray_design(Storage.FP32)
    lat = GrayLattice(st, gam)
    stream = torch.cuda.ExternalStream(lat.stream)
    lat.run(100)
    lat.reset()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record()
    lat.run(spec.steps)
    with torch.cuda.stream(stream):
        e1.record()
    torch.cuda.synchronize()
    fwd = e0.elapsed_time(e1)
    out = {"workload": "gray design 192x96x96, box 64x48x48, drag over steps 500-1000, checkpoint every 50, fp32",
           "forward_ms": round(fwd, 3), "forward_mlups": round(192 * 96 * 96 * spec.steps / fwd / 1e3, 1)}
    for rc in (True, False):
        spec.recompute = rc
        J, g = lat.backward(spec)
        t = lat.backward_times()
        tot = t["forward_ms"] + t["recompute_ms"] + t["reverse_ms"]
        out["recompute_all" if rc else "memory_sized"] = {"backward_ms": round(tot, 3), "ratio": round(tot / fwd, 3),
                                                           **{k: round(v, 3) for k, v in t.items()}}
    out["adjoint_over_forward"] = out["recompute_all"]["ratio"]
    # bytes per cell and step (FP32): forward 19 loads + 19 stores + a; the
    # recomputing step also writes rho - 1 and j; the reverse step reads and
    # writes lambda and reads the moments and a
    cells = 192 * 96 * 96
    hbm, _ = peaks()
    out["bytes_per_cell"] = {"forward": 156, "recompute": 172, "reverse": 172}
    out["hbm_frac"] = {"forward": round(156 * cells * spec.steps / (fwd * 1e-3) / 1e9 / hbm, 3),
                       "reverse": round(172 * cells * spec.steps / (out["recompute_all"]["reverse_ms"] * 1e-3) / 1e9 / hbm, 3)}
    out["objective"] = J
    lat.close()
    return out


def d3q27_levels():
    """MLUPS (finest-step definition, tunnel.rs:800-804) of the three-level
    D3Q27 lattice with the refinement layout of the propeller case (coarse
    256x128x128, each box 0.63 of its parent per axis), FP32 and FP16."""
    import torch

    from simlab_b200.lbm import FaceBc, Storage
    from simlab_b200.mlattice import LevelBox, MultiLattice, MultiSetup

    res = {}
    for storage, nl in ((Storage.FP32, 3), (Storage.FP16, 3), (Storage.FP16, 1)):
        F = FaceBc
        s = MultiSetup(dims0=[256, 128, 128], faces=[F.VELOCITY] + [F.OPEN] * 5, nu0=0.001, u_inf=[0.05, 0, 0], u_init=[0.05, 0, 0],
                       sponge=[0, 16, 8, 8, 8, 8], sponge_tau=1.0, sponge_sigma=0.1, total_pressure_inlet=True, storage=storage)
        for l in range(1, nl):
            d = s.dims(l - 1)
            n = [int(d[k] * 0.63) for k in range(3)]
            s.boxes.append(LevelBox(lo=[(d[k] - n[k]) // 2 for k in range(3)], n=n))
        g = MultiLattice(s)
        g.advance(16)
        g.synchronize()
        stream = torch.cuda.ExternalStream(g.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record()
        g.advance(64)
        with torch.cuda.stream(stream):
            e1.record()
        g.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        cells = g.level_cells()
        lups = sum(c * 2 ** l for l, c in enumerate(cells)) / 2 ** (len(cells) - 1) * 64
        if nl == 1:
            res["single_level_fp16"] = round(lups / ms / 1e3, 1)
        else:
            res[storage.name.lower()] = round(lups / ms / 1e3, 1)
            res["cells"] = cells
        g.close()
    return res


def c5_throughput(steps: int = 40, warmup: int = 4):
    """The at-scale throughput case: D3Q19 LES with FP16 populations on a
    1024x512x512 lattice (268,435,456 cells) around the arm scaled x2, MLUPS
    of the step and the bulk kernel's fraction of the measured copy
    bandwidth (80 B per cell)."""
    import torch

    from simlab_b200.cases import arm_les
    from simlab_b200.lbm import Lattice, Storage

    t0 = time.perf_counter()
    st, vox = arm_les(Storage.FP16, scale=2)
    t1 = time.perf_counter()
    lat = Lattice(st, vox)
    lat.synchronize()
    t2 = time.perf_counter()
    stream = torch.cuda.ExternalStream(lat.stream)
    lat.advance(warmup)
    lat.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record()
    lat.advance(steps)
    with torch.cuda.stream(stream):
        e1.record()
    lat.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    lat.profile(True)  # the bulk kernel's own time, events around it on the next steps
    lat.advance(10)
    lat.synchronize()
    kt = lat.kernel_times()
    lat.profile(False)
    mass, bad = lat.mass()
    cells = st.cells()
    bulk_ms = kt["bulk_ms"] / max(kt["steps"], 1)
    hbm, _ = peaks()
    res = {"dims": list(st.dims), "cells": cells, "mlups": round(cells * steps / ms / 1e3, 1), "ms_per_step": round(ms / steps, 4),
           "bulk_ms": round(bulk_ms, 4), "bulk_hbm_frac": round(80.0 * cells / (bulk_ms * 1e-3) / 1e9 / hbm, 4),
           "nonfinite": int(bad), "memory_gb": round(lat.info().memory_bytes / 1e9, 2),
           "setup_s": {"voxelize_host": round(t1 - t0, 3), "create": round(t2 - t1, 3)}}
    lat.close()
    return res


def c5_adjoint():
    """The at-scale adjoint (simlab_b200.cases.prop_gray_band): the rotor held
    still as a gray body on one 384x192x192 D3Q19 level, gradient of the mean
    torque over steps 301-600 with respect to the 3-cell band around it.
    FP16-stored forward with the FP32 adjoint, moments kept where they fit in
    device memory and the rest recomputed from checkpoints; the FP32-stored
    run alongside for the gradient's agreement."""
    import torch

    from simlab_b200.cases import prop_gray_band
    from simlab_b200.gray import GrayLattice
    from simlab_b200.lbm import Storage

    out = {"workload": "rotor R60 as a gray body, 384x192x192, torque over steps 301-600, 3-cell design band, checkpoint every 50"}
    grads = {}
    for storage in (Storage.FP16, Storage.FP32):
        st, gam, band, spec = prop_gray_band(storage)
        lat = GrayLattice(st, gam)
        stream = torch.cuda.ExternalStream(lat.stream)
        lat.run(20)
        lat.reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record()
        lat.run(spec.steps)
        with torch.cuda.stream(stream):
            e1.record()
        torch.cuda.synchronize()
        fwd = e0.elapsed_time(e1)
        J, g = lat.backward(spec)
        t = lat.backward_times()
        tot = t["forward_ms"] + t["recompute_ms"] + t["reverse_ms"]
        grads[storage] = g[band]
        out[storage.name.lower()] = {"forward_solve_ms": round(fwd, 3), "forward_mlups": round(st.cells() * spec.steps / fwd / 1e3, 1),
                                     "backward_ms": round(tot, 3), "ratio": round(tot / fwd, 3), "torque": J, "band_cells": int(band.sum()),
                                     "first_pass_ms": round(t["forward_ms"], 3), "recompute_ms": round(t["recompute_ms"], 3),
                                     "reverse_ms": round(t["reverse_ms"], 3)}
        lat.close()
    a, b = grads[Storage.FP16], grads[Storage.FP32]
    out["fp16_vs_fp32_grad_rel_l2"] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    return out


def c3_rotor(steps: int = 256, warmup: int = 32):
    """C3's workload: the three-level D3Q27 rotor case (simlab_b200.cases.
    prop_refined: coarse 256x128x128 + 8.1 M + 16.0 M cells, the two-blade
    rotor of radius 60 finest cells re-voxelized on the finest level every
    finest step), spinning at full speed; MLUPS by the finest-step definition
    of tunnel.rs:800-804, device time of `steps` finest steps through
    lbm_multi_run (force readback included), FP32 and FP16 storage."""
    import torch

    from simlab_b200.cases import prop_refined, spin_schedule
    from simlab_b200.lbm import Storage
    from simlab_b200.mlattice import MultiLattice

    res = {}
    for storage in (Storage.FP32, Storage.FP16):
        s, geo, om = prop_refined(storage)
        g = MultiLattice(s, geo)
        sched = spin_schedule(warmup + steps, om, 1)
        g.run(sched[:warmup])
        stream = torch.cuda.ExternalStream(g.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record()
        f = g.run(sched[warmup:])
        with torch.cuda.stream(stream):
            e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        cells = g.level_cells()
        lups = sum(c * 2 ** l for l, c in enumerate(cells)) / 2 ** (len(cells) - 1) * steps
        res[storage.name.lower()] = {"mlups": round(lups / ms / 1e3, 1), "ms_per_finest_step": round(ms / steps, 4),
                                     "records": int(g.nrec), "finite": bool(np.all(np.isfinite(f)))}
        g.close()
    res["cells"] = cells
    return res


def spin_overhead(steps: int = 100, warmup: int = 10):
    """A spinning part against the same part held still (the reference
    reports spinning runs taking 2.3x their estimate, crates/engine/src/wind.rs:
    537-543): the refined case's two-blade rotor (radius 40 cells) on one
    256x128x128 D3Q19 level, FP16 storage; spinning, every swept-box cell is a
    record and the GPU re-voxelizes the box every step.  Device time per step
    of each and their ratio."""
    import torch

    from simlab_b200.cases import rotor_tunnel, spin_schedule
    from simlab_b200.lbm import Lattice, Storage

    out = {}
    for spinning in (False, True):
        st, geo, om = rotor_tunnel(Storage.FP16, spinning=spinning)
        lat = Lattice(st, geo)
        sched = spin_schedule(warmup + steps, om if spinning else 0.0, 1)
        lat.run(sched[:warmup])
        stream = torch.cuda.ExternalStream(lat.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record()
        f = lat.run(sched[warmup:])
        with torch.cuda.stream(stream):
            e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out["spinning" if spinning else "static"] = {"ms_per_step": round(ms / steps, 4), "mlups": round(st.cells() * steps / ms / 1e3, 1),
                                                     "records": int(lat.nrec), "finite": bool(np.all(np.isfinite(f)))}
        lat.close()
    out["spin_over_static"] = round(out["spinning"]["ms_per_step"] / out["static"]["ms_per_step"], 3)
    return out


def voxelizer_times():
    """The static voxelizer on the host cores (voxel.cpp, OpenMP) and on the
    GPU (lbm_voxelize_static_gpu) for a sphere of radius 100 cells (81,920
    triangles) in a 222^3 lattice, D3Q19 and D3Q27 links: seconds per call
    (the GPU's after one warm-up call) and whether the results are identical."""
    from simlab_b200.lbm import voxelize_static
    from simlab_b200.shapes import sphere

    v, t = sphere([110.3, 110.7, 110.1], 100.0, 6)
    out = {"triangles": int(len(t)), "lattice_dims": [222, 222, 222]}
    for lat in (19, 27):
        t0 = time.perf_counter()
        a = voxelize_static(v, t, [222] * 3, lat)
        t_cpu = time.perf_counter() - t0
        voxelize_static(v, t, [222] * 3, lat, device=True)
        t0 = time.perf_counter()
        b = voxelize_static(v, t, [222] * 3, lat, device=True)
        t_gpu = time.perf_counter() - t0
        same = bool(np.array_equal(a.solid, b.solid) and np.array_equal(a.walls.view(np.uint32), b.walls.view(np.uint32)))
        out[f"d3q{lat}"] = {"cpu_s": round(t_cpu, 4), "gpu_s": round(t_gpu, 4), "walls": int(len(b.walls)), "solid": int(len(b.solid)),
                            "identical": same}
    out["cpu_threads"] = os.cpu_count()
    return out


def run_reference(args, ws, rank):
    """The reference arm: the oracle on the host cores, rank 0 only, on the
    same workload, metric and config as the engine's line; each step one
    sample step of cpu_oracle_sample."""
    if rank != 0:
        return
    cb, n, dt = cpu_oracle_sample(steps=args.steps, warmup=args.warmup)
    v = cb["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / max(args.steps, 1), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE, "data": "synthetic", "config": CONFIG,
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-extras", action="store_true", help="skip the adjoint and D3Q27 measurements (launch-list captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local = dist_init()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    import torch

    from simlab_b200.cases import BYTES_PER_LUP
    from simlab_b200.lbm import Storage

    torch.cuda.set_device(local)
    hbm, peak_kind = peaks()
    results = {}
    clocks = None
    e2e = None
    for storage in (Storage.FP16, Storage.FP32, Storage.BF16):
        headline = storage == Storage.FP16
        sampler = ClockSampler(local) if headline else None
        if sampler:
            sampler.start()
        lat, ms, kt, info = time_storage(storage, args.steps, args.warmup, ws, with_profile=headline)
        if sampler:
            clocks = sampler.stop()
        ms_max = max_over_ranks(ms, ws)
        mlups = info["cells"] * args.steps * ws / (ms_max * 1e-3) / 1e6
        r = {"mlups": mlups, "ms_per_step": ms_max / args.steps, "info": info}
        if kt:
            r["kernel_times"] = kt
        if headline:
            e_ms, hb, db, e_batch = e2e_time(lat, args.steps)
            e_ms = max_over_ranks(e_ms, ws)
            e2e = {"value": round(info["cells"] * args.steps * ws / (e_ms * 1e-3) / 1e6, 3), "unit": UNIT, "h2d_bytes_per_step": hb,
                   "d2h_bytes_per_step": db, "steps_per_call": e_batch}
        lat.close()
        del lat
        results[storage] = r
        torch.cuda.synchronize()
    h = results[Storage.FP16]
    kt = h["kernel_times"]
    ks = kt.pop("split")
    bulk_ms = kt["bulk_ms"] / max(kt["steps"], 1)
    cells = h["info"]["cells"]
    alg_bytes = BYTES_PER_LUP[Storage.FP16] * cells
    achieved = alg_bytes / (bulk_ms * 1e-3) / 1e9
    traffic = traffic_from_profile("fp16")
    line = {
        "metric": METRIC,
        "value": round(h["mlups"], 3),
        "unit": UNIT,
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(h["ms_per_step"], 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": DTYPE,
        "data": "synthetic",
        "config": CONFIG,
        "parallelism": "replicas" if ws > 1 else "single GPU",
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "traffic": traffic, "kernel": "k_bulk_tma<fp16>", "bytes_per_lup": BYTES_PER_LUP[Storage.FP16],
                     "kernel_ms": round(bulk_ms, 5), "peak_source": peak_kind},
        "storages": {s.name.lower(): {"mlups": round(r["mlups"], 3), "ms_per_step": round(r["ms_per_step"], 5),
                                      "hbm_frac_step": round(BYTES_PER_LUP[s] * cells * r["mlups"] / cells / 1e3 / hbm, 4)}
                     for s, r in results.items()},
        "fp16_over_fp32": round(h["mlups"] / results[Storage.FP32]["mlups"], 3),
        "clocks": clocks,
        "e2e": e2e,
        "gpu_launches": int(kt["launches"]),
        "kernel_share": {k.removesuffix("_ms"): round(v / max(ks["faces_ms"] + ks["walls_ms"] + ks["bulk_ms"], 1e-12), 4)
                         for k, v in ks.items() if k.endswith("_ms")},
    }
    if ws == 1 and not args.no_extras:
        line["adjoint"] = adjoint_ratio()
        line["d3q27_three_levels_mlups"] = d3q27_levels()
        # the collision kernels' own update rates: the D3Q19 bulk kernel's
        # event-timed duration, the single-level D3Q27 lattice's step
        line["alu"] = alu_line({"d3q19_bulk_fp16": cells / (bulk_ms * 1e-3),
                                "d3q27_step_fp16": line["d3q27_three_levels_mlups"]["single_level_fp16"] * 1e6},
                               float((clocks or {}).get("sm_mhz") or 1965.0))
        line["c5_fp16_1024x512x512"] = c5_throughput()
        line["c5_adjoint"] = c5_adjoint()
        line["c3_rotor"] = c3_rotor()
        line["spin_overhead"] = spin_overhead()
        line["voxelizer"] = voxelizer_times()
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_oracle_sample(budget_s=12.0)[0]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
