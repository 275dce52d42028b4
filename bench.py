"""Benchmark of the PFEM-2 particle path on B200.

Workload: 3D duct [0,8]x[0,1]^2, 128x32x32 Q1 hexes (131,072 cells), 27
particles per cell on a 3x3x3 reference grid (3,538,944 particles), max 2
per cell part, 3 sub-steps, dt = 2e-3, u = 16 y(1-y) z(1-z).  The nodal
velocity sequence stands in for the FEM step: V_k alternates between V and
0.9 V, and step k runs correct(V_k, V_{k-1}), so every step applies a +-10 %
velocity correction and particle velocities stay of the order of V, as in a
solver run.  A step is one time step of the
reference loop (src/pfem2solver.cpp:162-164): correct + move (3 sub-steps,
relocation, count correction) + project, over every particle.

value   : FP32 form, particle-steps/s, nodal velocities resident on the device
e2e     : FP32 form through the host C ABI (pfem2gpu_correct/move/project
          with pinned host vectors; H2D of V and Vold, D2H of the projected V
          inside the timed region)
fp64    : the plain FP64 form, same workload, device-resident
roofline: the dominant kernel (advect) against measured HBM bandwidth
adjoint : the differentiated window (20 steps, checkpoints every 5) and its
          adjoint on the same particles, both forms: forward and backward
          time, their ratio, and the gradient along the inflow amplitude
          against FP64 central differences

`--impl reference` times the CPU restatement of the reference's particle
path (the reference itself needs deal.II/Trilinos/MPI, absent here) on all
host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s FP32 vs FP64 form at <=1e-4 rel L2; HBM GB/s; bwd/fwd time"
UNIT = "particle-steps/s"
WORKLOAD = "3D duct 128x32x32 Q1 hexes, 27 ppc (3,538,944 particles), max 2/part, 3 sub-steps, dt 2e-3"

# Algorithmic bytes per particle of the advect kernel (3D): read cell u32 +
# xi[3] + v[3], write xi[3] + v[3] + key u32 + slot u32.
ADVECT_BYTES = {"fp32": 4 + 12 + 12 + 12 + 12 + 4 + 4, "fp64": 4 + 24 * 3 + 24 * 3 + 4 + 4}
# ... of the write pass (FP32, 3D): read key u32 + id u32 + moved xi[3] + v[3],
# write cell u32 + id u32 + xi[3] + v[3]; plus the cell's projection partials
# (32 floats = 128 B per cell, 27 particles per cell: ~5 B per particle).
WRITE_BYTES = {"fp32": 4 + 4 + 12 + 12 + 4 + 4 + 12 + 12 + 5}
# Per particle-step, whole step (compulsory passes 5s + 8, s = 4 + 2*dim*w).
STEP_BYTES = {"fp32": 5 * (4 + 24) + 8, "fp64": 5 * (4 + 48) + 8}
# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# two main kernels, from one ncu capture at time step 11 of this workload with
# the L2 not flushed between kernels (profiles/duct_fp32_step_traffic.md).
TRAFFIC_WRITE = 244.2e6  # bytes per launch (116.1 MB read + 128.1 MB written)
TRAFFIC_ADVECT = 222.6e6  # bytes per launch (123.7 MB read + 98.9 MB written)


def reduce_over_ranks(ms, particle_steps, world, device):
    """Whole-job figures of N replicas: the slowest rank's time (max) and the
    particle-steps of all ranks (sum).  Every rank calls it once, in the same
    place."""
    if world <= 1:
        return float(ms), float(particle_steps)
    import torch

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ps = torch.tensor([float(particle_steps)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(ps)
    return float(t.item()), float(ps.item())


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self, busy_mhz=None):
        rows = []
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        mx = max(r[1] for r in rows)
        load = [r for r in rows if r[0] > 0.5 * mx] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in load), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


WORKLOADS = {
    "duct": WORKLOAD,
    "cube": "3D perturbed cube [0,2pi]^3, 80^3 Q1 hexes (interior vertices moved by up to +-0.1 h, seed 0), "
            "64 ppc (32,768,000 particles), max 2/part, 3 sub-steps, dt 1e-3, u = (sin x cos y cos z, "
            "-cos x sin y cos z, 0)",
}
WORKLOADS["turek"] = ("2D channel 2.2x0.41 with a cylinder of radius 0.05 at (0.2, 0.2), synthetic Turek-type "
                      "unstructured mesh of 64,512 Q1 quads, 16 ppc (1,032,192 particles), max 2/part, 3 sub-steps, "
                      "dt 5e-4, parabolic inflow Umax 1.5, zero on the walls and the cylinder")
ADJOINT_K = {"duct": 20, "cube": 10, "turek": 20}


def build_case(name="duct"):
    from pfem2dealii_b200 import mesh as M
    from pfem2dealii_b200.handler import ParticleParams

    if name == "turek":
        m = M.turek_channel(96, 48, 480)
        V = M.field_at_dofs(m, M.cylinder_inflow(1.5))
        prm = ParticleParams(particles_per_cell=(4, 4), max_particles_per_cell_part=2,
                             particle_integration_steps=3, time_step=5e-4)
        return m, V, 0.9 * V, prm
    if name == "cube":
        m = M.perturbed_cube(80, amplitude=0.1, seed=0)
        V = M.field_at_dofs(m, M.taylor_green_3d())
        prm = ParticleParams(particles_per_cell=(4, 4, 4), max_particles_per_cell_part=2,
                             particle_integration_steps=3, time_step=1e-3)
        return m, V, 0.9 * V, prm
    m = M.hyper_rectangle((0.0, 0.0, 0.0), (8.0, 1.0, 1.0), (128, 32, 32), "duct")
    V = M.field_at_dofs(m, M.duct_profile(1.0))
    prm = ParticleParams(particles_per_cell=(3, 3, 3), max_particles_per_cell_part=2,
                         particle_integration_steps=3, time_step=2e-3)
    return m, V, 0.9 * V, prm


def timed_device_run(handler_cls, m, V, Vold, prm, precision, steps, warmup, torch, profile=False,
                     alternate=True):
    """Seed, warm up, then time `steps` device-resident steps with CUDA events
    on the handler's stream.  alternate: step k runs with (V_k, V_{k-1}) where
    V_k alternates between V and Vold; otherwise (V, Vold) every step."""
    g = handler_cls(m.dim, prm, precision)
    g.initialize_maps(m)
    dev = torch.device("cuda:0")
    dV = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
    dVo = torch.from_numpy(np.ascontiguousarray(Vold)).to(dev)
    dout = torch.empty_like(dV)
    g.seed_particles_device(dV)
    stream = torch.cuda.ExternalStream(g.stream_handle())
    pairs = [(dVo, dV), (dV, dVo)] if alternate else [(dV, dVo)] * 2
    k = [0]

    def step():
        a, b = pairs[k[0] & 1]
        k[0] += 1
        if profile:  # per-kernel events: the separate calls, launched eagerly
            g.correct_particle_velocity_device(a, b)
            g.move_particles_device(None)
            g.project_particle_fields_device(dout)
        else:  # one CUDA graph per step
            g.step_device(a, b, dout)

    for _ in range(warmup):
        step()
    g.synchronize()
    if profile:
        g.profile(True)
    s0 = g.stats()
    l0 = g.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    s1 = g.stats()
    res = {"ms": ms, "particle_steps": s1["particle_steps"] - s0["particle_steps"],
           "launches": g.launch_count() - l0, "n_particles": s1["n_particles"], "stats": s1,
           "V": dout.cpu().numpy()}
    if profile:
        res["profile"] = g.profile_report()
        g.profile(False)
    g.close()
    return res


def timed_output(handler_cls, m, V, Vold, prm, torch, steps=5, reps=5):
    """output_particle_solution's data for the workload after a few steps:
    packing on the device plus one pinned device-to-host copy (best of reps,
    CUDA events on the handler's stream)."""
    g = handler_cls(m.dim, prm, "fp32")
    g.initialize_maps(m)
    dev = torch.device("cuda:0")
    dV = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
    dVo = torch.from_numpy(np.ascontiguousarray(Vold)).to(dev)
    out = torch.empty_like(dV)
    g.seed_particles_device(dV)
    for k in range(steps):
        a, b = ((dVo, dV), (dV, dVo))[k & 1]
        g.step_device(a, b, out)
    g.synchronize()
    n = g.stats()["n_particles"]
    dout = torch.empty(2 * m.dim * n, dtype=torch.float32, device=dev)
    hout = torch.empty(2 * m.dim * n, dtype=torch.float32).pin_memory()
    stream = torch.cuda.ExternalStream(g.stream_handle())
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.pack_output_device(dout)
        with torch.cuda.stream(stream):
            hout.copy_(dout, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1)
        best = t if best is None else min(best, t)
    # release the buffers used on the handler's stream before the stream goes
    del hout, dout
    torch.cuda.synchronize()
    g.close()
    return {"particles": n, "ms": best, "bytes": 8 * m.dim * n}


def timed_mesh_setup(handler_cls, m, prm, torch, reps=3):
    """initialize_maps on the workload mesh through the C ABI with the vertex
    maps built on the device (host wall clock to the end of the call, best of
    reps; it ends with the map arrays resident)."""
    best = None
    for _ in range(reps):
        g = handler_cls(m.dim, prm, "fp32")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.initialize_maps(m)
        g.synchronize()
        t = (time.perf_counter() - t0) * 1e3
        best = t if best is None else min(best, t)
        g.close()
    return {"cells": m.n_cells, "vertices": m.n_verts, "ms": best}


def timed_fem(handler_cls, m, V, torch, reps=5):
    """The solver step's three Q1 systems (volume terms) on device vectors:
    CUDA-event time of one assembly each (best of reps), the FP64 oracle's
    time for the pressure system on one host thread, and the bytes the
    device passes must move (local values written and read back, the
    matrices and right-hand sides written, the cell geometry and DoF vectors
    read)."""
    from oracle import oracle as O

    g = handler_cls(m.dim, ParticleParamsDefault(m.dim), "fp64")
    g.initialize_maps(m)
    rp, cols = g.fem_pattern()
    nnz, nd, nc, nv = len(cols), m.n_dofs, m.n_cells, 1 << m.dim
    dev = torch.device("cuda:0")
    dU = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
    dU2 = 0.9 * dU
    dP = torch.zeros(nd, dtype=torch.float64, device=dev)
    stream = torch.cuda.ExternalStream(g.stream_handle())
    out = {"nnz": nnz, "cells": nc}
    for name, system in (("prediction", 0), ("pressure", 1), ("correction", 2)):
        nm = m.dim if system == 0 else 1
        ns = 1 if system == 1 else m.dim
        dA = torch.empty(nm * nnz, dtype=torch.float64, device=dev)
        dr = torch.empty(ns * nd, dtype=torch.float64, device=dev)
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g._ck(g.L.pfem2gpu_fem_assemble_device(g.h, system, 1.0, 0.01, 1e-3, dU.data_ptr(), dU2.data_ptr(),
                                                    dP.data_ptr(), dA.data_ptr(), dr.data_ptr()))
            e1.record(stream)
            e1.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        moved = (2 * nc * nv * nm * nv + nc * nv * ns * 2 + nm * nnz + ns * nd + nc * nv * m.dim
                 + 2 * m.dim * nd) * 8 + (nc * nv + nnz + 2 * nd) * 4
        out[name] = {"ms": best, "bytes": moved, "gbs": moved / (best / 1000.0) / 1e9}
        del dA, dr
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    O.fem_assemble(m, O.FEM_PRESSURE, 1.0, 0.01, 1e-3, U=V, pattern=(rp, cols))
    out["oracle_pressure_ms_1_thread"] = (time.perf_counter() - t0) * 1e3
    del dU, dU2, dP
    torch.cuda.synchronize()
    g.close()
    return out


def ParticleParamsDefault(dim):
    from pfem2dealii_b200.handler import ParticleParams

    return ParticleParams(particles_per_cell=(2,) * dim)


def timed_host_run(handler_cls, m, V, Vold, prm, precision, steps, warmup, torch):
    """The same steps through the host C ABI with pinned vectors: H2D of V
    and Vold, D2H of the projected velocity, every step."""
    g = handler_cls(m.dim, prm, precision)
    g.initialize_maps(m)
    hV = torch.from_numpy(np.ascontiguousarray(V)).pin_memory()
    hVo = torch.from_numpy(np.ascontiguousarray(Vold)).pin_memory()
    hout = torch.empty_like(hV).pin_memory()
    L, h = g.L, g.h
    import ctypes as C

    pV, pVo, pout = C.c_void_p(hV.data_ptr()), C.c_void_p(hVo.data_ptr()), C.c_void_p(hout.data_ptr())
    g._ck(L.pfem2gpu_seed(h, pV))
    pairs = [(pVo, pV), (pV, pVo)]
    k = [0]

    def step():
        a, b = pairs[k[0] & 1]
        k[0] += 1
        g._ck(L.pfem2gpu_correct(h, a, b))
        g._ck(L.pfem2gpu_move(h, None))
        g._ck(L.pfem2gpu_project(h, pout))

    for _ in range(warmup):
        step()
    stream = torch.cuda.ExternalStream(g.stream_handle())
    s0 = g.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    s1 = g.stats()
    g.close()
    nbytes = V.size * 8
    return {"ms": ms, "particle_steps": s1["particle_steps"] - s0["particle_steps"], "h2d": 2 * nbytes,
            "d2h": nbytes}


def timed_window(handler_cls, m, V, Vold, prm, precision, K, C, torch, pre_steps=5, reps=3, n_probe=64):
    """The differentiated window on the workload: K steps of correct + move
    (count correction left out) + projection, then its adjoint for
    J = sum over n_probe DoFs of (U - T)^2, T = U + 0.01.  Forward and
    backward are timed with CUDA events on the handler's stream (best of
    reps).  Also the directional derivative along the inflow amplitude
    (V -> a V at the DoFs where V != 0) against central differences of the
    FP64 form's window (h = 1e-6)."""
    g = handler_cls(m.dim, prm, precision)
    g.initialize_maps(m)
    dev = torch.device("cuda:0")
    dV = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
    dVo = torch.from_numpy(np.ascontiguousarray(Vold)).to(dev)
    out = torch.empty_like(dV)
    g.seed_particles_device(dV)
    for k in range(pre_steps):
        a, b = ((dVo, dV), (dV, dVo))[k & 1]
        g.step_device(a, b, out)
    g.synchronize()
    n = g.stats()["n_particles"]
    stream = torch.cuda.ExternalStream(g.stream_handle())
    U = torch.empty_like(dV)
    gv0 = torch.empty((n, 3), dtype=torch.float64, device=dev)
    gV, gVo = torch.empty_like(dV), torch.empty_like(dV)
    rng = np.random.default_rng(7)
    g.window_forward_device(K, C, dV, dVo, None, U)
    g.synchronize()
    Un = U.cpu().numpy()
    probe = rng.choice(np.where(np.all(np.isfinite(Un), 0))[0], n_probe, replace=False)
    T = Un[:, probe] + 0.01
    gUn = np.zeros_like(Un)
    gUn[:, probe] = 2.0 * (Un[:, probe] - T)
    gU = torch.from_numpy(gUn).to(dev)
    fwd, bwd = [], []
    for _ in range(reps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(stream)
        g.window_forward_device(K, C, dV, dVo, None, U)
        e1.record(stream)
        g.window_backward_device(gU, gv0, gV, gVo)
        e2.record(stream)
        e2.synchronize()
        fwd.append(e0.elapsed_time(e1))
        bwd.append(e1.elapsed_time(e2))
    gVn = gV.cpu().numpy()
    g.close()
    return {"fwd_ms": min(fwd), "bwd_ms": min(bwd), "bwd_over_fwd": min(bwd) / min(fwd), "particles": n,
            "dJ_da": float(np.sum(gVn * V)), "probe": probe, "T": T}


def fd_inflow(handler_cls, m, V, Vold, prm, K, C, probe, T, torch, pre_steps=5, h=1e-6):
    """Central difference of J along V -> (1 + t) V with the FP64 form."""
    g = handler_cls(m.dim, prm, "fp64")
    g.initialize_maps(m)
    dev = torch.device("cuda:0")
    dV = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
    dVo = torch.from_numpy(np.ascontiguousarray(Vold)).to(dev)
    out = torch.empty_like(dV)
    g.seed_particles_device(dV)
    for k in range(pre_steps):
        a, b = ((dVo, dV), (dV, dVo))[k & 1]
        g.step_device(a, b, out)
    js = []
    for t in (h, -h):
        U = g.window_forward_device(K, C, (1.0 + t) * dV, dVo)
        g.synchronize()
        Un = U.cpu().numpy()
        js.append(float(np.sum((Un[:, probe] - T) ** 2)))
    g.close()
    return (js[0] - js[1]) / (2 * h)


def adjoint_report(handler_cls, m, V, Vold, prm, torch, K=20, C=5, forms=("fp32", "fp64")):
    """K-step window + adjoint on the workload, both forms, with the
    directional derivative along the inflow amplitude against FP64 central
    differences (one form given: timing only)."""
    rep = {"steps": K, "checkpoint_every": C, "objective": "sum over 64 DoFs of (U - T)^2"}
    for form in forms:
        r = timed_window(handler_cls, m, V, Vold, prm, form, K, C, torch)
        rep[form] = {k: r[k] for k in ("fwd_ms", "bwd_ms", "bwd_over_fwd", "particles", "dJ_da")}
        if form == forms[0]:
            probe, T = r["probe"], r["T"]
    if len(forms) == 1:
        return rep
    fd = fd_inflow(handler_cls, m, V, Vold, prm, K, C, probe, T, torch)
    for form in ("fp32", "fp64"):
        rep[form]["fd_rel_err"] = abs(rep[form]["dJ_da"] - fd) / abs(fd)
    rep["fd_dJ_da"] = fd
    return rep


def cpu_baseline(m, V, Vold, prm, budget_s=20.0, max_steps=None, warmup=0, workload=WORKLOAD):
    """The FP64 CPU restatement (reference removal order) on all host cores,
    on the full workload; `warmup` untimed steps, then steps until the time
    budget is spent."""
    from oracle.oracle import ORDER_VECTOR, Oracle

    cores = os.cpu_count() or 1
    o = Oracle(m, prm.particles_per_cell, prm.max_particles_per_cell_part, prm.particle_integration_steps,
               prm.time_step, removal_order=ORDER_VECTOR, n_threads=cores)
    o.seed(V)
    pairs = [(Vold, V), (V, Vold)]
    for k in range(warmup):
        o.step(*pairs[k & 1])
    done, ps, t = 0, 0, 0.0
    while t < budget_s and (max_steps is None or done < max_steps):
        n = o.stats()["n_particles"]
        t0 = time.perf_counter()
        o.step(*pairs[(warmup + done) & 1])
        t += time.perf_counter() - t0
        ps += n
        done += 1
    return {"value": ps / t, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done} time step(s) of the full {workload} workload, FP64 restatement, "
                      f"{cores} threads (not the reference binary: deal.II/Trilinos/MPI absent)",
            "steps": done, "seconds": t}


def form_difference(V64, V32, particles64, particles32):
    """FP32 vs FP64 projected velocity: the relative L2 error, and how much of
    it sits on DoFs where the two forms' particle sets parted (a count
    correction or part decision taken differently moves such a DoF by the
    order of the velocity itself): DoFs off by more than 1e-3 of max |V|,
    and the relative L2 error over the other DoFs."""
    m = np.isfinite(V64) & np.isfinite(V32)
    d = np.where(m, np.abs(V64 - V32), 0.0)
    scale = float(np.max(np.abs(V64[m]))) if m.any() else 1.0
    off = (d > 1e-3 * scale).any(axis=0)
    keep = m & ~off[None, :]
    rest = float(np.linalg.norm((V64 - V32)[keep]) / np.linalg.norm(V64[keep])) if keep.any() else 0.0
    return {"rel_l2": rel_l2(V64, V32), "dofs_off_by_1e-3_of_max": int(off.sum()), "dofs": int(V64.shape[1]),
            "rel_l2_other_dofs": rest, "particles_fp64": int(particles64), "particles_fp32": int(particles32)}


def config2_report(handler_cls, torch, steps=200, warmup=3):
    """The 2D obstacle workload (the reference's Turek-type case): both forms
    over the same velocity sequence, and their projected-velocity error."""
    m, V, Vold, prm = build_case("turek")
    r32 = timed_device_run(handler_cls, m, V, Vold, prm, "fp32", steps, warmup, torch)
    r64 = timed_device_run(handler_cls, m, V, Vold, prm, "fp64", steps, warmup, torch)
    v32 = r32["particle_steps"] / (r32["ms"] / 1000.0)
    v64 = r64["particle_steps"] / (r64["ms"] / 1000.0)
    return {"workload": WORKLOADS["turek"], "steps": steps, "particles": r32["n_particles"],
            "fp32": {"value": v32, "ms_per_step": r32["ms"] / steps},
            "fp64": {"value": v64, "ms_per_step": r64["ms"] / steps}, "fp32_over_fp64": v32 / v64,
            "fp32_vs_fp64_rel_l2": rel_l2(r64["V"], r32["V"]), "tolerance": 1e-4, "unit": UNIT,
            "difference": form_difference(r64["V"], r32["V"], r64["n_particles"], r32["n_particles"])}


def rel_l2(a, b):
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.linalg.norm((a - b)[m]) / np.linalg.norm(a[m]))


def load_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    m, V, Vold, prm = build_case()
    budget = 60.0
    warm = min(args.warmup, 3)  # CPU steps: a few suffice to settle caches and threads
    cb = cpu_baseline(m, V, Vold, prm, budget_s=budget, max_steps=max(1, args.steps), warmup=warm)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": cb["steps"], "warmup": warm, "ms_per_step": 1000.0 * cb["seconds"] / cb["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "form": "fp64 CPU restatement"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="duct",
                    help="duct: the headline configuration; cube: the 32.8 M-particle perturbed-cube stress case; "
                         "turek: the 2D obstacle case (1.03 M particles)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="time the differentiated window and its adjoint only (prints one JSON object)")
    ap.add_argument("--only", choices=["fp32", "fp64"], default=None,
                    help="run one device-resident pass of one form and print its timing (profiling runs)")
    ap.add_argument("--fem-only", action="store_true",
                    help="time the three FEM system assemblies on the workload mesh only (prints one JSON object)")
    ap.add_argument("--e2e", action="store_true",
                    help="with --only: also the same steps through the host ABI (pinned H2D/D2H each step)")
    ap.add_argument("--kernels", action="store_true",
                    help="with --only: also the per-kernel times of a profiled run (CUDA events)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch

    rank, world, local = env_rank()
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    from pfem2dealii_b200.handler import ParticleHandler

    m, V, Vold, prm = build_case(args.workload)
    workload = WORKLOADS[args.workload]
    gpu_index = torch.cuda.current_device()
    if args.adjoint_only:
        forms = (args.only,) if args.only else ("fp32", "fp64")
        print(json.dumps(adjoint_report(ParticleHandler, m, V, Vold, prm, torch, K=ADJOINT_K[args.workload],
                                        forms=forms)), flush=True)
        return 0
    if args.fem_only:
        print(json.dumps(timed_fem(ParticleHandler, m, V, torch)), flush=True)
        return 0
    if args.only:
        r = timed_device_run(ParticleHandler, m, V, Vold, prm, args.only, args.steps, args.warmup, torch)
        out = {"form": args.only, "ms_per_step": r["ms"] / args.steps,
               "value": r["particle_steps"] / (r["ms"] / 1000.0), "unit": UNIT}
        if args.e2e:
            re = timed_host_run(ParticleHandler, m, V, Vold, prm, args.only, args.steps, args.warmup, torch)
            out["e2e"] = {"value": re["particle_steps"] / (re["ms"] / 1000.0), "ms_per_step": re["ms"] / args.steps}
        if args.kernels:
            rp = timed_device_run(ParticleHandler, m, V, Vold, prm, args.only, args.steps, args.warmup, torch,
                                  profile=True)
            out["kernel_ms_per_step"] = {k: v[0] / args.steps for k, v in sorted(rp["profile"].items())}
        print(json.dumps(out), flush=True)
        return 0

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # FP32 form, device-resident: the headline value
    barrier()
    with ClockSampler(gpu_index) as clk:
        r32 = timed_device_run(ParticleHandler, m, V, Vold, prm, "fp32", args.steps, args.warmup, torch)
        barrier()
    ms = r32["ms"]
    ms, total_ps = reduce_over_ranks(ms, r32["particle_steps"], world, "cuda")
    value = total_ps / (ms / 1000.0)
    # FP64 form (plain) and the FP32 vs FP64 error after the same steps
    r64 = timed_device_run(ParticleHandler, m, V, Vold, prm, "fp64", args.steps, args.warmup, torch)
    v64 = r64["particle_steps"] / (r64["ms"] / 1000.0)
    err = rel_l2(r64["V"], r32["V"])
    # the same comparison with Vold = 0.9 V held fixed (velocities grow by 0.1 V per step)
    f32 = timed_device_run(ParticleHandler, m, V, Vold, prm, "fp32", args.steps, args.warmup, torch, alternate=False)
    f64 = timed_device_run(ParticleHandler, m, V, Vold, prm, "fp64", args.steps, args.warmup, torch, alternate=False)
    err_fixed = rel_l2(f64["V"], f32["V"])
    # kernel-level timing pass (per-launch CUDA events)
    rp = timed_device_run(ParticleHandler, m, V, Vold, prm, "fp32", args.steps, args.warmup, torch, profile=True)
    prof = rp["profile"]
    adv_ms, adv_n = prof.get("advect", [0.0, 1])
    wr_ms, wr_n = prof.get("write", [0.0, 1])
    per_launch_particles = rp["particle_steps"] / max(adv_n, 1)
    peak, peak_kind = load_peak()
    achieved = ADVECT_BYTES["fp32"] * per_launch_particles / (adv_ms / adv_n / 1000.0) / 1e9
    achieved_w = WRITE_BYTES["fp32"] * per_launch_particles / (wr_ms / wr_n / 1000.0) / 1e9
    step_ms_prof = sum(v[0] for v in prof.values()) / args.steps
    # end to end through the host ABI
    re2e = timed_host_run(ParticleHandler, m, V, Vold, prm, "fp32", args.steps, args.warmup, torch)
    # output_particle_solution's data: packing on the device + one copy
    outp = timed_output(ParticleHandler, m, V, Vold, prm, torch)
    mesh_setup = timed_mesh_setup(ParticleHandler, m, prm, torch)
    cfg2 = config2_report(ParticleHandler, torch) if args.workload == "duct" else None
    fem = timed_fem(ParticleHandler, m, V, torch) if args.workload == "duct" else None
    # the differentiated window (K = 20, checkpoints every 5) and its adjoint
    adj = adjoint_report(ParticleHandler, m, V, Vold, prm, torch, K=ADJOINT_K[args.workload])
    e2e_value = re2e["particle_steps"] / (re2e["ms"] / 1000.0)
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0
    cb = None
    if not args.no_cpu_baseline:
        cb = cpu_baseline(m, V, Vold, prm, budget_s=args.cpu_budget, max_steps=3, workload=workload)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload, "form": "fp32", "particles": r32["n_particles"],
                   "l2": "inputs larger than L2 (particle arrays ~300 MB per form)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "fp64": {"value": v64, "unit": UNIT, "ms_per_step": r64["ms"] / args.steps, "dtype": "f64",
                 "fp32_over_fp64": value / v64},
        "fp32_vs_fp64_rel_l2": {"projected_velocity": err, "tolerance": 1e-4,
                                "steps": args.warmup + args.steps,
                                "fixed_vold_0.9v": err_fixed,
                                "fixed_vold_0.9v_difference": form_difference(f64["V"], f32["V"], f64["n_particles"],
                                                                              f32["n_particles"])},
        "step_effective_gbs": STEP_BYTES["fp32"] * value / 1e9,
        "roofline": {"bound": "hbm", "kernel": "k_write<3,float>", "achieved": achieved_w, "peak": peak,
                     "unit": "GB/s", "frac": achieved_w / peak, "traffic": TRAFFIC_WRITE,
                     "bytes_per_particle": WRITE_BYTES["fp32"], "peak_source": peak_kind,
                     "launch_ms": wr_ms / wr_n,
                     "advect": {"kernel": "k_advect32<3,1>", "achieved": achieved, "frac": achieved / peak,
                                "bytes_per_particle": ADVECT_BYTES["fp32"], "launch_ms": adv_ms / adv_n,
                                "traffic": TRAFFIC_ADVECT},
                     "step": {"achieved": STEP_BYTES["fp32"] * value / 1e9,
                              "frac": STEP_BYTES["fp32"] * value / 1e9 / peak,
                              "bytes_per_particle_step": STEP_BYTES["fp32"]}},
        "kernel_ms_per_step": {k: v[0] / args.steps for k, v in sorted(prof.items())},
        "profiled_ms_per_step": step_ms_prof,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": re2e["h2d"],
                "d2h_bytes_per_step": re2e["d2h"], "ms_per_step": re2e["ms"] / args.steps},
        "adjoint": adj,
        "output_pack": {"particles": outp["particles"], "ms": outp["ms"], "bytes": outp["bytes"],
                        "gbs": outp["bytes"] / (outp["ms"] / 1000.0) / 1e9},
        "mesh_setup": mesh_setup,
        "obstacle_2d": cfg2,
        "fem_assembly": fem,
        "gpu_launches": r32["launches"],
        "clocks": clk.summary(),
        "stats": {k: r32["stats"][k] for k in ("n_particles", "lost", "removed", "seeded", "searched",
                                               "fallback64", "error_flags")},
    }
    if cb:
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
