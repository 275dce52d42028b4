"""Benchmark of the PFEM-2 particle path on B200.

Headline workload: 3D duct [0,8]x[0,1]^2, 128x32x32 Q1 hexes (131,072
cells), 27 particles per cell on a 3x3x3 reference grid (3,538,944
particles), max 2 per cell part, 3 sub-steps, dt = 2e-3, u = 16 y(1-y)
z(1-z).  The nodal velocities follow the solver's data flow
(src/pfem2solver.cpp:162-165 with fem_step copying the projection into the
old solution, src/pfem2fem.cpp:523-524): V, the FEM solution, is held fixed
(the FEM solve is not part of the particle path) and every step corrects with
Vold = the previous step's projection.  A step is one time step of the
reference loop: correct + move (3 sub-steps, relocation, count correction) +
project, over every particle.

Line keys beyond the base contract:
  fp64     the plain FP64 form on the same workload and steps; the FP32/FP64
           throughput ratio and the relative L2 difference of the final
           projected velocities
  roofline the write pass (the step's longest kernel) against the measured HBM
           bandwidth; the advect pass and the whole step as fractions too
  e2e      the same steps through the host C ABI: one upload of V and one
           download of the projection per step (pinned host memory)
  cfg2     the 2D obstacle case on the reference's Turek mesh (Mesh3.unv,
           60,450 quads, 16 ppc, N(0, 0.01) initial velocity noise, 200 steps
           at dt 5e-4): both forms and their difference after the timed
           steps; per_step: the difference after each of 210 steps of the
           two forms run side by side (median, 95th percentile, maximum,
           the step of the maximum, steps above 1e-4)
  cfg4     the differentiated window (K = 20, checkpoints every 5) on the
           same case: forward/backward time of both forms and the gradient
           along the inflow amplitude against FP64 central differences (64
           probe DoFs off the no-slip walls, drawn from the FP64 window and
           used by both forms)
  cfg5     the perturbed 80^3 cube (32.8 M particles): both forms, their
           difference, and the K = 10 window's backward/forward ratio
Longer per-kernel, output, mesh-setup and FEM-assembly figures go to stderr
as one JSON object.

`--impl reference` times the CPU restatement of the reference's particle
path (the reference itself needs deal.II/Trilinos/MPI, absent here) on all
host cores, with the same data flow.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s FP32 vs FP64 form at <=1e-4 rel L2; HBM GB/s; bwd/fwd time"
UNIT = "particle-steps/s"
WORKLOAD = "3D duct 128x32x32 Q1 hexes, 27 ppc (3,538,944 particles), max 2/part, 3 sub-steps, dt 2e-3"
MESH3 = os.path.join(ROOT, "tests", "golden", "Mesh3.tgz")

# Algorithmic bytes per particle of the advect kernel (3D): read cell u32 +
# xi[3] + v[3], write xi[3] + v[3] + key u32 + slot u32.
ADVECT_BYTES = {"fp32": 4 + 12 + 12 + 12 + 12 + 4 + 4, "fp64": 4 + 24 * 3 + 24 * 3 + 4 + 4}
# ... of the write pass (FP32, 3D): read key u32 + id u32 + moved xi[3] + v[3],
# write cell u32 + id u32 + xi[3] + v[3]; plus the cell's projection partials
# (32 floats = 128 B per cell, 27 particles per cell: ~5 B per particle).
WRITE_BYTES = {"fp32": 4 + 4 + 12 + 12 + 4 + 4 + 12 + 12 + 5}
# Per particle-step, whole step (compulsory passes 5s + 8, s = 4 + 2*dim*w).
STEP_BYTES = {"fp32": 5 * (4 + 24) + 8, "fp64": 5 * (4 + 48) + 8}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one write-pass
# launch on this workload, from an ncu capture taken apart from the timed
# run (a profiler cannot run inside it); the line names it as such.
TRAFFIC_WRITE = 203.3e6
TRAFFIC_SRC = "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_write launch (time step 4), separate capture"


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


def sig(x, n=4):
    """x rounded to n significant digits (keeps the line short)."""
    if x is None or not np.isfinite(x) or x == 0:
        return x
    return float(f"{x:.{n}g}")


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

    def summary(self):
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


class Case:
    """A workload: mesh, the fixed FEM velocity V, particle parameters and
    the initial velocity noise (standard deviation; 0 = none)."""

    def __init__(self, name, mesh, V, prm, noise, text):
        self.name, self.mesh, self.V, self.prm, self.noise, self.text = name, mesh, V, prm, noise, text


def build_case(name="duct", cube_n=80):
    from pfem2dealii_b200 import mesh as M
    from pfem2dealii_b200.handler import ParticleParams

    if name == "turek":
        m = M.read_unv_native(MESH3)
        V = M.field_at_dofs(m, M.cylinder_inflow(1.5))
        prm = ParticleParams(particles_per_cell=(4, 4), max_particles_per_cell_part=2,
                             particle_integration_steps=3, time_step=5e-4)
        return Case(name, m, V, prm, 0.01, f"2D Turek channel, Mesh3.unv ({m.n_cells} Q1 quads), 16 ppc, "
                                           "max 2/part, 3 sub-steps, dt 5e-4, Umax 1.5, N(0,0.01) noise")
    if name == "cube":
        m = M.perturbed_cube(cube_n, amplitude=0.1, seed=0)
        V = M.field_at_dofs(m, M.taylor_green_3d())
        prm = ParticleParams(particles_per_cell=(4, 4, 4), max_particles_per_cell_part=2,
                             particle_integration_steps=3, time_step=1e-3)
        return Case(name, m, V, prm, 0.0, f"3D cube [0,2pi]^3 {cube_n}^3 hexes perturbed +-0.1h, 64 ppc, "
                                          "max 2/part, 3 sub-steps, dt 1e-3, Taylor-Green u")
    m = M.hyper_rectangle((0.0, 0.0, 0.0), (8.0, 1.0, 1.0), (128, 32, 32), "duct")
    V = M.field_at_dofs(m, M.duct_profile(1.0))
    prm = ParticleParams(particles_per_cell=(3, 3, 3), max_particles_per_cell_part=2,
                         particle_integration_steps=3, time_step=2e-3)
    return Case(name, m, V, prm, 0.0, WORKLOAD)


def noisy_particles(case, handler_cls):
    """The seeded particles (FP64 form) with N(0, noise) added to every
    velocity component, drawn in id order from a seeded generator."""
    g = handler_cls(case.mesh.dim, case.prm, "fp64")
    g.initialize_maps(case.mesh)
    g.seed_particles(case.V)
    P = g.particles()
    nid = g.stats()["next_id"]
    g.close()
    rng = np.random.default_rng(0)
    order = np.argsort(P["id"])
    P["v"] = P["v"].copy()
    P["v"][order] += rng.normal(0.0, case.noise, size=P["v"].shape)
    return P, nid


def start(handler_cls, case, precision, torch, start_particles=None, dV=None):
    """A handler with the case's particles (seeded, or given) and its first
    projection, the Vold of the first step."""
    g = handler_cls(case.mesh.dim, case.prm, precision)
    g.initialize_maps(case.mesh)
    if dV is None:
        dV = torch.from_numpy(np.ascontiguousarray(case.V)).cuda()
    g.seed_particles_device(dV)
    if start_particles is not None:
        g.set_particles(*start_particles)
    dout = torch.empty_like(dV)
    g.project_particle_fields_device(dout)
    return g, dV, dout


def timed_device_run(handler_cls, case, precision, steps, warmup, torch, profile=False, start_particles=None):
    """Warm up, then time `steps` device-resident steps with CUDA events on
    the handler's stream: one graph per step (correct from the last
    projection + move + project), or with profile the separate calls, each
    launch timed."""
    import ctypes as C

    g, dV, dout = start(handler_cls, case, precision, torch, start_particles)
    stream = torch.cuda.ExternalStream(g.stream_handle())
    pV, pout = C.c_void_p(dV.data_ptr()), C.c_void_p(dout.data_ptr())

    def step():
        if profile:
            g.correct_particle_velocity_from_projection_device(dV)
            g.move_particles_device(None)
            g.project_particle_fields_device(dout)
        else:  # the C ABI call itself, on the handle's stream (ordered by the synchronisations around the loop)
            g._ck(g.L.pfem2gpu_step_device(g.h, pV, None, pout))

    g.synchronize()
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


def timed_host_run(handler_cls, case, precision, steps, warmup, torch):
    """The same steps through the host C ABI with pinned vectors: every step
    uploads V (correct_from_projection: Vold is the last projection, already
    on the device) and downloads the projection."""
    import ctypes as C

    m = case.mesh
    g = handler_cls(m.dim, case.prm, precision)
    g.initialize_maps(m)
    hV = torch.from_numpy(np.ascontiguousarray(case.V)).pin_memory()
    hout = torch.empty_like(hV).pin_memory()
    L, h = g.L, g.h
    pV, pout = C.c_void_p(hV.data_ptr()), C.c_void_p(hout.data_ptr())
    g._ck(L.pfem2gpu_seed(h, pV))
    g._ck(L.pfem2gpu_project(h, pout))

    def step():
        g._ck(L.pfem2gpu_correct_from_projection(h, pV))
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
    nbytes = case.V.size * 8
    return {"ms": ms, "particle_steps": s1["particle_steps"] - s0["particle_steps"], "h2d": nbytes, "d2h": nbytes}


def timed_output(handler_cls, case, torch, steps=5, reps=5):
    """output_particle_solution's data after a few steps: packing on the
    device plus one pinned device-to-host copy (best of reps)."""
    g, dV, dout = start(handler_cls, case, "fp32", torch)
    for _ in range(steps):
        g.step_device(dV, None, dout)
    g.synchronize()
    n = g.stats()["n_particles"]
    dim = case.mesh.dim
    dpack = torch.empty(2 * dim * n, dtype=torch.float32, device="cuda")
    hpack = torch.empty(2 * dim * n, dtype=torch.float32).pin_memory()
    stream = torch.cuda.ExternalStream(g.stream_handle())
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.pack_output_device(dpack)
        with torch.cuda.stream(stream):
            hpack.copy_(dpack, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1)
        best = t if best is None else min(best, t)
    del hpack, dpack
    torch.cuda.synchronize()
    g.close()
    return {"particles": n, "ms": best, "bytes": 8 * dim * n}


def timed_mesh_setup(handler_cls, case, torch, reps=3):
    """initialize_maps with the vertex maps built on the device (host wall
    clock to the end of the call, best of reps)."""
    best = None
    for _ in range(reps):
        g = handler_cls(case.mesh.dim, case.prm, "fp32")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.initialize_maps(case.mesh)
        g.synchronize()
        t = (time.perf_counter() - t0) * 1e3
        best = t if best is None else min(best, t)
        g.close()
    return {"cells": case.mesh.n_cells, "ms": best}


def timed_fem(handler_cls, case, torch, reps=5):
    """The solver step's three Q1 systems (volume terms) on device vectors:
    CUDA-event time of one assembly each (best of reps)."""
    from pfem2dealii_b200.handler import ParticleParams

    m = case.mesh
    g = handler_cls(m.dim, ParticleParams(particles_per_cell=(2,) * m.dim), "fp64")
    g.initialize_maps(m)
    rp, cols = g.fem_pattern()
    nnz, nd = len(cols), m.n_dofs
    dU = torch.from_numpy(np.ascontiguousarray(case.V)).cuda()
    dU2 = 0.9 * dU
    dP = torch.zeros(nd, dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(g.stream_handle())
    out = {"nnz": nnz}
    for name, system in (("prediction", 0), ("pressure", 1), ("correction", 2)):
        nm = m.dim if system == 0 else 1
        ns = 1 if system == 1 else m.dim
        dA = torch.empty(nm * nnz, dtype=torch.float64, device="cuda")
        dr = torch.empty(ns * nd, dtype=torch.float64, device="cuda")
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
        out[name + "_ms"] = best
        del dA, dr
    del dU, dU2, dP
    torch.cuda.synchronize()
    g.close()
    return out


def timed_window(handler_cls, case, precision, K, C, torch, start_particles=None, pre_steps=5, reps=3, n_probe=64,
                 probe=None):
    """The differentiated window after pre_steps steps: K steps of correct +
    move (count correction left out) + projection, then its adjoint for
    J = sum over n_probe DoFs of (U - T)^2, T = U + 0.01.  Forward and
    backward timed with CUDA events on the handler's stream (best of reps).
    Vold of the window is the last projection, as in the solver."""
    g, dV, dout = start(handler_cls, case, precision, torch, start_particles)
    for _ in range(pre_steps):
        g.step_device(dV, None, dout)
    g.synchronize()
    n = g.stats()["n_particles"]
    dVo = dout.clone()
    stream = torch.cuda.ExternalStream(g.stream_handle())
    U = torch.empty_like(dV)
    gv0 = torch.empty((n, case.mesh.dim), dtype=torch.float64, device="cuda")
    gV, gVo = torch.empty_like(dV), torch.empty_like(dV)
    rng = np.random.default_rng(7)
    g.window_forward_device(K, C, dV, dVo, None, U)
    g.synchronize()
    Un = U.cpu().numpy()
    # probes off the no-slip walls: a wall DoF sees the particles pinned
    # against the wall, whose positions move with V in steps of the FP64
    # position's rounding, which no finite difference resolves
    if probe is None:
        probe = rng.choice(np.where(np.all(np.isfinite(Un), 0) & np.any(case.V != 0, 0))[0], n_probe, replace=False)
    T = Un[:, probe] + 0.01
    gUn = np.zeros_like(Un)
    gUn[:, probe] = 2.0 * (Un[:, probe] - T)
    gU = torch.from_numpy(gUn).cuda()
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
    return {"fwd_ms": min(fwd), "bwd_ms": min(bwd), "particles": n, "dJ_da": float(np.sum(gVn * case.V)),
            "probe": probe, "T": T}


def fd_inflow(handler_cls, case, K, C, probe, T, torch, start_particles=None, pre_steps=5, h=1e-6):
    """Central difference of J along V -> (1 + t) V with the FP64 form."""
    g, dV, dout = start(handler_cls, case, "fp64", torch, start_particles)
    for _ in range(pre_steps):
        g.step_device(dV, None, dout)
    dVo = dout.clone()
    js = []
    for t in (h, -h):
        U = g.window_forward_device(K, C, (1.0 + t) * dV, dVo)
        g.synchronize()
        js.append(float(np.sum((U.cpu().numpy()[:, probe] - T) ** 2)))
    g.close()
    return (js[0] - js[1]) / (2 * h)


def adjoint_report(handler_cls, case, torch, K, C=5, start_particles=None):
    """Window + adjoint of both forms, with the directional derivative along
    the inflow amplitude against FP64 central differences."""
    rep = {"K": K, "C": C}
    probe = T = None
    for form in ("fp64", "fp32"):  # probes and target from the FP64 form
        r = timed_window(handler_cls, case, form, K, C, torch, start_particles, probe=probe)
        if probe is None:
            probe, T = r["probe"], r["T"]
        rep[form] = r
    fd = fd_inflow(handler_cls, case, K, C, probe, T, torch, start_particles)
    out = {"K": K, "C": C, "particles": rep["fp32"]["particles"]}
    for form in ("fp32", "fp64"):
        r = rep[form]
        out[form] = {"fwd_ms": sig(r["fwd_ms"]), "bwd_ms": sig(r["bwd_ms"]),
                     "bwd_fwd": sig(r["bwd_ms"] / r["fwd_ms"], 3), "fd_err": sig(abs(r["dJ_da"] - fd) / abs(fd), 2)}
    return out


def rel_l2(a, b):
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.linalg.norm((a - b)[m]) / np.linalg.norm(a[m]))


def both_forms(handler_cls, case, steps, warmup, torch, steps64=None, start_particles=None):
    """Both forms over the same steps: throughput, ratio, final difference."""
    r32 = timed_device_run(handler_cls, case, "fp32", steps, warmup, torch, start_particles=start_particles)
    r64 = timed_device_run(handler_cls, case, "fp64", steps, warmup, torch, start_particles=start_particles)
    v32 = r32["particle_steps"] / (r32["ms"] / 1e3)
    v64 = r64["particle_steps"] / (r64["ms"] / 1e3)
    return r32, r64, {"particles": r32["n_particles"], "steps": warmup + steps, "fp32": sig(v32), "fp64": sig(v64),
                      "ratio": sig(v32 / v64, 3), "rel_l2": sig(rel_l2(r64["V"], r32["V"]), 2)}


def lockstep_rel_l2(handler_cls, case, steps, torch, start_particles=None, tol=1e-4):
    """Both forms step by step side by side (untimed): the relative L2
    difference of the projected velocities after every step."""
    hs = [start(handler_cls, case, f, torch, start_particles) for f in ("fp64", "fp32")]
    errs = []
    for _ in range(steps):
        Vs = []
        for g, dV, dout in hs:
            g.step_device(dV, None, dout)
            g.synchronize()
            Vs.append(dout.cpu().numpy())
        errs.append(rel_l2(Vs[0], Vs[1]))
    for g, _, _ in hs:
        g.close()
    e = np.array(errs)
    return {"steps": steps, "median": sig(float(np.median(e)), 2), "p95": sig(float(np.percentile(e, 95)), 2),
            "max": sig(float(e.max()), 2), "argmax": int(e.argmax()) + 1, "n_over_tol": int((e > tol).sum())}


def cpu_baseline(case, budget_s=20.0, max_steps=None, warmup=0):
    """The FP64 CPU restatement (reference removal order) on all host cores,
    same data flow: `warmup` untimed steps, then steps until the time budget
    is spent."""
    from oracle.oracle import ORDER_VECTOR, Oracle

    cores = os.cpu_count() or 1
    prm = case.prm
    o = Oracle(case.mesh, prm.particles_per_cell, prm.max_particles_per_cell_part, prm.particle_integration_steps,
               prm.time_step, removal_order=ORDER_VECTOR, n_threads=cores)
    o.seed(case.V)
    Vold = o.project()
    for _ in range(warmup):
        Vold = o.step(case.V, Vold)
    done, ps, t = 0, 0, 0.0
    while t < budget_s and (max_steps is None or done < max_steps):
        n = o.stats()["n_particles"]
        t0 = time.perf_counter()
        Vold = o.step(case.V, Vold)
        t += time.perf_counter() - t0
        ps += n
        done += 1
    return {"value": ps / t, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done} step(s) of the full duct, FP64 restatement on {cores} threads "
                      "(reference not buildable: deal.II/Trilinos/MPI absent)",
            "steps": done, "seconds": t}


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
    case = build_case()
    cb = cpu_baseline(case, budget_s=120.0, max_steps=max(1, args.steps), warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": cb["steps"], "warmup": args.warmup, "ms_per_step": 1000.0 * cb["seconds"] / cb["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": "fp64 CPU restatement",
                       "velocity": "V fixed, Vold = previous projection"},
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
    ap.add_argument("--no-extra", action="store_true", help="headline workload only (no cfg2/cfg4/cfg5 reports)")
    ap.add_argument("--cube-n", type=int, default=80,
                    help="cells per edge of the cube workload (smaller for profiler captures; 80 = config 5)")
    ap.add_argument("--workload", choices=["duct", "cube", "turek"], default="duct",
                    help="with --only/--adjoint-only: duct (the headline), cube (32.8 M particles) or turek "
                         "(Mesh3.unv, 0.97 M particles)")
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
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    from pfem2dealii_b200.handler import ParticleHandler as H

    case = build_case(args.workload if (args.only or args.adjoint_only or args.fem_only) else "duct", args.cube_n)
    noisy = noisy_particles(case, H) if case.noise else None
    if args.adjoint_only:
        rep = adjoint_report(H, case, torch, K=10 if case.name == "cube" else 20, start_particles=noisy)
        print(json.dumps(rep), flush=True)
        return 0
    if args.fem_only:
        print(json.dumps(timed_fem(H, case, torch)), flush=True)
        return 0
    if args.only:
        r = timed_device_run(H, case, args.only, args.steps, args.warmup, torch, start_particles=noisy)
        out = {"form": args.only, "workload": case.text, "ms_per_step": r["ms"] / args.steps,
               "value": r["particle_steps"] / (r["ms"] / 1000.0), "unit": UNIT}
        if args.e2e:
            re = timed_host_run(H, case, args.only, args.steps, args.warmup, torch)
            out["e2e"] = {"value": re["particle_steps"] / (re["ms"] / 1000.0), "ms_per_step": re["ms"] / args.steps}
        if args.kernels:
            rp = timed_device_run(H, case, args.only, args.steps, args.warmup, torch, profile=True,
                                  start_particles=noisy)
            out["kernel_ms_per_step"] = {k: v[0] / args.steps for k, v in sorted(rp["profile"].items())}
        print(json.dumps(out), flush=True)
        return 0

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # FP32 form, device-resident: the headline value
    barrier()
    with ClockSampler(torch.cuda.current_device()) as clk:
        r32 = timed_device_run(H, case, "fp32", args.steps, args.warmup, torch)
        barrier()
    ms, total_ps = reduce_over_ranks(r32["ms"], r32["particle_steps"], world, "cuda")
    value = total_ps / (ms / 1000.0)
    # FP64 form (plain) and the FP32 vs FP64 difference after the same steps
    r64 = timed_device_run(H, case, "fp64", args.steps, args.warmup, torch)
    v64 = r64["particle_steps"] / (r64["ms"] / 1000.0)
    err = rel_l2(r64["V"], r32["V"])
    # kernel-level timing pass (per-launch CUDA events)
    rp = timed_device_run(H, case, "fp32", args.steps, args.warmup, torch, profile=True)
    prof = rp["profile"]
    adv_ms, adv_n = prof.get("advect", [0.0, 1])
    wr_ms, wr_n = prof.get("write", [0.0, 1])
    per_launch = rp["particle_steps"] / max(adv_n, 1)
    peak, peak_kind = load_peak()
    achieved_a = ADVECT_BYTES["fp32"] * per_launch / (adv_ms / adv_n / 1000.0) / 1e9
    achieved_w = WRITE_BYTES["fp32"] * per_launch / (wr_ms / wr_n / 1000.0) / 1e9
    # end to end through the host ABI
    re2e = timed_host_run(H, case, "fp32", args.steps, args.warmup, torch)
    e2e_value = re2e["particle_steps"] / (re2e["ms"] / 1000.0)
    details = {"kernel_ms_per_step": {k: sig(v[0] / args.steps) for k, v in sorted(prof.items())},
               "stats_fp32": {k: r32["stats"][k] for k in ("n_particles", "lost", "removed", "seeded", "searched",
                                                            "fallback64", "error_flags")}}
    extra = {}
    if not args.no_extra and world == 1:
        details["output_pack"] = timed_output(H, case, torch)
        details["mesh_setup"] = timed_mesh_setup(H, case, torch)
        details["fem_assembly"] = timed_fem(H, case, torch)
        # config 2: the reference's Turek mesh with noisy initial velocities
        t2 = build_case("turek")
        p2 = noisy_particles(t2, H)
        _, _, extra["cfg2"] = both_forms(H, t2, 200, 3, torch, start_particles=p2)
        extra["cfg2"]["mesh"] = f"Mesh3.unv {t2.mesh.n_cells} quads"
        extra["cfg2"]["per_step"] = lockstep_rel_l2(H, t2, 210, torch, start_particles=p2)
        # config 4: the window and its adjoint on the same case
        extra["cfg4"] = adjoint_report(H, t2, torch, K=20, start_particles=p2)
        del t2, p2
        # config 5: the perturbed 80^3 cube
        c5 = build_case("cube")
        _, _, extra["cfg5"] = both_forms(H, c5, 10, 3, torch)
        a5 = adjoint_report(H, c5, torch, K=10)
        extra["cfg5"]["adj"] = {"K": 10, "fp32_bwd_fwd": a5["fp32"]["bwd_fwd"], "fp32_fwd_ms": a5["fp32"]["fwd_ms"],
                                "fd_err": a5["fp32"]["fd_err"]}
        del c5
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0
    cb = None
    if not args.no_cpu_baseline:
        cb = cpu_baseline(case, budget_s=args.cpu_budget, max_steps=3)
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
        "gpu_launches": r32["launches"],
        "config": {"workload": WORKLOAD, "form": "fp32", "velocity": "V fixed, Vold = previous projection",
                   "l2": "inputs > L2 (particle arrays ~0.5 GB)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": re2e["h2d"],
                "d2h_bytes_per_step": re2e["d2h"], "ms_per_step": sig(re2e["ms"] / args.steps)},
        "roofline": {"bound": "hbm", "kernel": "k_write<3,float>", "achieved": sig(achieved_w), "peak": peak,
                     "unit": "GB/s", "frac": sig(achieved_w / peak, 3), "traffic": TRAFFIC_WRITE,
                     "traffic_src": TRAFFIC_SRC, "peak_src": peak_kind, "bytes_per_particle": WRITE_BYTES["fp32"],
                     "launch_ms": sig(wr_ms / wr_n),
                     "advect": {"achieved": sig(achieved_a), "frac": sig(achieved_a / peak, 3),
                                "launch_ms": sig(adv_ms / adv_n)},
                     "step_frac": sig(STEP_BYTES["fp32"] * value / 1e9 / peak, 3)},
    }
    if cb:
        line["cpu_baseline"] = {k: (sig(cb[k]) if k == "value" else cb[k])
                                for k in ("value", "unit", "cores", "kind", "sample")}
    line["fp64"] = {"value": sig(v64), "ms_per_step": sig(r64["ms"] / args.steps), "fp32_over_fp64": sig(value / v64, 3),
                    "rel_l2": sig(err, 2), "tol": 1e-4}
    line.update(extra)
    print(json.dumps(details), file=sys.stderr, flush=True)
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
