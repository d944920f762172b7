#!/usr/bin/env python
"""Throughput of one solver step on a seeded synthetic sparse grid, on 1..N GPUs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload shell512|box64|plume256|fire512|fire1024] [--forces]
                    [--precision mixed|fp32]

A step is one pass of the hot path over the grid: the SOP operator chain
HNanoAdvect + HNanoAdvectVelocity + HNanoProjectNonDivergent (scalars and velocity advected
along one MacCormack trace, divergence, pressure solve to a relative FP64 Poisson residual of
1e-5, gradient subtraction), through the C ABI of libhns.so. The metric is active
voxel-steps/s. --precision mixed (default): BF16 velocity, FP16 density, FP64 iterative
refinement around FP16 red-black inner solves; the FP32 forms (plain red-black SOR, and the
same refinement with FP32 inner solves) are measured in the same run at the same residual. Under torchrun every rank runs an independent replica of the workload
(the solver does not shard a grid across GPUs), so scaling is weak.

--impl reference times the reference's own CPU implementation of the same step (its
src/Cuda/Kernel.cu kernels compiled as host C++, oracle/_ref, all host threads) on a
bounded sample of the same workload: every launch of the step runs an evenly spaced subset
of its thread blocks, with the red-black iteration count the GPU solve needed.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

# Workloads: the grid, the step parameters and the red-black iteration count the FP32 solve
# needs to reach the tolerance on it (the reference arm runs that fixed count: its operator
# takes an iteration count, not a tolerance).
WORKLOADS = {
    "shell512": dict(desc="512^3 box, 16-voxel band (+ leaf half-diagonal) around a seeded radius-200 sphere, "
                          "fields: value-noise density, value-noise velocity in (-1,1)",
                     # omega_refined / inner: the refinement's inner SOR factor and iterations per outer step,
                     # the fastest to 1e-5 in a sweep of 1.85-1.96 x 16-90 (they also serve the FP32 refinement).
                     # omega: plain FP32 SOR, the fastest that reaches 1e-5 (1.84 and above stall near 1.2e-5).
                     # fp32_iterations: red-black iterations the plain FP32 GPU solve takes to 1e-5 on this grid
                     # (measured on the B200 with checks every 10); both CPU legs run exactly this count.
                     dx=0.1, dt=0.1, omega=1.82, omega_refined=1.92, inner=36, tolerance=1e-5, cap=3000, check_every=10,
                     fp32_iterations=470),
    "plume256": dict(desc="256^3 box, leaves inside 8 seeded spheres of radius 20-60",
                     dx=0.1, dt=1.0 / 24.0, omega=1.8, omega_refined=1.9, inner=30, tolerance=1e-5, cap=3000,
                     check_every=10, fp32_iterations=None),
}
RBGS_BYTES_PER_VOXEL = 12  # one fused red+black iteration: read p, read div, write p (FP32)
# The solve kernels' unit of work is a half-sweep (one colour): half an iteration's pass-model
# bytes, counted by the library's device counter of red-black sweeps that ran.
F32_HALF_SWEEP_BYTES = RBGS_BYTES_PER_VOXEL // 2
F16_HALF_SWEEP_BYTES = 3  # read e, read r, write e at 2 bytes each, halved
KERNELS = {("f32", "per-colour"): "rbgs_split_half_f32_kernel (FP32 solve, colour-split leaves, one launch per colour)",
           ("f16", "per-colour"): "rbgs_split_half_kernel (FP16 inner solve, colour-split leaves, one launch per colour)",
           ("f32", "persistent"): "rbgs_split_solve_kernel<float> (FP32 solve, colour-split leaves, persistent: one "
                                  "launch per run of half-sweeps between checks)",
           ("f16", "persistent"): "rbgs_split_solve_kernel<__half> (FP16 inner solve, colour-split leaves, persistent: "
                                  "one launch per inner solve)"}

# The fire step (HNS_Advance with the configurations' forces): the sparse plume runs it in FP32
# with a fixed 100 red-black iterations per step, the large sparse fire on BF16/FP16 storage with
# the refined solve to 1e-5. Forces: buoyancy alpha 0.1 (density) and beta 0.5 (temperature,
# ambient 0), vorticity confinement 0.3 with a one-voxel offset, the rate/heat burn (rate 0.5,
# heat 1.0, ignition 0), no gravity, no disturbance re-solve; sources of fuel 1.0 and heat 2.0 in
# a radius-10 sphere at the first sphere's centre (synth.fire_state).
FIRE = dict(alpha=0.1, beta=0.5, ambient=0.0, confinement=0.3, factor_scale=1.0, burn_rate=0.5, heat_release=1.0,
            ignition=0.0, source_radius=10.0, source_fuel=1.0, source_temperature=2.0)
FIRE_WORKLOADS = {
    "plume256": dict(desc="256^3 box, leaves inside 8 seeded spheres of radius 20-60; fields density, temperature, "
                          "fuel, flame and velocity (FP32); fire forces and sources; 100 red-black iterations per step",
                     dx=0.1, dt=1.0 / 24.0, iterations=100, precision="fp32", fp32_iterations=100),
    "fire512": dict(desc="512^3 box, leaves inside 32 seeded spheres of radius 15-60; fields density, temperature, "
                         "fuel, flame (FP16) and velocity (BF16); fire forces and sources; refined solve to 1e-5",
                    dx=0.1, dt=1.0 / 24.0, tolerance=1e-5, omega=1.9, omega_refined=1.95, inner=80, cap=6000,
                    check_every=20, precision="mixed", fp32_iterations=None),
    "fire1024": dict(desc="1024^3 box, leaves inside 32 seeded spheres of radius 30-120; fields density, temperature, "
                          "fuel, flame (FP16) and velocity (BF16); fire forces and sources; refined solve to 1e-5",
                     # omega_refined / inner: the fastest to 1e-5 in a sweep of 1.94-1.99 x 40-160 (mixed and FP32
                     # refinement alike); plain FP32 SOR stalls above 1e-5 on this grid at every omega of 1.9-1.98
                     # (1.8e-5 after 6000 iterations at 1.9), so its timing is reported only when it converges.
                     dx=0.1, dt=1.0 / 24.0, tolerance=1e-5, omega=1.9, omega_refined=1.97, inner=80, cap=6000,
                     check_every=20, precision="mixed", fp32_iterations=6000),
}


def measured_peak_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def apply_options(g, hl, args):
    """The library options the command line selects."""
    form = getattr(args, "split_solve", "per-colour")
    g.set_option(hl.OPT_SPLIT_SOLVE, hl.SPLIT_PERSISTENT if form == "persistent" else hl.SPLIT_PER_COLOUR)
    coarse = getattr(args, "coarse_solve", "cluster")
    g.set_option(hl.OPT_COARSE_SOLVE, hl.COARSE_CLUSTER if coarse == "cluster" else hl.COARSE_LAUNCHES)
    g.set_option(hl.OPT_L2_PERSIST, 0 if getattr(args, "no_l2_persist", False) else 1)


def profiled_traffic(workload: str, kind: str):
    """DRAM bytes per launch of the red-black kernel (kind f32 or split) from the committed ncu
    summary profiles/rbgs_<kind>_<workload>.md (line `dram_bytes_per_launch: <int>`), or None."""
    path = os.path.join(ROOT, "profiles", f"rbgs_{kind}_{workload}.md")
    try:
        with open(path) as fh:
            for line in fh:
                if line.strip().startswith("dram_bytes_per_launch:"):
                    return int(line.split(":", 1)[1].strip().split()[0])
    except (OSError, ValueError):
        pass
    return None


class ClockSampler:
    """SM clock and clock-event reasons sampled while the timed region runs: NVML polled every
    20 ms from a thread (the device matched by PCI bus id), else `nvidia-smi -lms 200`."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    PERIOD_S = 0.02

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None
        self.nvml = None
        self.sm = []
        self.smax = None
        self.reasons = set()
        self.halt = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.dev)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.nvml = (nv, h, {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                                 "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                                 "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                                 "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap})
            self._poll_once()
        except Exception:  # no NVML binding or no matching device: fall back to nvidia-smi
            self.nvml = None
        if self.nvml is not None:
            self.sm.clear()
            self.reasons.clear()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _poll_once(self):
        nv, h, bits = self.nvml
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
        mask = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        for name, bit in bits.items():
            if mask & bit:
                self.reasons.add(name)

    def _poll(self):
        while not self.halt.is_set():
            try:
                self._poll_once()
            except Exception:
                return
            self.halt.wait(self.PERIOD_S)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.halt.set()
            if self.thread:
                self.thread.join(timeout=2)
            try:
                self._poll_once()  # the state at the end of the timed region
            except Exception:
                pass
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml, 20 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(self.NAMES, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def dist_info():
    from hnanosolver_b200 import replicas

    r = replicas.ranks_from_env()
    return r.rank, r.world, r.local


def workload_config(args, wl, origins):
    """The workload-defining `config`, printed identically by both arms."""
    n = 512 * len(origins)
    return {"workload": args.workload, "description": wl["desc"], "voxels": n, "leaves": len(origins),
            "dt": wl["dt"], "dx": wl["dx"], "tolerance": wl["tolerance"],
            "residual": "relative FP64 Poisson residual ||b - L p|| / ||b||, b = div dx^2",
            "fp32_red_black_iterations": wl["fp32_iterations"],
            "l2": "inputs larger than L2 (%.0f MB of fields and solver state per GPU)" % (((12 + 4) * 2 + 8 + 16) * n / 1e6)}


def reference_arm(args, wl):
    """Reference CPU implementation of the step on a bounded sample (rank 0 only)."""
    rank, world, _ = dist_info()
    if rank != 0:
        return
    from hnanosolver_b200 import synth
    from oracle import binding

    ref = binding.RefOracle()
    cores = ref.lib.ref_num_threads()
    origins = synth.topology(args.workload)
    dens, vel = synth.noise_fields(origins, seed=0)
    g = ref.grid(synth.leaf_dense_coords(origins))
    iters = wl["fp32_iterations"]
    n = len(dens)
    blocks = (n + 255) // 256
    stride = max(1, blocks // 2048)
    ref.lib.ref_set_block_stride(stride)
    scratch = None
    for _ in range(args.warmup):
        scratch = g.plain_step(vel, [dens], wl["dt"], wl["dx"], iters, wl["omega"], scratch)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        scratch = g.plain_step(vel, [dens], wl["dt"], wl["dx"], iters, wl["omega"], scratch)
        times.append(time.perf_counter() - t0)
    ref.lib.ref_set_block_stride(1)
    sampled = (blocks + stride - 1) // stride * 256
    t = sum(times) / len(times)
    value = sampled / t
    sample = (f"every launch of the step over 1/{stride} of its 256-voxel blocks ({sampled} of {n} voxels), "
              f"{iters} red-black iterations, {args.steps} steps")
    line = {
        "impl": "reference", "metric": "active voxel-steps/s", "value": value, "unit": "voxel-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, wl, origins),
        "details": {"step": "the plain step in FP32 (advect velocity and density, divergence, red-black SOR from p = 0, "
                            "gradient subtraction)", "red_black_iterations": iters, "omega": wl["omega"]},
        "cpu_baseline": {"value": value, "unit": "voxel-steps/s", "cores": cores, "kind": "reference",
                         "sample": sample, "cpu": binding.cpu_model(), "library": os.path.basename(ref.path)},
        "e2e": {"value": value, "unit": "voxel-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(args, wl, iters):
    """The reference's CPU step on a bounded sample, for the cpu_baseline key of our line."""
    from hnanosolver_b200 import synth
    from oracle import binding

    ref = binding.RefOracle()
    origins = synth.topology(args.workload)
    dens, vel = synth.noise_fields(origins, seed=0)
    g = ref.grid(synth.leaf_dense_coords(origins))
    n = len(dens)
    blocks = (n + 255) // 256
    stride = max(1, blocks // 2048)
    ref.lib.ref_set_block_stride(stride)
    scratch = g.plain_step(vel, [dens], wl["dt"], wl["dx"], iters, wl["omega"])
    reps, t0 = 0, time.perf_counter()
    while reps < 3 and (reps == 0 or time.perf_counter() - t0 < 15.0):
        scratch = g.plain_step(vel, [dens], wl["dt"], wl["dx"], iters, wl["omega"], scratch)
        reps += 1
    t = (time.perf_counter() - t0) / reps
    ref.lib.ref_set_block_stride(1)
    sampled = (blocks + stride - 1) // stride * 256
    return {"value": sampled / t, "unit": "voxel-steps/s", "cores": ref.lib.ref_num_threads(), "kind": "reference",
            "sample": f"{reps} steps, every launch over 1/{stride} of its 256-voxel blocks ({sampled} of {n} voxels), "
                      f"{iters} red-black iterations", "cpu": binding.cpu_model()}


def field_error_vs_fp64(torch, origins, wl, vel_in, dens_in, vel_out, dens_out, dev):
    """Field error of one step's result against the same step in FP64 from the same stored
    inputs: MacCormack advection of velocity and density, then the projection with the exact
    solve (conjugate gradients to an FP64 residual of 1e-12). The checker is the torch FP64
    restatement tests/fp64_box.py on a dense box holding the grid's active voxels, pinned there
    against the FP64 oracle. Errors are max |step - fp64| / max |fp64| per field, after the
    timed region and outside it."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from fp64_box import Box, active_mask, from_dense, to_dense

    from hnanosolver_b200 import synth

    t0 = time.perf_counter()
    coords = torch.from_numpy(synth.leaf_dense_coords(origins)).to(dev)
    lo = coords.min(dim=0).values.cpu().numpy()
    shape = tuple(int(v) for v in (coords.max(dim=0).values.cpu().numpy() - lo + 1))
    box = Box(shape, lo, wl["dx"], dev, active=active_mask(coords, lo, shape, dev))
    v64 = to_dense(vel_in.double(), coords, lo, shape, dev)
    d64 = to_dense(dens_in.double(), coords, lo, shape, dev)
    v_adv, (d_adv,), _ = box.advect(v64, [d64], wl["dt"])
    del v64, d64
    v_prj, cg_iterations, cg_residual = box.project_exact(v_adv)
    del v_adv
    torch.cuda.empty_cache()

    def rel(got, ref):
        return float((got.double() - ref).abs().max() / ref.abs().max().clamp_min(1e-300))

    ref_v = from_dense(v_prj[0], coords, lo, numpy=False)
    ref_d = from_dense(d_adv[0], coords, lo, numpy=False)
    err = {"velocity": rel(vel_out.reshape(-1, 3), ref_v), "density": rel(dens_out.reshape(-1), ref_d),
           "checker": "torch FP64 restatement (tests/fp64_box.py) of advection + exact projection from the step's "
                      "stored inputs; max |step - fp64| / max |fp64|",
           "fp64_solve": {"cg_iterations": cg_iterations, "residual": cg_residual}, "seconds": time.perf_counter() - t0}
    del box, v_prj, d_adv, ref_v, ref_d, coords
    torch.cuda.empty_cache()
    return err


def _timed_steps(torch, stream, fn, steps):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


# Pass-model bytes per voxel-step of the adjoint plain step in FP32 (transposes of the forward
# passes, scatters counted as read-modify-write): gradient^T 16, adjoint copies and zeroing 16,
# red-black^T 12 per half-sweep (read lambda, write lambda, read-modify-write of div_bar on the
# colour) x 2 x iterations, divergence^T 28, velocity advection^T 48, scalar advection^T 52.
def adjoint_step_bytes(iters):
    return 16 + 16 + 24 * iters + 28 + 48 + 52


def adjoint_rollout(torch, hl, synth, dev, steps=16, every=4, iters=60):
    """Reverse pass of a checkpointed rollout through the C ABI, for the differentiable-rollout
    configuration: 128^3 fully active (2,097,152 voxels), K = 16 plain steps of advect (velocity
    and density) + project with 60 red-black iterations (omega 1, from p = 0), the state kept
    every 4 steps, loss 1/2 |rho_K - rho_target|^2 (target: seed-1 smoothed noise). The forward
    keeps the checkpoints; the backward recomputes each segment's step inputs from its
    checkpoint and runs hns_adjoint_step_plain on them in reverse. CUDA events on the grid's
    stream; one untimed pass first."""
    origins = synth.topology("box128")
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    target, _ = synth.smoothed_fields(origins, seed=1, box_passes=3)
    n = len(dens)
    g = hl.Grid(origins, voxel_size=0.1)
    stream = torch.cuda.Stream(device=dev)
    g.set_stream(stream.cuda_stream)
    desc = hl.StepDesc(dt=0.1, max_iterations=iters, omega=1.0, tolerance=0.0, check_every=0, flags=0)
    v0, d0 = torch.from_numpy(vel).to(dev), torch.from_numpy(dens).to(dev)
    tg = torch.from_numpy(target).to(dev)
    torch.cuda.synchronize()

    def step(v, d):
        v2, d2 = torch.empty_like(v), torch.empty_like(d)
        g.step_plain(v, v2, [d], [d2], desc)
        return v2, d2

    def forward():
        ckpt, v, d = [], v0, d0
        for k in range(steps):
            if k % every == 0:
                ckpt.append((v, d))  # each step writes new tensors, so no copy is needed
            v, d = step(v, d)
        return ckpt, d

    def backward(ckpt, dk):
        vb, db = torch.zeros_like(v0), dk - tg
        for seg in reversed(range(len(ckpt))):
            k0 = seg * every
            states = [ckpt[seg]]
            for _ in range(k0, min(k0 + every, steps) - 1):
                states.append(step(*states[-1]))
            for v_in, d_in in reversed(states):
                vi, di = torch.zeros_like(vb), torch.zeros_like(db)
                g.adjoint_step_plain(v_in, [d_in], vb, [db], vi, [di], desc.dt, iters, desc.omega)
                vb, db = vi, di
        return vb, db

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    with torch.cuda.stream(stream):
        backward(*forward())
        torch.cuda.synchronize()
        ev[0].record(stream)
        ckpt, dk = forward()
        ev[1].record(stream)
        backward(ckpt, dk)
        ev[2].record(stream)
    torch.cuda.synchronize()
    f_ms, b_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    g.close()
    recomputed = steps - (steps + every - 1) // every
    # The forward plain step's pass model (FP32, one scalar): advect velocity 24, divergence 16,
    # 12 per red-black iteration, gradient 28, the velocity written once more 12, density 8.
    fwd_bytes = 24 + 16 + 12 * iters + 28 + 12 + 8
    moved = (adjoint_step_bytes(iters) * steps + fwd_bytes * recomputed) * n
    return {"workload": "box128 rollout: 128^3 fully active, 16 steps of advect + project, 60 red-black iterations, "
                        "checkpoint every 4 steps, loss 1/2 |rho_K - rho_target|^2",
            "voxels": n, "steps": steps, "checkpoint_every": every, "iterations": iters,
            "forward_ms": f_ms, "backward_ms": b_ms, "backward_over_forward": b_ms / f_ms,
            "value": n * steps / (b_ms / 1e3), "unit": "voxel-steps/s (reverse pass, recomputation included)",
            "adjoint_step_bytes_per_voxel": adjoint_step_bytes(iters), "recomputed_steps": recomputed,
            "achieved_gbs": moved / (b_ms / 1e3) / 1e9}


def ours(args, wl):
    import torch

    from hnanosolver_b200 import lib as hl
    from hnanosolver_b200 import replicas, synth

    R = replicas.ranks_from_env()
    rank, world, local = R.rank, R.world, R.local
    replicas.start(R, "nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    origins = synth.topology(args.workload)
    dens, vel = synth.noise_fields(origins, seed=replicas.seed_of(R))
    n = len(dens)
    g = hl.Grid(origins, voxel_size=wl["dx"], device=local)
    apply_options(g, hl, args)
    stream = torch.cuda.Stream(device=dev)
    g.set_stream(stream.cuda_stream)
    mixed = args.precision == "mixed"
    multigrid = mixed and args.inner == "multigrid"
    tol = wl["tolerance"]

    # ---- FP32 forms (always measured: the comparison at equal residual) ----
    v = [torch.from_numpy(vel).to(dev), torch.empty((n, 3), device=dev)]
    d = [torch.from_numpy(dens).to(dev), torch.empty(n, device=dev)]

    def plain_desc(cap, refine=False):
        if refine:
            return hl.StepDesc(dt=wl["dt"], max_iterations=0, omega=wl["omega_refined"], tolerance=tol, check_every=10,
                               flags=hl.SOLVE_REFINE, max_outer=cap, inner_iterations=wl["inner"])
        return hl.StepDesc(dt=wl["dt"], max_iterations=cap, omega=wl["omega"], tolerance=tol,
                           check_every=wl["check_every"], flags=0)

    def solve_once(fn, last):
        try:
            return fn()
        except hl.HnsError as e:
            if e.status != 6:  # HNS_ERR_NOT_CONVERGED: keep the cap
                raise
            return last()

    info32 = solve_once(lambda: g.step_plain(v[0], v[1], [d[0]], [d[1]], plain_desc(wl["cap"]), info=True), g.last_solve)
    if args.no_fp32_comparison and mixed:
        info32 = hl.SolveInfo(iterations=wl["fp32_iterations"] or info32.iterations, residual=info32.residual)
    cap32 = info32.iterations if tol == 0 else info32.iterations + 2 * max(2, wl["check_every"])
    if args.no_fp32_comparison and mixed:
        infor = hl.SolveInfo(iterations=wl["inner"], residual=0.0)
    else:
        infor = solve_once(lambda: g.step_plain(v[0], v[1], [d[0]], [d[1]], plain_desc(16, True), info=True), g.last_refine)
    outer_r = max(1, infor.iterations // wl["inner"]) + 1
    state = [0]

    def step32(desc):
        def f():
            s0 = state[0]
            g.step_plain(v[s0], v[1 - s0], [d[s0]], [d[1 - s0]], desc)
            state[0] = 1 - s0
        return f

    cmp_steps = max(1, min(args.steps, 3))
    if args.no_fp32_comparison and mixed:
        cmp_steps = 0
    for _ in range(2 if cmp_steps else 0):
        step32(plain_desc(cap32))()
    fp32 = None
    if cmp_steps:
        ms_plain = _timed_steps(torch, stream, step32(plain_desc(cap32)), cmp_steps) / cmp_steps
        last32 = g.last_solve()
        for _ in range(2):
            step32(plain_desc(outer_r, True))()
        ms_ref = _timed_steps(torch, stream, step32(plain_desc(outer_r, True)), cmp_steps) / cmp_steps
        lastr = g.last_refine()
        fp32 = {"plain": {"value": n / (ms_plain / 1e3), "ms_per_step": ms_plain, "omega": wl["omega"],
                          "red_black_iterations": last32.iterations, "residual_checked": last32.residual},
                "refined": {"value": n / (ms_ref / 1e3), "ms_per_step": ms_ref, "omega": wl["omega_refined"],
                            "inner_iterations": wl["inner"], "red_black_iterations": lastr.iterations,
                            "residual": lastr.residual}}

    # ---- the timed form ----
    if mixed:
        vb = [torch.from_numpy(vel).to(dev).to(torch.bfloat16).contiguous(), torch.empty((n, 3), dtype=torch.bfloat16, device=dev)]
        dh = [torch.from_numpy(dens).to(dev).to(torch.float16).contiguous(), torch.empty(n, dtype=torch.float16, device=dev)]

        def mdesc(outer, mg):
            if mg:
                return hl.MixedDesc(dt=wl["dt"], omega=wl["omega_refined"], tolerance=tol, max_outer=outer,
                                    inner_iterations=args.cycles, flags=hl.SOLVE_MULTIGRID)
            return hl.MixedDesc(dt=wl["dt"], omega=wl["omega_refined"], tolerance=tol, max_outer=outer,
                                inner_iterations=wl["inner"], flags=0)

        ms_state = [0]

        def mixed_form(mg):
            """(solve info of a calibration step, the step at an outer cap one above its need)."""
            info = solve_once(lambda: g.step_mixed(vb[0], vb[1], [dh[0]], [dh[1]], mdesc(16, mg), info=True),
                              g.last_refine)
            outer = max(1, info.iterations // (args.cycles if mg else wl["inner"])) + 1
            st = mdesc(outer, mg)

            def step():
                s0 = ms_state[0]
                g.step_mixed(vb[s0], vb[1 - s0], [dh[s0]], [dh[1 - s0]], st)
                ms_state[0] = 1 - s0
            return info, outer, st, step

        red_black = None
        if multigrid:
            # The red-black inner solve in the same run: its time, and the time of its half-sweep
            # launches, the kernel that is also the multigrid's fine smoother (the roofline).
            _, _, _, step_rb = mixed_form(False)
            for _ in range(2):
                step_rb()
            rb_steps = max(1, min(args.steps, 3))
            g.profile_read()
            g.profile_enable(True)
            ms_rb = _timed_steps(torch, stream, step_rb, rb_steps) / rb_steps
            g.profile_enable(False)
            prof_rb = g.profile_read()
            last_rb = g.last_refine()
            red_black = {"ms_per_step": ms_rb, "value": n / (ms_rb / 1e3), "inner_iterations": wl["inner"],
                         "omega": wl["omega_refined"], "red_black_iterations": last_rb.iterations,
                         "residual": last_rb.residual,
                         "half_sweep_ms": prof_rb.phase_ms[hl.PHASES["inner"]] / max(1, prof_rb.solver_launches),
                         "half_sweeps_timed": int(prof_rb.solver_launches)}
        info, outer, st, step = mixed_form(multigrid)

        # record packing, advection, divergence, first residual, convergence log, gradient; per
        # outer iteration scale, 2 half-sweeps per inner iteration, update, residual (the face
        # table is made once per context).
        kernel_bytes, kernel_name, phase = F16_HALF_SWEEP_BYTES, KERNELS[("f16", args.split_solve)], "inner"
    else:
        info, outer = info32, None
        st = plain_desc(cap32)
        step = step32(st)
        kernel_bytes, kernel_name, phase = F32_HALF_SWEEP_BYTES, KERNELS[("f32", args.split_solve)], "solve"

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    replicas.barrier(R)
    clocks = ClockSampler(local)
    clocks.start()
    g.profile_read()
    g.profile_enable(True)
    g.solve_log(capacity=0, reset=True)
    ms = _timed_steps(torch, stream, step, args.steps)
    replicas.barrier(R)
    clk = clocks.stop()
    g.profile_enable(False)
    prof = g.profile_read()
    last = g.last_refine() if mixed else g.last_solve()
    # Every timed step's solve, from the device-side convergence log.
    logged, entries = g.solve_log(capacity=args.steps, reset=True)
    worst = max((e.residual for e in entries), default=float("nan"))
    not_converged = sum(1 for e in entries if e.residual > tol)
    ms = replicas.max_over_ranks(R, ms, dev)
    ms_step = ms / args.steps
    value = replicas.aggregate_rate(R, n, args.steps, ms)

    # Dominant kernel: average duration of its launches inside the timed region (phase
    # events around them / device counter of launches that ran). With the multigrid inner solve
    # the inner phase also holds the coarse levels: the half-sweep's launches are timed in the
    # red-black form of the same step, in the same run.
    if mixed and multigrid:
        k_ms = red_black["half_sweep_ms"]
        launches = red_black["half_sweeps_timed"]
    else:
        kms = prof.phase_ms[hl.PHASES[phase]]
        launches = max(1, prof.solver_launches)
        k_ms = kms / launches
    peak, peak_kind = measured_peak_gbs()
    achieved = kernel_bytes * n / (k_ms / 1e3) / 1e9
    traffic = profiled_traffic(args.workload, "split" if mixed else "f32")

    # End to end through the C ABI with FP32 host buffers: each step uploads velocity and
    # density from pinned host memory, steps, and downloads both.
    hv = torch.from_numpy(vel).pin_memory().numpy()
    hd = torch.from_numpy(dens).pin_memory().numpy()
    e2e_steps = max(1, min(args.steps, 5))
    if mixed:
        run_host = lambda: g.step_mixed_host(hv, [hd], st)  # noqa: E731
    else:
        run_host = lambda: g.step_plain_host(hv, [hd], st)  # noqa: E731
    run_host()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        run_host()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_s = replicas.max_over_ranks(R, e2e_s, dev)

    # The last timed step's result against FP64 (its inputs are the other buffer of the pair).
    field_error = None
    if rank == 0 and not args.no_field_error:
        out_i = ms_state[0] if mixed else state[0]
        if mixed:
            field_error = field_error_vs_fp64(torch, origins, wl, vb[1 - out_i], dh[1 - out_i], vb[out_i], dh[out_i], dev)
        else:
            field_error = field_error_vs_fp64(torch, origins, wl, v[1 - out_i], d[1 - out_i], v[out_i], d[out_i], dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, wl, wl["fp32_iterations"])
    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = adjoint_rollout(torch, hl, synth, dev)

    if rank == 0:
        phase_ms = {k: prof.phase_ms[i] / args.steps for k, i in hl.PHASES.items() if prof.phase_count[i]}
        cfg = workload_config(args, wl, origins)
        det = {"precision": args.precision, "split_solve": args.split_solve, "coarse_solve": args.coarse_solve, "l2_persist": not args.no_l2_persist, "parallelism": f"{world} independent replicas" if world > 1 else "1 GPU",
               "phase_ms_per_step": phase_ms, "fp32_forms_same_run": fp32,
               "mixed_vs_fp32_plain": (value / world) / fp32["plain"]["value"] if fp32 else None,
               "mixed_vs_fp32_refined": (value / world) / fp32["refined"]["value"] if fp32 else None,
               "timed_solves_logged": logged, "worst_residual_timed_steps": worst,
               "timed_steps_above_tolerance": not_converged, "field_error_vs_fp64": field_error}
        if mixed and multigrid:
            det.update({"storage": "velocity bf16, scalars f16, divergence f32, pressure f64, inner solve f16",
                        "inner_solve": "multigrid V-cycles: colour-split FP16 red-black half-sweeps (omega 1) as the "
                                       "fine smoother, FP32 leaf-local levels of 4, 2, 1 cells per leaf side",
                        "cycles_per_outer": args.cycles, "outer_cap": outer, "cycles": last.iterations,
                        "residual_reached": last.residual, "mixed_red_black_same_run": red_black,
                        "mixed_vs_mixed_red_black": red_black["ms_per_step"] / ms_step})
        elif mixed:
            det.update({"storage": "velocity bf16, scalars f16, divergence f32, pressure f64, inner solve f16",
                        "inner_solve": "red-black SOR iterations",
                        "omega_inner": wl["omega_refined"], "inner_iterations": wl["inner"], "outer_cap": outer,
                        "red_black_iterations": last.iterations, "residual_reached": last.residual})
        else:
            det.update({"omega": wl["omega"], "red_black_iterations": last.iterations, "iteration_cap": cap32,
                        "residual_checked": last.residual})
        line = {
            "metric": "active voxel-steps/s", "value": value, "unit": "voxel-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 arithmetic; bf16/f16 storage, f64 refinement" if mixed else "f32", "data": "synthetic",
            "config": cfg, "details": det,
            "roofline": {"kernel": kernel_name, "bound": "hbm", "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": kernel_bytes * n, "launch_ms": k_ms,
                         "launches_timed": int(launches)},
            "cpu_baseline": cpu,
            "e2e": {"value": world * n / e2e_s, "unit": "voxel-steps/s", "h2d_bytes_per_step": 16 * n,
                    "d2h_bytes_per_step": 16 * n, "steps": e2e_steps,
                    "path": ("hns_step_mixed_host" if mixed else "hns_step_plain_host") + " (C ABI, pinned FP32 host buffers)"},
            "gpu_launches": int(prof.kernel_launches),
            "clocks": clk,
            "adjoint": adjoint,
        }
        print(json.dumps(line), flush=True)
    g.close()
    replicas.finish(R)


def fire_params(mod):
    """(CombustionParams, ForceModel) of the fire step, from the module `mod` (the library's
    lib or the oracle's binding)."""
    p = mod.CombustionParams()
    p.expansionRate, p.temperatureRelease = 0.1, 0.5  # the oxygen burn's; unused by the rate burn
    p.buoyancyStrength, p.ambientTemp = FIRE["beta"], FIRE["ambient"]
    p.vorticityScale, p.factorScale = FIRE["confinement"], FIRE["factor_scale"]
    p.disturbanceEnable, p.substeps, p.gravity = 0.0, 1, 0.0
    m = mod.ForceModel(combustion=1, burn_rate=FIRE["burn_rate"], heat_release=FIRE["heat_release"],
                       ignition_temp=FIRE["ignition"], density_buoyancy=FIRE["alpha"])
    return p, m


def fire_config(args, wl, origins):
    n = 512 * len(origins)
    cfg = {"workload": args.workload, "step": "fire", "description": wl["desc"], "voxels": n, "leaves": len(origins),
           "dt": wl["dt"], "dx": wl["dx"], "forces": FIRE, "fp32_red_black_iterations": wl["fp32_iterations"],
           "l2": "inputs larger than L2 (%.0f MB of fields and solver state per GPU)" % (80 * n / 1e6)}
    if "tolerance" in wl:
        cfg["tolerance"] = wl["tolerance"]
        cfg["residual"] = "relative FP64 Poisson residual ||b - L p|| / ||b||, b = div dx^2"
    return cfg


def fire_cpu_sample(args, wl, iters, omega, steps, warmup, budget_s=None):
    """The reference's HNS_Advance with its `combustion` kernel (oracle/_ref, all host threads)
    on a bounded sample: every launch over 1/S of its 256-voxel blocks. Returns (rate, sample
    description, threads)."""
    from hnanosolver_b200 import synth
    from oracle import binding

    ref = binding.RefOracle()
    origins, fields, sources = synth.fire_state(args.workload)
    g = ref.grid(synth.leaf_dense_coords(origins))
    n = 512 * len(origins)
    blocks = (n + 255) // 256
    stride = max(1, blocks // 2048)
    params, model = fire_params(binding)
    state = {k: v for k, v in fields.items() if k != "velocity"}
    ref.lib.ref_set_block_stride(stride)

    def one(k):
        return g.hns_advance_model(fields["velocity"], state, sources, wl["dx"], k, wl["dt"], params,
                                   combustion=1, burn_rate=model.burn_rate, heat_release=model.heat_release,
                                   ignition_temp=model.ignition_temp, omega=omega)

    def timed(k, reps):
        for _ in range(warmup):
            one(k)
        times, t_start = [], time.perf_counter()
        while len(times) < reps and (budget_s is None or not times or time.perf_counter() - t_start < budget_s):
            t0 = time.perf_counter()
            one(k)
            times.append(time.perf_counter() - t0)
        return sum(times) / len(times), len(times)

    # Up to 200 iterations the step runs as is; above, its fixed part (0 iterations) and 40
    # iterations are timed and the iterations' cost is extrapolated linearly to `iters`.
    if iters <= 200:
        t, reps = timed(iters, steps)
        how = f"{reps} steps"
    else:
        t0, r0 = timed(0, steps)
        t40, r40 = timed(40, steps)
        t = t0 + (t40 - t0) / 40.0 * iters
        how = (f"{r0} steps with 0 and {r40} with 40 red-black iterations, the iterations' time extrapolated "
               f"linearly to {iters}")
    ref.lib.ref_set_block_stride(1)
    sampled = (blocks + stride - 1) // stride * 256
    sample = (f"{how}, of the reference's HNS_Advance kernels with its combustion kernel (no density buoyancy "
              f"term: the reference has none), every launch over 1/{stride} of its 256-voxel blocks ({sampled} of "
              f"{n} voxels), {iters} red-black iterations at omega {omega or 'from dx'}")
    return sampled / t, sample, ref.lib.ref_num_threads(), binding.cpu_model(), os.path.basename(ref.path)


def reference_arm_fire(args, wl):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    from hnanosolver_b200 import synth

    origins = synth.topology(args.workload)
    iters = wl["fp32_iterations"] or 1000
    value, sample, cores, cpu, library = fire_cpu_sample(args, wl, iters, wl.get("omega", 0.0), args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": "active voxel-steps/s", "value": value, "unit": "voxel-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 512 * len(origins) / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": fire_config(args, wl, origins),
        "cpu_baseline": {"value": value, "unit": "voxel-steps/s", "cores": cores, "kind": "reference", "sample": sample,
                         "cpu": cpu, "library": library},
        "e2e": {"value": value, "unit": "voxel-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fire_adjoint_rollout(torch, hl, g, stream, state0, src, dt, params, model, desc, n, steps=8, every=4):
    """Reverse pass of a checkpointed rollout of the mixed fire step through the C ABI: `steps`
    steps of hns_advance_mixed from state0 (BF16/FP16 device tensors), the state kept every
    `every` steps, loss 1/2 |rho_K - rho_target|^2 (target: seed-1 value noise); the backward
    recomputes each segment's step inputs from its checkpoint and runs hns_adjoint_advance_mixed
    on them in reverse (FP32 adjoints). CUDA events on the grid's stream; one untimed pass first."""
    target = torch.rand(n, device=state0["density"].device, generator=torch.Generator(device=state0["density"].device).manual_seed(1))

    def step(cur):
        nxt = {k: torch.empty_like(v) for k, v in cur.items()}
        g.advance_mixed(cur, nxt, src, dt, params, model, desc)
        return nxt

    def forward():
        ckpt, cur = [], state0
        for k in range(steps):
            if k % every == 0:
                ckpt.append(cur)  # each step writes new tensors
            cur = step(cur)
        return ckpt, cur

    def backward(ckpt, last):
        bar = {k: torch.zeros(v.numel(), device=v.device) for k, v in last.items()}
        bar["density"] = last["density"].float() - target
        for seg in reversed(range(len(ckpt))):
            states = [ckpt[seg]]
            for _ in range(seg * every, min(seg * every + every, steps) - 1):
                states.append(step(states[-1]))
            for s_in in reversed(states):
                ib = {k: torch.zeros_like(v) for k, v in bar.items()}
                g.adjoint_advance_mixed(s_in, src, bar, ib, dt, params, model, desc)
                bar = ib
        return bar

    with torch.cuda.stream(stream):
        backward(*forward())
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(stream)
        ckpt, last = forward()
        ev[1].record(stream)
        grads = backward(ckpt, last)
        ev[2].record(stream)
    torch.cuda.synchronize()
    f_ms, b_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    finite = all(bool(torch.isfinite(v).all()) for v in grads.values())
    recomputed = steps - (steps + every - 1) // every
    return {"workload": f"{steps}-step rollout of the mixed fire step, checkpoint every {every} steps, "
                        "loss 1/2 |rho_K - rho_target|^2; adjoints FP32, solves refined to the step's tolerance",
            "voxels": n, "steps": steps, "checkpoint_every": every, "recomputed_steps": recomputed,
            "forward_ms": f_ms, "backward_ms": b_ms, "backward_over_forward": b_ms / f_ms,
            "value": n * steps / (b_ms / 1e3), "unit": "voxel-steps/s (reverse pass, recomputation included)",
            "gradients_finite": finite}


def ours_fire(args, wl):
    import torch

    from hnanosolver_b200 import lib as hl
    from hnanosolver_b200 import replicas, synth

    R = replicas.ranks_from_env()
    rank, world, local = R.rank, R.world, R.local
    replicas.start(R, "nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    origins, fields, sources = synth.fire_state(args.workload, seed=replicas.seed_of(R))
    n = 512 * len(origins)
    g = hl.Grid(origins, voxel_size=wl["dx"], device=local)
    apply_options(g, hl, args)
    stream = torch.cuda.Stream(device=dev)
    g.set_stream(stream.cuda_stream)
    params, model = fire_params(hl)
    mixed = args.precision == "mixed"
    multigrid = mixed and args.inner == "multigrid"
    dt = wl["dt"]
    tol = wl.get("tolerance")

    def load_fp32():
        for k, a in {**fields, **sources}.items():
            g.field_set(k, a)

    # ---- FP32 forms of the fire step at the same residual (the solve-to-tolerance workloads) ----
    fp32 = None
    cap32 = None
    if tol is not None and not args.no_fp32_comparison:
        def pdesc(cap):
            return hl.StepDesc(dt=0.0, max_iterations=cap, omega=wl["omega"], tolerance=tol,
                               check_every=wl["check_every"], flags=0)

        def rdesc(outer):
            return hl.StepDesc(dt=0.0, max_iterations=0, omega=wl["omega_refined"], tolerance=tol, check_every=10,
                               flags=hl.SOLVE_REFINE, max_outer=outer, inner_iterations=wl["inner"])

        def tolerant(fn):
            try:
                return fn()
            except hl.HnsError as e:
                if e.status != 6:
                    raise
                return None

        cmp_steps = 0 if args.no_fp32_comparison else max(1, min(args.steps, 3))
        load_fp32()
        i32 = tolerant(lambda: g.advance_solve(dt, params, model, pdesc(wl["cap"]), info=True))
        stalled = i32 is None
        i32 = i32 or g.last_solve()
        cap32 = i32.iterations + 2 * wl["check_every"]
        load_fp32()
        ir = tolerant(lambda: g.advance_solve(dt, params, model, rdesc(60), info=True)) or g.last_refine()
        outer_r = max(1, ir.iterations // wl["inner"]) + 2
        if cmp_steps:
            if stalled:
                plain = {"converged": False, "omega": wl["omega"], "red_black_iterations": i32.iterations,
                         "residual_checked": i32.residual,
                         "note": "plain FP32 SOR stops above the tolerance (its rounding floor): no equal-residual time"}
            else:
                load_fp32()
                g.advance_solve(dt, params, model, pdesc(cap32))
                ms_plain = _timed_steps(torch, stream, lambda: g.advance_solve(dt, params, model, pdesc(cap32)),
                                        cmp_steps) / cmp_steps
                lp = g.last_solve()
                plain = {"value": n / (ms_plain / 1e3), "ms_per_step": ms_plain, "omega": wl["omega"],
                         "red_black_iterations": lp.iterations, "residual_checked": lp.residual}
            load_fp32()
            g.advance_solve(dt, params, model, rdesc(outer_r))
            ms_ref = _timed_steps(torch, stream, lambda: g.advance_solve(dt, params, model, rdesc(outer_r)),
                                  cmp_steps) / cmp_steps
            lr = g.last_refine()
            fp32 = {"plain": plain,
                    "refined": {"value": n / (ms_ref / 1e3), "ms_per_step": ms_ref, "omega": wl["omega_refined"],
                                "inner_iterations": wl["inner"], "red_black_iterations": lr.iterations,
                                "residual": lr.residual}}

    # ---- the timed form ----
    red_black = None
    if mixed:
        def to_dev(d):
            out = {}
            for k, a in d.items():
                t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
                out[k] = (t.to(torch.bfloat16) if k == "velocity" else t.to(torch.float16)).reshape(-1).contiguous()
            return out

        cur = to_dev(fields)
        bufs = [cur, {k: torch.empty_like(v) for k, v in cur.items()}]
        src = to_dev({"fuel": sources["src_fuel"], "temperature": sources["src_temperature"]})

        def mdesc(outer, mg):
            if mg:
                return hl.MixedDesc(dt=0.0, omega=wl["omega_refined"], tolerance=tol, max_outer=outer,
                                    inner_iterations=args.cycles, flags=hl.SOLVE_MULTIGRID)
            return hl.MixedDesc(dt=0.0, omega=wl["omega_refined"], tolerance=tol, max_outer=outer,
                                inner_iterations=wl["inner"], flags=0)

        ms_state = [0]

        def fire_form(mg):
            torch.cuda.synchronize()
            try:
                info = g.advance_mixed(bufs[0], bufs[1], src, dt, params, model, mdesc(60, mg), info=True)
            except hl.HnsError as e:
                if e.status != 6:
                    raise
                info = g.last_refine()
            outer = max(1, info.iterations // (args.cycles if mg else wl["inner"])) + 2
            st = mdesc(outer, mg)

            def step():
                s0 = ms_state[0]
                g.advance_mixed(bufs[s0], bufs[1 - s0], src, dt, params, model, st)
                ms_state[0] = 1 - s0
            return info, outer, st, step

        red_black = None
        if multigrid:
            # The red-black inner solve in the same run (time, and its half-sweeps for the roofline).
            _, _, _, step_rb = fire_form(False)
            step_rb()
            rb_steps = max(1, min(args.steps, 2))
            g.profile_read()
            g.profile_enable(True)
            ms_rb = _timed_steps(torch, stream, step_rb, rb_steps) / rb_steps
            g.profile_enable(False)
            prof_rb = g.profile_read()
            last_rb = g.last_refine()
            red_black = {"ms_per_step": ms_rb, "value": n / (ms_rb / 1e3), "inner_iterations": wl["inner"],
                         "omega": wl["omega_refined"], "red_black_iterations": last_rb.iterations,
                         "residual": last_rb.residual,
                         "half_sweep_ms": prof_rb.phase_ms[hl.PHASES["inner"]] / max(1, prof_rb.solver_launches),
                         "half_sweeps_timed": int(prof_rb.solver_launches)}
        info, outer, st, step = fire_form(multigrid)

        # record packing, velocity advection, confinement, divergence/burn/buoyancy, first residual,
        # convergence log, gradient, scalar advection; per outer iteration scale, 2 half-sweeps per
        # inner iteration, update, residual.
        kernel_bytes, kernel_name, phase = F16_HALF_SWEEP_BYTES, KERNELS[("f16", args.split_solve)], "inner"
    else:
        load_fp32()
        iters = wl["iterations"]
        outer = None

        def step():
            g.advance(iters, dt, params, model)

        # velocity advection, confinement and sources, divergence/burn/buoyancy, the red-black
        # iterations, gradient, scalar advection.
        kernel_bytes, kernel_name, phase = F32_HALF_SWEEP_BYTES, KERNELS[("f32", args.split_solve)], "solve"

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    replicas.barrier(R)
    clocks = ClockSampler(local)
    clocks.start()
    g.profile_read()
    g.profile_enable(True)
    g.solve_log(capacity=0, reset=True)
    ms = _timed_steps(torch, stream, step, args.steps)
    replicas.barrier(R)
    clk = clocks.stop()
    g.profile_enable(False)
    prof = g.profile_read()
    logged, entries = g.solve_log(capacity=args.steps, reset=True)
    worst = max((e.residual for e in entries), default=None)
    ms = replicas.max_over_ranks(R, ms, dev)
    value = replicas.aggregate_rate(R, n, args.steps, ms)
    launches = max(1, prof.solver_launches)
    k_ms = prof.phase_ms[hl.PHASES[phase]] / launches
    if red_black is not None:  # the multigrid inner phase also holds the coarse levels
        k_ms, launches = red_black["half_sweep_ms"], red_black["half_sweeps_timed"]
    peak, peak_kind = measured_peak_gbs()
    achieved = kernel_bytes * n / (k_ms / 1e3) / 1e9

    # End to end through the C ABI with FP32 host buffers (pinned).
    e2e_steps = max(1, min(args.steps, 3))
    hf = {k: torch.from_numpy(np.ascontiguousarray(v.reshape(-1))).pin_memory().numpy() for k, v in fields.items()}
    hs = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy() for k, v in sources.items()}
    if mixed:
        hsrc = {"fuel": hs["src_fuel"], "temperature": hs["src_temperature"]}
        run_host = lambda: g.advance_mixed_host(hf, hsrc, dt, params, model, st)  # noqa: E731
        h2d = (12 + 4 * 4 + 2 * 4) * n
        d2h = (12 + 4 * 4) * n
        path = "hns_advance_mixed_host (C ABI, pinned FP32 host buffers: fields and sources up, fields down)"
    else:
        def run_host():
            for k, a in hs.items():
                g.field_set(k, a)
            g.advance(wl["iterations"], dt, params, model)
            for k in fields:
                g.field_get(k, out=hf[k])
        h2d = 2 * 4 * n
        d2h = (12 + 4 * 4) * n
        path = ("hns_field_set of the sources, hns_advance_model, hns_field_get of every field (the reference's "
                "per-cook HNS_UploadSources / HNS_Advance / HNS_DownloadForOutput crossing)")
    run_host()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        run_host()
    e2e_s = replicas.max_over_ranks(R, (time.perf_counter() - t0) / e2e_steps, dev)

    adjoint = None
    if rank == 0 and world == 1 and mixed and not args.no_adjoint:
        adjoint = fire_adjoint_rollout(torch, hl, g, stream, bufs[0], src, dt, params, model, mdesc(outer + 4, multigrid), n)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        iters_cpu = wl["iterations"] if not mixed else (wl["fp32_iterations"] or cap32 or wl["cap"])
        v, sample, cores, cpu_name, library = fire_cpu_sample(args, wl, iters_cpu, wl.get("omega", 0.0), 3, 0,
                                                              budget_s=20.0)
        cpu = {"value": v, "unit": "voxel-steps/s", "cores": cores, "kind": "reference", "sample": sample,
               "cpu": cpu_name}

    if rank == 0:
        phase_ms = {k: prof.phase_ms[i] / args.steps for k, i in hl.PHASES.items() if prof.phase_count[i]}
        det = {"precision": args.precision, "split_solve": args.split_solve, "coarse_solve": args.coarse_solve, "l2_persist": not args.no_l2_persist, "parallelism": f"{world} independent replicas" if world > 1 else "1 GPU",
               "phase_ms_per_step": phase_ms, "fp32_forms_same_run": fp32,
               "mixed_vs_fp32_plain": (value / world) / fp32["plain"]["value"] if fp32 and "value" in fp32["plain"] else None,
               "mixed_vs_fp32_refined": (value / world) / fp32["refined"]["value"] if fp32 else None,
               "timed_solves_logged": logged, "worst_residual_timed_steps": worst,
               "timed_steps_above_tolerance": (sum(1 for e in entries if e.residual > tol) if tol else None)}
        if mixed and multigrid:
            det.update({"storage": "velocity bf16, scalars f16, divergence f32, pressure f64, inner solve f16",
                        "inner_solve": "multigrid V-cycles: colour-split FP16 red-black half-sweeps (omega 1) as the "
                                       "fine smoother, FP32 leaf-local levels of 4, 2, 1 cells per leaf side",
                        "cycles_per_outer": args.cycles, "outer_cap": outer, "mixed_red_black_same_run": red_black,
                        "mixed_vs_mixed_red_black": red_black["ms_per_step"] / (ms / args.steps)})
        elif mixed:
            det.update({"storage": "velocity bf16, scalars f16, divergence f32, pressure f64, inner solve f16",
                        "inner_solve": "red-black SOR iterations",
                        "omega_inner": wl["omega_refined"], "inner_iterations": wl["inner"], "outer_cap": outer})
        else:
            det.update({"red_black_iterations": wl["iterations"], "omega": "2/(1+sin(3.14159 dx)) (the reference's)"})
        line = {
            "metric": "active voxel-steps/s", "value": value, "unit": "voxel-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 arithmetic; bf16/f16 storage, f64 refinement" if mixed else "f32", "data": "synthetic",
            "config": fire_config(args, wl, origins), "details": det,
            "roofline": {"kernel": kernel_name, "bound": "hbm", "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                         "algorithmic_bytes_per_launch": kernel_bytes * n, "launch_ms": k_ms,
                         "launches_timed": int(launches)},
            "cpu_baseline": cpu,
            "e2e": {"value": world * n / e2e_s, "unit": "voxel-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps, "path": path},
            "gpu_launches": int(prof.kernel_launches),
            "clocks": clk,
            "adjoint": adjoint,
        }
        print(json.dumps(line), flush=True)
    g.close()
    replicas.finish(R)


# The CPU-runnable single step: a 64^3 box fully active (512 leaves), smoothed noise fields,
# the plain FP32 step with 40 red-black iterations at omega 1.0 from p = 0.
BOX64 = dict(desc="64^3 box fully active (512 leaves); density value noise and velocity U(-1,1), each box-filtered "
                  "3 times; the plain FP32 step, 40 red-black iterations at omega 1.0",
             dx=0.1, dt=0.1, omega=1.0, iterations=40)


def box64_config(args):
    return {"workload": args.workload, "description": BOX64["desc"], "voxels": 262144, "leaves": 512,
            "dt": BOX64["dt"], "dx": BOX64["dx"], "red_black_iterations": BOX64["iterations"], "omega": BOX64["omega"],
            "walls": "zero-gradient (the spec's), the reference's Dirichlet-0 reported beside",
            "l2": "the 16 MB state fits in L2 (126 MB); no flush between steps"}


def box64_cpu(args, steps, warmup):
    from hnanosolver_b200 import synth
    from oracle import binding

    ref = binding.RefOracle()
    origins = synth.topology("box64")
    dens, vel = synth.smoothed_fields(origins, seed=0, box_passes=3)
    g = ref.grid(synth.leaf_dense_coords(origins))
    scratch = None
    for _ in range(warmup):
        scratch = g.plain_step(vel, [dens], BOX64["dt"], BOX64["dx"], BOX64["iterations"], BOX64["omega"], scratch)
    t0 = time.perf_counter()
    for _ in range(steps):
        scratch = g.plain_step(vel, [dens], BOX64["dt"], BOX64["dx"], BOX64["iterations"], BOX64["omega"], scratch)
    t = (time.perf_counter() - t0) / steps
    return {"value": 262144 / t, "unit": "voxel-steps/s", "cores": ref.lib.ref_num_threads(), "kind": "reference",
            "sample": f"{steps} full steps (no sampling) of the reference's kernels, Dirichlet-0 walls (the reference "
                      f"has no zero-gradient walls), 40 red-black iterations at omega 1.0",
            "cpu": binding.cpu_model(), "library": os.path.basename(ref.path)}


def box64_reference(args):
    rank, _, _ = dist_info()
    if rank != 0:
        return
    cpu = box64_cpu(args, args.steps, args.warmup)
    print(json.dumps({"impl": "reference", "metric": "active voxel-steps/s", "value": cpu["value"],
                      "unit": "voxel-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": 262144 / cpu["value"] * 1e3, "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": box64_config(args),
                      "cpu_baseline": cpu,
                      "e2e": {"value": cpu["value"], "unit": "voxel-steps/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def box64_ours(args):
    """The CPU-runnable single step on the GPU, zero-gradient walls (the spec's) and the reference's
    Dirichlet-0 walls, through hns_step_plain; e2e through hns_step_plain_host."""
    import torch

    from hnanosolver_b200 import lib as hl
    from hnanosolver_b200 import replicas, synth

    R = replicas.ranks_from_env()
    rank, world, local = R.rank, R.world, R.local
    replicas.start(R, "nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    origins = synth.topology("box64")
    dens, vel = synth.smoothed_fields(origins, seed=replicas.seed_of(R), box_passes=3)
    n = len(dens)
    g = hl.Grid(origins, voxel_size=BOX64["dx"], device=local)
    apply_options(g, hl, args)
    stream = torch.cuda.Stream(device=dev)
    g.set_stream(stream.cuda_stream)
    v = [torch.from_numpy(vel).to(dev), torch.empty((n, 3), device=dev)]
    d = [torch.from_numpy(dens).to(dev), torch.empty(n, device=dev)]
    forms = {}
    for name, flags in (("dirichlet", 0), ("zero_gradient", hl.SOLVE_NEUMANN)):
        desc = hl.StepDesc(dt=BOX64["dt"], max_iterations=BOX64["iterations"], omega=BOX64["omega"], tolerance=0.0,
                           check_every=0, flags=flags)
        st = [0]

        def step():
            a = st[0]
            g.step_plain(v[a], v[1 - a], [d[a]], [d[1 - a]], desc)
            st[0] = 1 - a

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        replicas.barrier(R)
        clocks = ClockSampler(local)
        clocks.start()
        g.profile_read()
        g.profile_enable(True)
        ms = _timed_steps(torch, stream, step, args.steps)
        g.profile_enable(False)
        prof = g.profile_read()
        replicas.barrier(R)
        clk = clocks.stop()
        ms = replicas.max_over_ranks(R, ms, dev)
        info = g.step_plain(v[0], v[1], [d[0]], [d[1]], desc, info=True)
        forms[name] = {"value": replicas.aggregate_rate(R, n, args.steps, ms), "ms_per_step": ms / args.steps,
                       "residual_after_40": info.residual, "clocks": clk,
                       "solve_ms_per_step": prof.phase_ms[hl.PHASES["solve"]] / args.steps,
                       "launches": int(prof.solver_launches), "kernel_launches": int(prof.kernel_launches)}
    hv = torch.from_numpy(vel).pin_memory().numpy()
    hd = torch.from_numpy(dens).pin_memory().numpy()
    desc = hl.StepDesc(dt=BOX64["dt"], max_iterations=BOX64["iterations"], omega=BOX64["omega"], tolerance=0.0,
                       check_every=0, flags=hl.SOLVE_NEUMANN)
    g.step_plain_host(hv, [hd], desc)
    e2e_steps = max(1, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        g.step_plain_host(hv, [hd], desc)
    e2e_s = replicas.max_over_ranks(R, (time.perf_counter() - t0) / e2e_steps, dev)
    cpu = box64_cpu(args, 3, 1) if rank == 0 and world == 1 and not args.no_cpu_baseline else None
    if rank == 0:
        z = forms["zero_gradient"]
        # The iteration kernel's pass model: read p, read div, write p (12 B per voxel); the state
        # sits in L2, so this is a rate, not an HBM bound.
        it_ms = z["solve_ms_per_step"] / max(1, z["launches"] / args.steps)
        peak, peak_kind = measured_peak_gbs()
        achieved = 12 * n / (it_ms / 1e3) / 1e9
        line = {"metric": "active voxel-steps/s", "value": z["value"], "unit": "voxel-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": z["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": box64_config(args), "details": {"walls": forms},
                "roofline": {"kernel": "rbgs_iteration_kernel<true> (zero-gradient walls)", "bound": "hbm",
                             "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None, "launch_ms": it_ms,
                             "note": "262,144 voxels sit in L2: launch-bound, the fraction is not an HBM bound"},
                "cpu_baseline": cpu,
                "e2e": {"value": world * n / e2e_s, "unit": "voxel-steps/s", "h2d_bytes_per_step": 16 * n,
                        "d2h_bytes_per_step": 16 * n, "steps": e2e_steps,
                        "path": "hns_step_plain_host (C ABI, pinned FP32 host buffers), zero-gradient walls"},
                "gpu_launches": z["kernel_launches"], "clocks": z["clocks"]}
        print(json.dumps(line), flush=True)
    g.close()
    replicas.finish(R)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(set(WORKLOADS) | set(FIRE_WORKLOADS) | {"box64"}), default="shell512")
    ap.add_argument("--forces", action="store_true",
                    help="the fire step (HNS_Advance with the configurations' forces) instead of the SOP chain; "
                         "implied by fire1024")
    ap.add_argument("--precision", choices=["mixed", "fp32"], default=None,
                    help="mixed (default for the SOP chain and fire1024) or fp32 (default for plume256 --forces)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint rollout measured beside the step")
    ap.add_argument("--no-field-error", action="store_true",
                    help="skip the FP64 check of the last timed step's fields (shell512 and plume256 steps)")
    ap.add_argument("--inner", choices=["multigrid", "red-black"], default="multigrid",
                    help="inner solve of the mixed-precision refinement: V-cycles with red-black smoothing "
                         "(HNS_SOLVE_MULTIGRID, default) or red-black SOR iterations")
    ap.add_argument("--cycles", type=int, default=2, help="V-cycles per outer refinement step (--inner multigrid)")
    ap.add_argument("--split-solve", choices=["persistent", "per-colour"], default="per-colour",
                    help="launch form of the colour-split red-black solves (same results to the bit)")
    ap.add_argument("--coarse-solve", choices=["cluster", "launches"], default="cluster",
                    help="the multigrid cycle's coarsest level: one thread-block cluster launch or two "
                         "launches per SOR sweep (same results to the bit)")
    ap.add_argument("--no-l2-persist", action="store_true",
                    help="ordinary caching for the FP16 inner solve's correction array (HNS_OPT_L2_PERSIST 0; "
                         "by default it persists in L2 where it fits)")
    ap.add_argument("--no-fp32-comparison", action="store_true",
                    help="skip the FP32 forms measured beside the mixed one (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.workload == "box64":
        (box64_reference if args.impl == "reference" else box64_ours)(args)
        return
    fire = args.forces or args.workload not in WORKLOADS
    if fire:
        if args.workload not in FIRE_WORKLOADS:
            ap.error(f"--forces has no fire workload {args.workload!r}")
        wl = FIRE_WORKLOADS[args.workload]
        args.precision = args.precision or wl["precision"]
        if args.precision == "mixed" and "tolerance" not in wl:
            ap.error("the mixed fire step solves to a tolerance; this workload runs a fixed iteration count")
        (reference_arm_fire if args.impl == "reference" else ours_fire)(args, wl)
        return
    args.precision = args.precision or "mixed"
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        reference_arm(args, wl)
    else:
        ours(args, wl)


if __name__ == "__main__":
    main()
