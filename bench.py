#!/usr/bin/env python
"""Benchmark of the B200 PBF solver on the reference's headline workload.

Metric: PBF particle-substeps/s of the 1,048,576-particle dam break (128x64x128 lattice, h = 0.025,
box [0,4]^3, 8 Jacobi iterations, dt = 1/120), and, as a second figure, differentiable grad-steps/s
of the 65,536-particle rollout (4 iterations, trajectory checkpoint every 10 steps).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One process per GPU (torchrun for N > 1).  The single-scene substep does not shard, so N GPUs run
N independent replicas (weak scaling); rank 0 prints one JSON line.  Timing: W untimed steps,
then K steps between a barrier + synchronize on both sides; every step is timed with CUDA events
on the solver's stream, with a 256 MiB write between steps to flush the 126 MB L2; the reported
time is the maximum over ranks.  `--impl reference` times the reference's own CUDA PBF (compiled
from its sources into oracle/_ref) on the same workload and GPU; the reference has no CPU path.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

METRIC = "PBF particle-substeps/s at 1M (fwd) & grad-steps/s at 64k, vs plain, same GPU"
UNIT = "particle-substeps/s"
FLUSH_BYTES = 256 << 20


def peaks():
    try:
        p = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s)"


# Nominal FP32 FMA peak of a B200: 148 SMs x 128 lanes x 2 FLOP x 1.965 GHz (not measured here).
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


class Clocks:
    """SM clock and throttle-reason samples taken while the timed region runs.

    A thread reads NVML (the source nvidia-smi prints) every 10 ms between start() and stop(), so
    even a timed region of a few hundred milliseconds has dozens of samples; if NVML cannot be
    loaded, nvidia-smi -lms 100 runs for the same window instead.  Reading clocks changes nothing.
    """

    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
                   "hw_power_brake_slowdown": 0x80}

    def __init__(self, index: int):
        self.index = index
        self.samples = []     # (sm_mhz, reason bits)
        self.max_mhz = None
        self.source = None
        self._stop = None
        self._thread = None
        self._proc = None
        self._path = pathlib.Path(f"/tmp/pbf_clocks_{os.getpid()}.csv")

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
            self._stop = threading.Event()

            def run():
                while not self._stop.is_set():
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(reasons(h))))
                    except Exception:
                        pass
                    self._stop.wait(0.01)

            self.source = "nvml"
            self._thread = threading.Thread(target=run, daemon=True)
            self._thread.start()
        except Exception:
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            try:
                self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                               "--format=csv,noheader,nounits", "-lms", "100"],
                                              stdout=open(self._path, "w"), stderr=subprocess.DEVNULL)
                self.source = "nvidia-smi"
            except Exception:
                self._proc = None

    def stop(self):
        if self._thread:
            self._stop.set()
            self._thread.join(timeout=5)
            self._thread = None
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            self._proc = None
            try:
                for r in self._path.read_text().strip().splitlines():
                    f = [x.strip() for x in r.split(",")]
                    if len(f) < 9 or not f[1].replace(".", "").isdigit():
                        continue
                    bits = 0
                    for name, col in (("hw_slowdown", 5), ("hw_thermal_slowdown", 6), ("sw_thermal_slowdown", 7),
                                      ("sw_power_cap", 8)):
                        if f[col].startswith("Active"):
                            bits |= self.REASON_BITS[name]
                    self.samples.append((float(f[1]), bits))
                    if f[2].replace(".", "").isdigit():
                        self.max_mhz = float(f[2])
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "samples": 0, "reasons": ["unsampled"], "source": self.source}
        reasons = sorted(name for name, bit in self.REASON_BITS.items() if any(b & bit for _, b in self.samples))
        return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "samples": len(self.samples), "reasons": reasons, "source": self.source}


def setup_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"   # gloo (CPU tests) reduces host tensors
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed(step, steps, warmup, world, stream, flush, clocks=None):
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    if clocks is not None:
        clocks.start()
    events = []
    t0 = time.perf_counter()
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.add_(1.0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
        step()
        b.record(stream)
        events.append((a, b))
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.stop()
    barrier(world)
    wall = time.perf_counter() - t0
    ms = sum(a.elapsed_time(b) for a, b in events)
    return ms, wall


# ------------------------------------------------------------------------------ B200 arm
def bench_b200(args, world, rank):
    from physica_b200 import pbf, scenes, trajectory
    from physica_b200.pbf import CacheField

    sc = scenes.plain_large(seed=2 + rank)
    n = sc.count
    solver, state, control, params = pbf.solver_for_scene(sc)
    cache = solver.allocate_step_cache()
    cur, nxt = state, solver.allocate_state()
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = solver.stream
    holder = {"cur": cur, "nxt": nxt}

    def step():
        solver.forward_step(holder["cur"], control, params, holder["nxt"], cache)
        holder["cur"], holder["nxt"] = holder["nxt"], holder["cur"]

    if args.launch_shape:   # a fixed shape (e.g. to profile one kernel variant); else the autotuner picks it
        shape, tuned_ms = fixed_shape(args.launch_shape), float("nan")
        solver.launch_shape = shape
    else:
        shape, tuned_ms = solver.autotune(state, control, params, repeats=4)   # outside the timing; 4 steps per shape steady the choice
    solver.set_graph_mode(True)   # one CUDA graph launch per substep (captured in the warm-up)
    launches0 = pbf.launch_count()
    clk = Clocks(torch.cuda.current_device())
    ms, wall = timed(step, args.steps, args.warmup, world, stream, flush, clk)
    launches = pbf.launch_count() - launches0
    per_step_launches = launches / (args.steps + args.warmup)
    ms_max = max_over_ranks(ms, world)
    ms_per_step = ms_max / args.steps
    value = world * n / (ms_per_step * 1e-3)

    # per-pass timing (profiled rerun, events around each kernel group on the same stream)
    lib = pbf.library()
    lib.pbf_profile_enable(solver.handle, 1)
    for _ in range(3):
        flush.add_(1.0)
        step()
    passes = read_profile(lib, solver.handle)
    lib.pbf_profile_enable(solver.handle, 0)
    neighbors = float(cache.read(CacheField.NEIGHBOR_COUNTS).double().mean())

    # throughput past the ejections (they start at substep 27): advance the scene to substep 97,
    # then time 20 more substeps after 3 warm-up ones, the same way
    late = None
    if not args.no_late:
        done = args.warmup + args.steps + 3
        for _ in range(max(0, 97 - done)):
            step()
        ms_late, _ = timed(step, 20, 3, world, stream, flush)
        ms_late = max_over_ranks(ms_late, world) / 20
        first_late = max(done, 97) + 3
        late = {"substeps": f"{first_late}-{first_late + 20}", "ms_per_step": round(ms_late, 4),
                "value": round(world * n / (ms_late * 1e-3), 1), "unit": UNIT,
                "mean_neighbors": round(float(cache.read(CacheField.NEIGHBOR_COUNTS).double().mean()), 3)}
    K = sc.pressure_iterations
    cells = solver.cells
    bytes_per_particle = {"list_scan": 16, "density_lambda": 16, "correction_project": 28, "vorticity": 36, "normal_confinement": 48,
                          "xsph": 48, "list_scan_density_lambda": 20}
    flops_per_pair = {"list_scan": 9, "density_lambda": 14 + 30, "correction_project": 25, "vorticity": 34, "normal_confinement": 26,
                      "xsph": 21, "list_scan_density_lambda": 9 + 14 + 30}
    hbm, hbm_src = peaks()
    top = max((p for p in passes if p["name"] in bytes_per_particle), key=lambda p: p["ms"], default=None)
    roofline = None
    per_pass = {}
    for p in passes:
        avg = p["ms"] / max(p["launches"], 1)
        entry = {"launches_per_step": p["launches"] / 3, "avg_ms": round(avg, 5)}
        if p["name"] in bytes_per_particle:
            entry["algorithmic_GBps"] = round(bytes_per_particle[p["name"]] * n / (avg * 1e-3) / 1e9, 2)
            entry["fp32_TFLOPs"] = round(neighbors * flops_per_pair[p["name"]] * n / (avg * 1e-3) / 1e12, 3)
        per_pass[p["name"]] = entry
    if top is not None:
        avg = top["ms"] / top["launches"]
        achieved = bytes_per_particle[top["name"]] * n / (avg * 1e-3) / 1e9
        roofline = {"bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                    "frac": round(achieved / hbm, 5), "traffic": traffic_from_profiles(top["name"]),
                    "kernel": top["name"], "peak_source": hbm_src, "issue": issue_roofline(top["name"], avg),
                    "note": "gather passes are FP32/issue bound; fp32 fraction in per_pass and step_roofline"}
    b_alg = (192 + 44 * K) * n + 12 * cells
    f_alg = neighbors * (69 * K + 81) * n
    step_s = ms_per_step * 1e-3
    step_roofline = {"algorithmic_bytes": b_alg, "algorithmic_flops": round(f_alg),
                     "hbm_fraction": round(b_alg / step_s / (hbm * 1e9), 5),
                     "fp32_fraction_nominal": round(f_alg / step_s / (FP32_NOMINAL_TFLOPS * 1e12), 5),
                     "mean_neighbors": round(neighbors, 3)}

    # end to end through the host-buffer C ABI entry: H2D of the state, the step, D2H of the result
    e2e = None
    if not args.no_e2e:
        hx = torch.from_numpy(sc.positions.copy()).pin_memory()
        hv = torch.from_numpy(sc.velocities.copy()).pin_memory()
        ox, ov = torch.empty_like(hx).pin_memory(), torch.empty_like(hv).pin_memory()
        host = {"x": hx, "v": hv, "ox": ox, "ov": ov, "step": 0}

        def host_step():
            host["step"] = solver.forward_step_host(host["x"], host["v"], control, params, host["ox"], host["ov"], cache,
                                                    host["step"])
            host["x"], host["ox"] = host["ox"], host["x"]
            host["v"], host["ov"] = host["ov"], host["v"]

        for _ in range(2):
            host_step()
        barrier(world)
        ke = max(3, min(args.steps, 10))
        total = 0.0
        for _ in range(ke):
            with torch.cuda.stream(stream):   # the same L2 flush as the device-timed loop, outside the timing
                flush.add_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            host_step()   # returns after its downloads completed
            total += time.perf_counter() - t0
        dt = max_over_ranks(total / ke, world)
        # the copies alone: CUDA events around the uploads and the downloads of three profiled host steps
        lib.pbf_profile_enable(solver.handle, 1)
        for _ in range(3):
            with torch.cuda.stream(stream):
                flush.add_(1.0)
            host_step()
        copies = {q["name"]: q["ms"] / 3 for q in read_profile(lib, solver.handle)}
        lib.pbf_profile_enable(solver.handle, 0)
        e2e = {"value": world * n / dt, "unit": UNIT, "h2d_bytes_per_step": 6 * 4 * n, "d2h_bytes_per_step": 6 * 4 * n,
               "ms_per_step": round(dt * 1e3, 4), "h2d_ms_per_step": round(copies.get("host_upload", float("nan")), 4),
               "d2h_ms_per_step": round(copies.get("host_download", float("nan")), 4),
               "timing": "host wall clock around each pbf_forward_step_host call (pinned host buffers, L2 flushed "
                         "before each call); d2h overlaps the post-loop passes (positions on a second stream)"}

    # differentiable rollout: grad-steps/s at 64k
    grad = None
    tangent = None
    if not args.no_grad:
        grad = bench_grad(args, world, rank)
        tangent = tangent_ms(args, world, sc)

    batched = None
    if not args.no_batch:
        batched = bench_batch(args, world, rank)
    batched_grad = None
    if not args.no_batch and not args.no_grad:
        batched_grad = bench_batch_grad(args, world, rank)

    sph_family = None if args.no_sph else bench_sph(args, world, rank)
    cpu, oracle_error = None, None
    if rank == 0 and not args.no_cpu_baseline:
        cpu, first, small_100 = cpu_baseline(sc)
        oracle_error = oracle_errors(sc, first, small_100)
    return {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded jittered-lattice dam break)",
        "config": {"workload": "dam_break_1m: 1,048,576 particles (128x64x128 lattice, spacing 0.5h, h=0.025), "
                               "box [0,4]^3, 8 Jacobi iterations, dt=1/120, XSPH c=0.01, vorticity eps=1e-4",
                   "particles_per_gpu": n, "pressure_iterations": K, "cells": cells, "replicas": world,
                   "l2": "flushed between timed steps (256 MiB write)", "wall_s": round(wall, 3), "graphs": True,
                   "launch_shape": {"list_scan": SCAN_VARIANTS[shape.list_scan],
                                    "scan_block": shape.scan_block_size, "block": shape.block_size,
                                    "autotune_ms_per_step": None if math.isnan(tuned_ms) else round(tuned_ms, 4)}},
        "roofline": roofline, "step_roofline": step_roofline, "per_pass": per_pass, "after_ejections": late,
        "cpu_baseline": cpu, "oracle_error": oracle_error, "e2e": e2e,
        "gpu_launches": int(round(per_step_launches * args.steps)),
        "clocks": clk.summary(), "grad_steps_per_s": grad, "tangent_ms_per_step": tangent, "batched_scenes": batched,
        "batched_grad_steps_per_s": batched_grad, "sph_family": sph_family,
    }


def read_profile(lib, handle, batch=False):
    import ctypes
    from physica_b200 import pbf

    class PassTime(ctypes.Structure):
        _fields_ = [("name", ctypes.c_char_p), ("launches", ctypes.c_uint64), ("milliseconds", ctypes.c_double)]

    arr = (PassTime * 32)()
    cnt = ctypes.c_uint32()
    fn = lib.pbf_batch_profile_read if batch else lib.pbf_profile_read
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(PassTime), ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
    pbf.check(fn(handle, arr, 32, ctypes.byref(cnt)))
    return [{"name": arr[k].name.decode(), "launches": int(arr[k].launches), "ms": float(arr[k].milliseconds)}
            for k in range(cnt.value)]


def profile_figure(name: str, kernel: str):
    """A per-launch figure `name [kernel] = value` recorded from an ncu capture under profiles/ (or None)."""
    for p in sorted((ROOT / "profiles").glob("*.md")):
        for line in p.read_text().splitlines():
            if line.startswith(name) and f"[{kernel}]" in line:
                try:
                    return int(line.split("=")[-1].strip())
                except ValueError:
                    pass
    return None


def traffic_from_profiles(kernel: str):
    """DRAM bytes per launch of `kernel` recorded from an ncu capture under profiles/ (or None)."""
    return profile_figure("traffic_bytes_per_launch", kernel)


def issue_roofline(kernel: str, launch_ms: float):
    """The bound the gather passes actually meet: instruction issue.  The warp instructions of one
    launch (ncu, profiles/) over its live CUDA-event duration, against the SM's issue limit of one
    warp instruction per scheduler per cycle (4 per SM) at the maximum SM clock."""
    instructions = profile_figure("warp_instructions_per_launch", kernel)
    if instructions is None or launch_ms <= 0:
        return None
    try:
        mhz = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["sm_max_mhz"])
    except Exception:
        mhz = 1965.0
    peak = 148 * 4 * mhz * 1e6 / 1e9
    achieved = instructions / (launch_ms * 1e-3) / 1e9
    return {"achieved": round(achieved, 1), "peak": round(peak, 1), "unit": "G warp-instructions/s",
            "frac": round(achieved / peak, 4), "warp_instructions": instructions}


SCAN_VARIANTS = ["per_lane", "cooperative", "staged", "fused_density", "fused_masks"]   # pbf_launch_shape.list_scan 0..4


def fixed_shape(text: str):
    """A launch shape from "variant:scan_block[:gather_block]", e.g. per_lane:128 or per_lane:128:32
    (the gather block defaults to 128): under a profiler the autotuner's timings mean nothing, so a
    profiled run fixes the shape that the plain run chose."""
    from physica_b200 import pbf
    parts = text.split(":")
    return pbf.LaunchShape(SCAN_VARIANTS.index(parts[0]), int(parts[1]),
                           int(parts[2]) if len(parts) > 2 else 128)


def bench_grad(args, world, rank):
    """grad-steps/s of the 64k rollout, with every Jacobi iterate kept (the default) and with the
    reference's in-step checkpoints (checkpoint_interval 2, the iterations between recomputed)."""
    from physica_b200 import pbf, scenes, trajectory
    sc = scenes.differentiable(seed=3 + rank)
    targets = torch.from_numpy(sc.targets).cuda()
    steps = 20

    def run(recompute, shape=None):
        solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable,
                                                              checkpoint_interval=2 if recompute else 1)
        if shape is not None:
            solver.launch_shape = shape
        elif args.launch_shape:
            solver.launch_shape = fixed_shape(args.launch_shape)
        else:
            solver.autotune(state, control, params, repeats=2)
        solver.set_checkpoint_recompute(recompute)
        solver.set_graph_mode(True)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        rollout = trajectory.Rollout(solver, control, params, steps, 10)   # buffers allocated once, outside the timing
        g = trajectory.loss_and_gradients(solver, state, control, params, targets, steps, rollout=rollout)   # warm-up
        torch.cuda.synchronize()
        held = free0 - torch.cuda.mem_get_info()[0]
        barrier(world)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(solver.stream)
        g = trajectory.loss_and_gradients(solver, state, control, params, targets, steps, rollout=rollout)
        b.record(solver.stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(a.elapsed_time(b), world)
        shape = solver.launch_shape
        del rollout, solver
        return ms, g, shape, held

    ms, g, shape, held = run(False)
    ms_r, g_r, _, held_r = run(True, shape)
    return {"value": round(world * steps / (ms * 1e-3), 3), "unit": "grad-steps/s",
            "rollout_memory_bytes": held,
            "checkpoint_recompute": {"value": round(world * steps / (ms_r * 1e-3), 3), "unit": "grad-steps/s",
                                     "in_step_checkpoint_interval": 2, "rollout_memory_bytes": held_r,
                                     "same_gradient": bool(torch.equal(g.initial_velocities, g_r.initial_velocities))},
            "config": {"workload": "differentiable_64k: 65,536 particles (32x64x32 lattice), v0 ~ N(0, 0.1), "
                                   "4 iterations, target-cloud loss", "rollout_steps": steps,
                       "trajectory_checkpoint_every": 10, "graphs": True,
                       "launch_shape": {"list_scan": SCAN_VARIANTS[shape.list_scan],
                                        "scan_block": shape.scan_block_size, "block": shape.block_size}},
            "loss": g.loss}


def tangent_ms(args, world, sc):
    """One differentiable substep and its jvp_step (unit position tangent, zero control and
    parameter tangents) on the 1M dam break, per step in ms."""
    from physica_b200 import pbf
    solver, state, control, params = pbf.solver_for_scene(sc, mode=pbf.ExecutionMode.differentiable)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    st, nt = solver.allocate_state_tangent(), solver.allocate_state_tangent()
    st.positions.fill_(1.0)
    ct, pt = solver.allocate_control(), solver.allocate_parameter_tangent()
    for t in pt.tensors.values():
        t.zero_()
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step():
        solver.forward_step(state, control, params, nxt, cache)
        solver.jvp_step(state, control, params, nxt, cache, st, ct, pt, nt)

    steps = max(3, min(args.steps, 5))
    ms, _ = timed(step, steps, 3, world, solver.stream, flush)
    del cache, solver
    torch.cuda.synchronize()
    return round(max_over_ranks(ms, world) / steps, 4)


def bench_batch(args, world, rank):
    """256 independent scenes (2,048-65,536 particles, log-uniform): one batched launch sequence per
    substep against one solver per scene, both on the same stream with CUDA events."""
    from physica_b200 import pbf, scenes
    scs = scenes.batched_forward(seed=4 + rank)
    total = sum(s.count for s in scs)
    batch, state, control, params = pbf.batch_for_scenes(scs)
    shape, _ = batch.autotune(state, control, params, repeats=2)
    batch.set_graph_mode(True)
    nxt = batch.allocate_state()
    holder = {"cur": state, "nxt": nxt}

    def batched_step():
        batch.forward_step(holder["cur"], control, params, holder["nxt"])
        holder["cur"], holder["nxt"] = holder["nxt"], holder["cur"]

    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    steps = max(3, min(args.steps, 10))
    ms_b, _ = timed(batched_step, steps, 3, world, batch.stream, flush)
    ms_b = max_over_ranks(ms_b, world) / steps

    solvers = []
    for sc in scs:
        solver, st, ctl, prm = pbf.solver_for_scene(sc)
        solver.set_graph_mode(True)
        solvers.append([solver, st, solver.allocate_state(), ctl, prm, solver.allocate_step_cache()])

    def loop_step():
        for e in solvers:
            e[0].forward_step(e[1], e[3], e[4], e[2], e[5])
            e[1], e[2] = e[2], e[1]

    ms_l, _ = timed(loop_step, steps, 3, world, solvers[0][0].stream, flush)
    ms_l = max_over_ranks(ms_l, world) / steps
    del solvers
    buckets = bucket_shapes(scs, shape, world, flush)
    return {"unit": UNIT, "batched": round(world * total / (ms_b * 1e-3), 1), "count_buckets": buckets,
            "per_scene_solvers": round(world * total / (ms_l * 1e-3), 1), "speedup": round(ms_l / ms_b, 3),
            "batched_ms_per_step": round(ms_b, 4), "per_scene_ms_per_step": round(ms_l, 4),
            "config": {"workload": "batched_forward_256: 256 dam-break scenes, counts log-uniform in [2048, 65536], "
                                   "4 iterations", "particles_per_gpu": total, "scenes_per_gpu": len(scs),
                       "graphs": True, "launch_shape": {"list_scan": SCAN_VARIANTS[shape.list_scan],
                                                         "scan_block": shape.scan_block_size, "block": shape.block_size}}}


def bucket_shapes(scs, shape, world, flush):
    """Per particle-count bucket (powers of two): the bucket's scenes as a batch of their own, timed
    with the shape its own autotuning picks and with the whole batch's shape.  One batch runs one
    launch per pass over all its scenes, so it runs one shape; this shows what a shape per bucket
    would gain."""
    from physica_b200 import pbf
    out = {}
    edges = [2048, 4096, 8192, 16384, 32768, 65537]
    for lo, hi in zip(edges[:-1], edges[1:]):
        sub = [s for s in scs if lo <= s.count < hi]
        if not sub:
            continue
        b, st, ct, pr = pbf.batch_for_scenes(sub)
        own, _ = b.autotune(st, ct, pr, repeats=2)
        b.set_graph_mode(True)

        def time_shape(sh):
            b.launch_shape = sh
            h = {"cur": pbf.State(st.positions.clone(), st.velocities.clone(), 0), "nxt": b.allocate_state()}

            def stp():
                b.forward_step(h["cur"], ct, pr, h["nxt"])
                h["cur"], h["nxt"] = h["nxt"], h["cur"]

            ms, _ = timed(stp, 5, 3, world, b.stream, flush)
            return max_over_ranks(ms, world) / 5

        own_ms, batch_ms = time_shape(own), time_shape(shape)
        out[f"{lo}-{hi - 1}"] = {"scenes": len(sub), "particles": sum(s.count for s in sub),
                                 "own_shape": [SCAN_VARIANTS[own.list_scan], own.scan_block_size, own.block_size],
                                 "own_ms_per_step": round(own_ms, 4), "batch_shape_ms_per_step": round(batch_ms, 4),
                                 "batch_shape_over_own": round(batch_ms / own_ms, 4)}
        del b, st, ct, pr
    return out


def bench_batch_grad(args, world, rank):
    """32 differentiable scenes (16,384-131,072 particles, uniform), each with its own target-cloud
    loss: one checkpointed batched rollout against one rollout per scene, CUDA events on the stream."""
    import ctypes
    import gc
    from physica_b200 import pbf, scenes, trajectory
    scs = scenes.batched_adjoint(seed=5 + rank)
    total = sum(s.count for s in scs)
    steps, every = 20, 10
    diff = pbf.ExecutionMode.differentiable

    def timed_rollout(solver, state, control, params, targets):
        rollout = trajectory.Rollout(solver, control, params, steps, every)
        trajectory.loss_and_gradients(solver, state, control, params, targets, steps, rollout=rollout)   # warm-up
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(solver.stream)
        trajectory.loss_and_gradients(solver, state, control, params, targets, steps, rollout=rollout)
        b.record(solver.stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    batch, state, control, params = pbf.batch_for_scenes(scs, mode=diff)
    batch.autotune(state, control, params, repeats=1)
    batch.set_graph_mode(True)
    targets = torch.from_numpy(np.concatenate([s.targets for s in scs], axis=1)).cuda()
    barrier(world)
    ms_b = max_over_ranks(timed_rollout(batch, state, control, params, targets), world)
    # where the batched rollout's time goes: one more rollout with per-pass CUDA events (no graphs)
    lib = pbf.library()
    lib.pbf_batch_profile_enable.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.pbf_batch_profile_enable(batch.handle, 1)
    trajectory.loss_and_gradients(batch, state, control, params, targets, steps, every)
    passes = read_profile(lib, batch.handle, batch=True)
    lib.pbf_batch_profile_enable(batch.handle, 0)
    total_pass_ms = sum(q["ms"] for q in passes) or 1.0
    pass_shares = {q["name"]: {"ms": round(q["ms"], 3), "share": round(q["ms"] / total_pass_ms, 4)}
                   for q in sorted(passes, key=lambda q: -q["ms"])}
    del batch, state, control, params, targets
    gc.collect()
    torch.cuda.synchronize()
    ms_l = 0.0
    for sc in scs:   # one scene at a time (its buffers allocated outside its timing)
        solver, st, ctl, prm = pbf.solver_for_scene(sc, mode=diff)
        solver.autotune(st, ctl, prm, repeats=1)
        solver.set_graph_mode(True)
        ms_l += timed_rollout(solver, st, ctl, prm, torch.from_numpy(sc.targets).cuda())
        del solver, st, ctl, prm
        gc.collect()
    ms_l = max_over_ranks(ms_l, world)
    return {"unit": "grad-steps/s", "batched": round(world * steps / (ms_b * 1e-3), 3),
            "per_scene_rollouts": round(world * steps / (ms_l * 1e-3), 3), "speedup": round(ms_l / ms_b, 3),
            "particle_grad_steps_per_s": round(world * total * steps / (ms_b * 1e-3), 1),
            "batched_passes": pass_shares,
            "config": {"workload": "batched_adjoint_32: 32 dam-break scenes, counts uniform in [16384, 131072], "
                                   "v0 ~ N(0, 0.1), 4 iterations, per-scene target-cloud loss and dL/dc_s",
                       "particles_per_gpu": total, "scenes_per_gpu": len(scs), "rollout_steps": steps,
                       "trajectory_checkpoint_every": every, "graphs": True}}


SPH_METHODS = ("wcsph", "pcisph", "iisph", "dfsph")
SPH_WORKLOAD = ("sph_dam_break_1m: 1,048,576 particles (128x64x128 lattice, spacing 0.5h, h=0.025), box [0,4]^3, "
                "dt=4e-4; PCISPH/IISPH 6 pressure iterations, DFSPH 4 divergence + 6 density iterations (the "
                "reference's defaults), DFSPH warm start from zero")


def bench_sph(args, world, rank, methods=SPH_METHODS):
    """The SPH family's forward substep (SPH<Method>::forward_step) at 1M particles, one solver per method."""
    from physica_b200 import sph, scenes
    out = {"unit": UNIT, "config": {"workload": SPH_WORKLOAD, "l2": "flushed between timed steps (256 MiB write)"}}
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    steps = max(3, min(args.steps, 8))
    for name in methods:
        sc = scenes.sph_large(seed=6 + rank, method=name)
        solver, state, control, params = sph.solver_for_scene(sc, sph.Method[name])
        cache = solver.allocate_step_cache()
        holder = {"cur": state, "nxt": solver.allocate_state()}

        def step():
            solver.forward_step(holder["cur"], control, params, holder["nxt"], cache)
            holder["cur"], holder["nxt"] = holder["nxt"], holder["cur"]

        ms, _ = timed(step, steps, args.warmup, world, solver.stream, flush)
        ms_per_step = max_over_ranks(ms, world) / steps
        out[name] = {"value": round(world * sc.count / (ms_per_step * 1e-3), 1), "ms_per_step": round(ms_per_step, 4)}
        del cache, solver
        torch.cuda.synchronize()
        if not args.no_grad:
            out[name]["gradient_ms_per_step"] = round(sph_gradient_ms(args, world, sc, name), 4)
            out[name]["tangent_ms_per_step"] = round(sph_tangent_ms(args, world, sc, name), 4)
    return out


def sph_gradient_ms(args, world, sc, name):
    """One differentiable SPH substep and its vjp_step (a unit next-state adjoint), per step in ms."""
    from physica_b200 import pbf, sph
    solver, state, control, params = sph.solver_for_scene(sc, sph.Method[name], mode=pbf.ExecutionMode.differentiable)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    n = sc.count
    na = solver.allocate_state_adjoint()
    na.positions.fill_(1.0)
    pa, ca, qa = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step():
        solver.forward_step(state, control, params, nxt, cache)
        solver.vjp_step(state, control, params, nxt, cache, na, pa, ca, qa)

    steps = max(3, min(args.steps, 5))
    ms, _ = timed(step, steps, 3, world, solver.stream, flush)
    del cache, solver
    torch.cuda.synchronize()
    return max_over_ranks(ms, world) / steps


def sph_tangent_ms(args, world, sc, name):
    """One differentiable SPH substep and its jvp_step (unit position tangent), per step in ms."""
    from physica_b200 import pbf, sph
    solver, state, control, params = sph.solver_for_scene(sc, sph.Method[name], mode=pbf.ExecutionMode.differentiable)
    cache = solver.allocate_step_cache()
    nxt = solver.allocate_state()
    st, nt = solver.allocate_state_tangent(), solver.allocate_state_tangent()
    st.positions.fill_(1.0)
    ct, pt = solver.allocate_control(), solver.allocate_parameter_tangent()
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step():
        solver.forward_step(state, control, params, nxt, cache)
        solver.jvp_step(state, control, params, nxt, cache, st, ct, pt, nt)

    steps = max(3, min(args.steps, 5))
    ms, _ = timed(step, steps, 3, world, solver.stream, flush)
    del cache, solver
    torch.cuda.synchronize()
    return max_over_ranks(ms, world) / steps


def reference_sph_tangent_ms(args, world, sc, name):
    """The reference's differentiable SPH substep and its jvp_step, per step in ms."""
    from oracle import reference
    from physica_b200 import sph
    n = sc.count
    ref = reference.ReferenceSPH(sc, int(sph.Method[name]), differentiable=True)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    z = lambda: torch.zeros(n, device="cuda")
    warm, warm_out = (z(), z()), (z(), z())
    tangent = {"positions": torch.ones((3, n), dtype=torch.float32, device="cuda"),
               "velocities": torch.zeros((3, n), dtype=torch.float32, device="cuda")}
    next_tangent = {k: torch.zeros_like(t) for k, t in tangent.items()}
    control_tangent = torch.zeros((3, n), dtype=torch.float32, device="cuda")
    warm_tangent, next_warm_tangent = (z(), z()), (z(), z())
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    def step():
        ref.forward_step(x, v, xo, vo, 0, warm=warm, warm_out=warm_out, synchronize=False)
        ref.jvp_step(x, v, tangent, control_tangent, {}, next_tangent, 0, warm=warm, warm_tangent=warm_tangent,
                     next_warm_tangent=next_warm_tangent, synchronize=False)

    steps = max(3, min(args.steps, 5))
    ms, _ = timed(step, steps, 3, world, torch.cuda.ExternalStream(ref.stream), flush)
    ref.close()
    torch.cuda.synchronize()
    return max_over_ranks(ms, world) / steps


def bench_reference_sph(args, world, rank, methods=SPH_METHODS):
    """The same SPH workloads through the reference's SPH kernels replayed by the harness."""
    from oracle import reference
    from physica_b200 import sph, scenes
    out = {"unit": UNIT, "config": {"workload": SPH_WORKLOAD, "l2": "flushed between timed steps (256 MiB write)"}}
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    steps = max(3, min(args.steps, 8))
    for name in methods:
        sc = scenes.sph_large(seed=6 + rank, method=name)
        ref = reference.ReferenceSPH(sc, int(sph.Method[name]))
        x = torch.from_numpy(sc.positions).cuda().contiguous()
        v = torch.from_numpy(sc.velocities).cuda().contiguous()
        warm = (torch.zeros(sc.count, device="cuda"), torch.zeros(sc.count, device="cuda"))
        warm_out = (torch.zeros(sc.count, device="cuda"), torch.zeros(sc.count, device="cuda"))
        h = {"x": x, "v": v, "xo": torch.zeros_like(x), "vo": torch.zeros_like(v), "k": 0, "w": warm, "wo": warm_out}
        torch.cuda.synchronize()

        def step():
            ref.forward_step(h["x"], h["v"], h["xo"], h["vo"], h["k"], warm=h["w"], warm_out=h["wo"], synchronize=False)
            h["x"], h["xo"], h["v"], h["vo"], h["w"], h["wo"] = h["xo"], h["x"], h["vo"], h["v"], h["wo"], h["w"]
            h["k"] += 1

        ms, _ = timed(step, steps, args.warmup, world, torch.cuda.ExternalStream(ref.stream), flush)
        ms_per_step = max_over_ranks(ms, world) / steps
        out[name] = {"value": round(world * sc.count / (ms_per_step * 1e-3), 1), "ms_per_step": round(ms_per_step, 4)}
        ref.close()
        torch.cuda.synchronize()
        if not args.no_grad:
            out[name]["gradient_ms_per_step"] = round(reference_sph_gradient_ms(args, world, sc, name), 4)
            out[name]["tangent_ms_per_step"] = round(reference_sph_tangent_ms(args, world, sc, name), 4)
    return out


def reference_sph_gradient_ms(args, world, sc, name):
    """The reference's differentiable SPH substep and its vjp_step (checkpoint recomputation
    included), per step in ms."""
    from oracle import reference
    from physica_b200 import sph
    n = sc.count
    ref = reference.ReferenceSPH(sc, int(sph.Method[name]), differentiable=True)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    z = lambda: torch.zeros(n, device="cuda")
    warm, warm_out = (z(), z()), (z(), z())
    z3 = lambda: torch.zeros((3, n), dtype=torch.float64, device="cuda")
    na = {"positions": torch.ones((3, n), dtype=torch.float64, device="cuda"), "velocities": z3()}
    prev = {"positions": z3(), "velocities": z3()}
    ctrl = z3()
    q = {k: torch.zeros(n, dtype=torch.float64, device="cuda") for k in sph.PARAMETER_NAMES}
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step():
        ref.forward_step(x, v, xo, vo, 0, warm=warm, warm_out=warm_out, synchronize=False)
        ref.vjp_step(x, v, na, prev, ctrl, q, 0)

    steps = max(3, min(args.steps, 5))
    ms, _ = timed(step, steps, 3, world, torch.cuda.ExternalStream(ref.stream), flush)
    ref.close()
    torch.cuda.synchronize()
    return max_over_ranks(ms, world) / steps


def cpu_baseline(sc):
    """FP64 host oracle on all host cores (the reference's PBF has no CPU path):
    - consecutive substeps of the same 1M workload from its initial state until at least 10 s of
      CPU work (at most 4 substeps): the reported value;
    - the 32,768-particle dam break (4 iterations) run for its full 100 substeps.
    Returns the baseline, the oracle's first 1M substep and its 32k state after 100 substeps (for
    the oracle-error check)."""
    from oracle import oracle
    x, v = sc.positions, sc.velocities
    first = None
    steps, t0 = 0, time.perf_counter()
    while steps < 4 and (steps == 0 or time.perf_counter() - t0 < 10.0):
        x, v = oracle.forward_step(sc, x, v, step_index=steps)
        if first is None:
            first = (x, v)
        steps += 1
    dt = time.perf_counter() - t0
    from physica_b200 import scenes
    small = scenes.plain_small()
    xs, vs = small.positions, small.velocities
    t1 = time.perf_counter()
    for k in range(100):
        xs, vs = oracle.forward_step(small, xs, vs, step_index=k)
    dt_small = time.perf_counter() - t1
    out = {"value": round(steps * sc.count / dt, 1), "unit": UNIT, "cores": oracle.thread_count(), "kind": "port",
           "sample": f"{steps} consecutive substeps of the 1,048,576-particle workload from rest "
                     f"(FP64 OpenMP oracle, {dt:.2f} s)",
           "dam_break_32k_100_steps": {"value": round(100 * small.count / dt_small, 1), "unit": UNIT,
                                       "seconds": round(dt_small, 2),
                                       "sample": "the 32,768-particle dam break (32x32x32 lattice, 4 iterations) for "
                                                 "its full 100 substeps (FP64 OpenMP oracle)"}}
    return out, first, (xs, vs)


def _errors(x, v, xo, vo, h, dt):
    """max |x - x_oracle| / h and max |v - v_oracle| * dt / h of FP32 (3, N) results against FP64 ones."""
    ex = float(np.abs(x.astype(np.float64) - xo).max()) / h if x.size else 0.0
    ev = float(np.abs(v.astype(np.float64) - vo).max()) * dt / h if v.size else 0.0
    return {"max_dx_over_h": float(f"{ex:.3e}"), "max_dv_dt_over_h": float(f"{ev:.3e}")}


def oracle_errors(sc_large, first_large, small_100):
    """Error of this library's FP32 substep against the FP64 host oracle for every configuration.

    One substep from each configuration's initial state (the dam break is chaotic, so longer runs
    measure the divergence of two roundings, not an error; the 32k run's 100-substep divergence is
    given beside its one-step error).  Batched configurations check a stated subset of their scenes;
    the differentiable ones also give the relative max-norm error of the one-step adjoint of the
    target-cloud loss with respect to the initial velocities."""
    from oracle import oracle
    from physica_b200 import pbf, scenes
    out = {}

    def one(sc, mode=pbf.ExecutionMode.forward):
        solver, state, control, params = pbf.solver_for_scene(sc, mode=mode)
        cache = solver.allocate_step_cache()
        nxt = solver.allocate_state()
        solver.forward_step(state, control, params, nxt, cache)
        torch.cuda.synchronize()
        return solver, state, control, params, cache, nxt

    sc = sc_large
    *_, nxt = one(sc)
    out["dam_break_1m"] = {**_errors(nxt.positions.cpu().numpy(), nxt.velocities.cpu().numpy(), *first_large,
                                     sc.support_radius, sc.time_step), "substeps": 1}
    small = scenes.plain_small()
    solver, state, control, params, cache, nxt = one(small)
    x1, v1 = oracle.forward_step(small, small.positions, small.velocities)
    e = _errors(nxt.positions.cpu().numpy(), nxt.velocities.cpu().numpy(), x1, v1, small.support_radius, small.time_step)
    cur, other = nxt, solver.allocate_state()
    for _ in range(99):
        solver.forward_step(cur, control, params, other, cache)
        cur, other = other, cur
    torch.cuda.synchronize()
    e["after_100_substeps"] = _errors(cur.positions.cpu().numpy(), cur.velocities.cpu().numpy(), *small_100,
                                      small.support_radius, small.time_step)
    out["dam_break_32k"] = {**e, "substeps": 1}

    def with_adjoint(sc):
        solver, state, control, params, cache, nxt = one(sc, pbf.ExecutionMode.differentiable)
        n = sc.count
        x1 = nxt.positions.double()
        wx = (x1 - torch.from_numpy(sc.targets).cuda().double()) * (2.0 / n)
        na = pbf.StateAdjoint(wx, torch.zeros_like(wx))
        pa, ca, qa = solver.allocate_state_adjoint(), solver.allocate_control_adjoint(), solver.allocate_parameter_adjoint()
        solver.vjp_step(state, control, params, nxt, cache, na, pa, ca, qa)
        torch.cuda.synchronize()
        xo, vo = oracle.forward_step(sc, sc.positions, sc.velocities)
        e = _errors(nxt.positions.cpu().numpy(), nxt.velocities.cpu().numpy(), xo, vo, sc.support_radius, sc.time_step)
        adj = oracle.vjp_step(sc, sc.positions, sc.velocities, wx.cpu().numpy(), np.zeros((3, n)))
        got = pa.velocities.cpu().numpy()
        e["adjoint_velocity_rel"] = float(f"{np.abs(got - adj['velocity']).max() / np.abs(adj['velocity']).max():.3e}")
        return e

    out["differentiable_64k"] = {**with_adjoint(scenes.differentiable()), "substeps": 1}
    subset = list(range(0, 256, 32))
    scs = scenes.batched_forward()
    batch, state, control, params = pbf.batch_for_scenes(scs)
    nxt = batch.allocate_state()
    batch.forward_step(state, control, params, nxt)
    torch.cuda.synchronize()
    worst = {"max_dx_over_h": 0.0, "max_dv_dt_over_h": 0.0}
    for k in subset:
        r = batch.particle_range(k)
        xo, vo = oracle.forward_step(scs[k], scs[k].positions, scs[k].velocities)
        e = _errors(nxt.positions[:, r].cpu().numpy(), nxt.velocities[:, r].cpu().numpy(), xo, vo,
                    scs[k].support_radius, scs[k].time_step)
        worst = {q: max(worst[q], e[q]) for q in worst}
    out["batched_forward_256"] = {**worst, "substeps": 1, "scenes_checked": subset}
    del batch, state, control, params, nxt
    adj_subset = [0, 11, 22, 31]
    scs = scenes.batched_adjoint()
    worst = {"max_dx_over_h": 0.0, "max_dv_dt_over_h": 0.0, "adjoint_velocity_rel": 0.0}
    for k in adj_subset:   # each checked scene through a one-scene differentiable solver of the same scene
        e = with_adjoint(scs[k])
        worst = {q: max(worst[q], e[q]) for q in worst}
    out["batched_adjoint_32"] = {**worst, "substeps": 1, "scenes_checked": adj_subset}
    return out


# --------------------------------------------------------------------------- reference arm
def bench_reference(args, world, rank):
    from oracle import reference
    from physica_b200 import scenes
    if not reference.available():
        return {"impl": "reference", "unavailable": "reference kernels not built (oracle/_ref/libpbf_ref.so missing)"}
    sc = scenes.plain_large(seed=2 + rank)
    n = sc.count
    ref = reference.ReferencePBF(sc)
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    stream = torch.cuda.ExternalStream(ref.stream)
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    holder = {"x": x, "v": v, "xo": xo, "vo": vo, "k": 0}
    torch.cuda.synchronize()

    def step():
        ref.forward_step(holder["x"], holder["v"], holder["xo"], holder["vo"], holder["k"], synchronize=False)
        holder["x"], holder["xo"] = holder["xo"], holder["x"]
        holder["v"], holder["vo"] = holder["vo"], holder["v"]
        holder["k"] += 1

    clk = Clocks(torch.cuda.current_device())
    ms, wall = timed(step, args.steps, args.warmup, world, stream, flush, clk)
    ms_max = max_over_ranks(ms, world)
    ms_per_step = ms_max / args.steps
    value = world * n / (ms_per_step * 1e-3)
    grad = None if args.no_grad else bench_reference_grad(world, rank)
    tangent = None if args.no_grad else reference_tangent_ms(args, world, sc)
    batched = None if args.no_batch else bench_reference_batch(args, world, rank)
    sph_family = None if args.no_sph else bench_reference_sph(args, world, rank)
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded jittered-lattice dam break)",
        "config": {"workload": "dam_break_1m: 1,048,576 particles (128x64x128 lattice, spacing 0.5h, h=0.025), "
                               "box [0,4]^3, 8 Jacobi iterations, dt=1/120, XSPH c=0.01, vorticity eps=1e-4",
                   "particles_per_gpu": n, "replicas": world, "l2": "flushed between timed steps (256 MiB write)",
                   "wall_s": round(wall, 3)},
        "cpu_baseline": None,
        "reference_arm": {"device": "cuda (the same B200)", "kind": "reference",
                          "sample": "the reference's own CUDA PBF kernels (pbf.cu, density.cu, neighborhood.cu, domain.cu "
                                    "compiled from its sources) replaying PBF::forward_step; the reference has no CPU "
                                    "implementation of this path, so this line carries no CPU figure"},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary(), "grad_steps_per_s": grad, "tangent_ms_per_step": tangent, "batched_scenes": batched,
        "sph_family": sph_family,
    }


def bench_reference_batch(args, world, rank):
    """The 256-scene batched workload through the reference: one reference solver per scene, each on
    its own stream as the reference's solvers are, stepped in turn (the reference has no batched form)."""
    from oracle import reference
    from physica_b200 import scenes
    scs = scenes.batched_forward(seed=4 + rank)
    total = sum(s.count for s in scs)
    entries = []
    for sc in scs:
        ref = reference.ReferencePBF(sc)
        x = torch.from_numpy(sc.positions).cuda().contiguous()
        v = torch.from_numpy(sc.velocities).cuda().contiguous()
        entries.append({"ref": ref, "x": x, "v": v, "xo": torch.zeros_like(x), "vo": torch.zeros_like(v), "k": 0})
    torch.cuda.synchronize()

    def step():
        for e in entries:
            e["ref"].forward_step(e["x"], e["v"], e["xo"], e["vo"], e["k"], synchronize=False)
            e["x"], e["xo"] = e["xo"], e["x"]
            e["v"], e["vo"] = e["vo"], e["v"]
            e["k"] += 1

    # each reference solver owns a non-blocking stream: the timed window opens with an event on the
    # first stream that every other stream waits on, and closes after the first stream waits on all
    streams = [torch.cuda.ExternalStream(e["ref"].stream) for e in entries]
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    steps = max(3, min(args.steps, 10))
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    barrier(world)
    total_ms = 0.0
    for _ in range(steps):
        flush.add_(1.0)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(streams[0])
        for st in streams[1:]:
            st.wait_event(a)
        step()
        for st in streams[1:]:
            done = torch.cuda.Event()
            done.record(st)
            streams[0].wait_event(done)
        b.record(streams[0])
        b.synchronize()
        total_ms += a.elapsed_time(b)
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(total_ms, world) / steps
    return {"unit": UNIT, "per_scene_solvers": round(world * total / (ms * 1e-3), 1), "per_scene_ms_per_step": round(ms, 4),
            "config": {"workload": "batched_forward_256: 256 dam-break scenes, counts log-uniform in [2048, 65536], "
                                   "4 iterations", "particles_per_gpu": total, "scenes_per_gpu": len(scs)}}


def reference_tangent_ms(args, world, sc):
    """The same differentiable substep and jvp_step through the reference's kernels, per step in ms."""
    from oracle import reference
    ref = reference.ReferencePBF(sc, differentiable=True)
    n = sc.count
    x = torch.from_numpy(sc.positions).cuda().contiguous()
    v = torch.from_numpy(sc.velocities).cuda().contiguous()
    xo, vo = torch.zeros_like(x), torch.zeros_like(v)
    tangent = {"positions": torch.ones((3, n), dtype=torch.float32, device="cuda"),
               "velocities": torch.zeros((3, n), dtype=torch.float32, device="cuda")}
    next_tangent = {k: torch.zeros_like(t) for k, t in tangent.items()}
    control_tangent = torch.zeros((3, n), dtype=torch.float32, device="cuda")
    names = ("masses", "rest_densities", "relaxation", "artificial_pressure_strength", "artificial_pressure_exponent",
             "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")
    param_tangent = {k: torch.zeros(n, dtype=torch.float32, device="cuda") for k in names}
    stream = torch.cuda.ExternalStream(ref.stream)
    flush = torch.zeros(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    def step():
        ref.forward_step(x, v, xo, vo, 0, synchronize=False)
        ref.jvp_step(x, v, tangent, control_tangent, param_tangent, next_tangent, synchronize=False)

    steps = max(3, min(args.steps, 5))
    ms, _ = timed(step, steps, 3, world, stream, flush)
    ref.close()
    torch.cuda.synchronize()
    return round(max_over_ranks(ms, world) / steps, 4)


def bench_reference_grad(world, rank):
    """The same 64k rollout through the reference's vjp_step: one harness (solver + cache) per step of a segment."""
    from oracle import reference
    from physica_b200 import scenes
    sc = scenes.differentiable(seed=3 + rank)
    steps, every = 20, 10
    refs = [reference.ReferencePBF(sc, checkpoint_interval=2, differentiable=True) for _ in range(every)]
    dev = "cuda"
    n = sc.count
    names = ("masses", "rest_densities", "relaxation", "artificial_pressure_strength", "artificial_pressure_exponent",
             "artificial_pressure_radius", "xsph_viscosity", "vorticity_confinement")
    targets = torch.from_numpy(sc.targets).cuda()

    def run():
        x = torch.from_numpy(sc.positions).to(dev).contiguous()
        v = torch.from_numpy(sc.velocities).to(dev).contiguous()
        checkpoints = []
        for k in range(steps):
            if k % every == 0:
                checkpoints.append((x.clone(), v.clone()))
            xo, vo = torch.empty_like(x), torch.empty_like(v)
            refs[k % every].forward_step(x, v, xo, vo, k)
            x, v = xo, vo
        adj = {"positions": (x.double() - targets.double()) * (2.0 / n),
               "velocities": torch.zeros((3, n), dtype=torch.float64, device=dev)}
        pa = {k: torch.zeros(n, dtype=torch.float64, device=dev) for k in names}
        ctrl = torch.zeros((3, n), dtype=torch.float64, device=dev)
        for seg in reversed(range(len(checkpoints))):
            xs, vs = [checkpoints[seg][0]], [checkpoints[seg][1]]
            begin = seg * every
            for k in range(begin, min(begin + every, steps)):
                xo, vo = torch.empty_like(xs[-1]), torch.empty_like(vs[-1])
                refs[k - begin].forward_step(xs[-1], vs[-1], xo, vo, k)
                xs.append(xo)
                vs.append(vo)
            for k in reversed(range(begin, min(begin + every, steps))):
                j = k - begin
                prev = {"positions": torch.zeros((3, n), dtype=torch.float64, device=dev),
                        "velocities": torch.zeros((3, n), dtype=torch.float64, device=dev)}
                refs[j].vjp_step(xs[j], vs[j], adj, prev, ctrl, pa)
                adj = prev
        torch.cuda.synchronize()

    run()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run()
    dt = max_over_ranks(time.perf_counter() - t0, world)
    return {"value": round(world * steps / dt, 3), "unit": "grad-steps/s",
            "config": {"workload": "differentiable_64k", "rollout_steps": steps, "trajectory_checkpoint_every": every,
                       "in_step_checkpoint_interval": 2}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-grad", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-sph", action="store_true", help="skip the SPH family's substeps")
    ap.add_argument("--no-late", action="store_true", help="skip the window timed after substep 100 (profiling)")
    ap.add_argument("--sph-only", default="", help="time only these SPH methods (comma list, e.g. pcisph) and print "
                                                   "their line (profiling)")
    ap.add_argument("--grad-only", action="store_true", help="time only the 64k differentiable rollout and print its "
                                                             "line (profiling)")
    ap.add_argument("--tangent-only", action="store_true", help="time only the 1M differentiable substep + jvp_step "
                                                                "and print its line (profiling)")
    ap.add_argument("--batch-grad-only", action="store_true", help="time only the 32-scene batched rollout against "
                                                                   "one rollout per scene and print its line (profiling)")
    ap.add_argument("--launch-shape", default="", help="fixed list-scan variant, its block size and optionally the "
                                                        "gather passes' block size, e.g. per_lane:128 or per_lane:128:32 "
                                                        "(gather passes at 128 unless given; default: autotuned)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = setup_dist()
    if args.sph_only:
        methods = tuple(m for m in args.sph_only.split(",") if m)
        run = bench_reference_sph if args.impl == "reference" else bench_sph
        out = {"impl": args.impl, "sph_family": run(args, world, rank, methods)}
    elif args.tangent_only:
        from physica_b200 import scenes
        sc = scenes.plain_large(seed=2 + rank)
        run = reference_tangent_ms if args.impl == "reference" else tangent_ms
        out = {"impl": args.impl, "tangent_ms_per_step": run(args, world, sc)}
    elif args.batch_grad_only:   # the reference has no batched form
        out = {"impl": args.impl,
               "batched_grad_steps_per_s": None if args.impl == "reference" else bench_batch_grad(args, world, rank)}
    elif args.grad_only:
        out = {"impl": args.impl,
               "grad_steps_per_s": bench_reference_grad(world, rank) if args.impl == "reference" else bench_grad(args, world, rank)}
    elif args.impl == "reference":
        out = bench_reference(args, world, rank)
    else:
        out = bench_b200(args, world, rank)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
