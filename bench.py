#!/usr/bin/env python
"""Benchmark: implicit time steps of 256^3 TVD convection-diffusion on one B200.

Workload (one "step" = one implicit Euler step of the reference's driver loop:
Build, BiCGStab2 solve to a 1e-10 relative residual, CopyTo, ExchangeHaloCells,
CopyDataVectorsToOldTimeStep): periodic unit cube, 256^3 cells, FP64,
D = 1e-4, divergence-free seeded velocity (cell Peclet 5, CFL 0.5), van Leer
TVD by deferred correction, Jacobi-preconditioned BiCGStab(2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dare|reference]

Prints one JSON line.  ``value`` is steps/s with every input resident in HBM;
``e2e`` is the same metric through the public API with the field uploaded from
and downloaded to pinned host memory every step.  Under torchrun (N > 1) each
rank runs an independent replica (the path is not sharded here), timing is
the max over ranks and ``value`` counts the steps of all ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "implicit steps/s & time-to-1e-10 residual: learned vs plain BiCGStab2, 1 B200"
UNIT = "steps/s"
# Algorithmic bytes per cell and launch (FP64, each operand streamed once; the
# SpMV inputs at the 6 neighbours come from cache).
BYTES_PER_CELL = {
    "assemble": 8 + 8 + 24 + 56 + 8 + 8,   # phi, phi_old, 3 face velocities; 7 diagonals, rhs, x0
    "step1": 88,    # r, u, 6 off-diagonals, r_hat; u', v
    "step2": 88,    # r, v, 6 off-diagonals, r_hat; r', s
    "step3": 88,    # s, v, 6 off-diagonals, r_hat; v', w
    "step4": 104,   # s, w, 6 off-diagonals, r', v'; r'', s', t
    "step5": 96,    # x, r'', s', t, u', r', v', w, r_hat; x, r, u
}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["dare", "reference"], default="dare")
    ap.add_argument("--n", "--cells-per-side", dest="n", type=int, default=256,
                    help="cells per side (--cells-per-side under torchrun, whose parser claims --n)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-steps", type=int, default=2,
                    help="implicit steps of the CPU oracle: the cpu_baseline sample and the parity check")
    ap.add_argument("--profile-steps", type=int, default=3,
                    help="untimed steps with per-kernel CUDA events (roofline.kernels)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", choices=["tvd", "gauss64", "hetero", "batched", "unet"], default="tvd",
                    help="tvd: the headline 256^3 line; the others print their own measurement line")
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner comparison")
    ap.add_argument("--no-slabs", action="store_true", help="skip the slab comparison")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 64^3 trajectory, 512^3 mixed-precision and 4096-box batch measurements")
    ap.add_argument("--learn-operators", type=int, default=64,
                    help="128^3 operators of the training distribution the preconditioner is trained on")
    ap.add_argument("--learn-steps", type=int, default=76,
                    help="implicit steps per training operator (each gives the plain solver's iterates as pairs)")
    return ap.parse_args(argv)


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, interval_ms: int = 50):
        self.path = tempfile.mktemp(prefix="dare_clocks_", suffix=".csv")
        self.proc = None
        self.skip = 0
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-i",
                 str(gpu_index), "-lms", str(interval_ms)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi takes a while to start: wait (at most 5 s) for its first
        # sample, so that sampling runs before the timed region begins
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.01)

    def _complete_lines(self) -> list:
        with open(self.path) as fh:
            return [line for line in fh if line.endswith("\n")]

    def mark(self):
        """Call right before the timed region: earlier samples are not counted."""
        if self.proc is not None:
            self.skip = len(self._complete_lines())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self._complete_lines()[self.skip:]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


NCU_NAMES = {"assemble": "k_assemble3", "step1": "k_march<FStep1>", "step2": "k_march<FStep2>",
             "step3": "k_march<FStep3>", "step4": "k_march<FStep4>", "step5": "k_step5"}


def ncu_traffic(kernel: str, n: int):
    """DRAM bytes of one launch (dram__bytes_read.sum + dram__bytes_write.sum)
    from the committed ncu summary profiles/traffic.json, with where the
    figure comes from: a capture of one launch at this grid size when the
    summary holds one, else per-cell figures of a smaller capture scaled by
    the cell count (on small grids part of the writes stay in L2, so a
    scaled figure understates DRAM traffic)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            t = json.load(fh)
    except Exception:
        return None, None
    name = NCU_NAMES[kernel]
    for cap in t.get("captures", []):
        if cap.get("cells") == n ** 3 and name in cap.get("kernels", {}):
            k = cap["kernels"][name]
            return k["read_bytes"] + k["write_bytes"], f"ncu, one launch at {cap['grid']}"
    for cap in t.get("captures", []):
        if name in cap.get("kernels", {}):
            k = cap["kernels"][name]
            return ((k["read_bytes"] + k["write_bytes"]) * n ** 3 / cap["cells"],
                    f"ncu at {cap['grid']}, scaled by cells")
    return None, None


# ----------------------------------------------------------------------------
# CPU (oracle) arm: the reference's algorithm restated on the host cores
# ----------------------------------------------------------------------------
# The reference's own code is built as oracle/_ref (its assembly and
# BiCGStab2, checked bit for bit against the oracle) and is the CPU baseline
# of the 64^3 diffusion workload under 'configs'.  It cannot run this one.
REF_CANNOT_RUN = ("the reference's own code (oracle/_ref) cannot run this workload: its face-velocity TVD "
                  "constructor does not compile (TVD_Cartesian.inl:34 assigns a Vector<1> to a scalar), and "
                  "the divergence-free velocity varies per face")


def cpu_steps(case, steps: int, n: int):
    from oracle import oracle as O
    og = O.make_grid(3, case["n"], case["size"], 2, case["periodic"])
    fv = [np.ascontiguousarray(a) for a in case["face_vel"]]
    desc = O.AssemblyDesc(og, dt=case["dt"], D=case["D"], face_vel=fv, limiter=O.LIM_VANLEER)
    phi = np.ascontiguousarray(case["phi0"].reshape(-1)).copy()
    old = phi.copy()
    times, iters = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        diag, rhs, mask = O.assemble(desc, phi, old)
        rp, cols, vals = O.export_csr(og, diag, mask)
        x0 = O.field_to_vector(og, phi)
        x, info = O.bicgstab2(rp, cols, vals, rhs, x0, 1e-10 * float(np.linalg.norm(rhs)), 5000)
        O.copy_to_field(og, x, phi)
        O.exchange_halo(og, phi)
        old[:] = phi
        times.append(time.perf_counter() - t0)
        iters.append(info["iters"])
        del diag, rp, cols, vals
    return times, iters, O.num_threads(), phi


def host_case(n, seed):
    from dare_b200 import workloads as W
    return W.tvd_convection_diffusion(n=n, seed=seed)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    case = host_case(args.n, args.seed)
    times, iters, cores, _ = cpu_steps(case, args.warmup + args.steps, args.n)
    timed = times[args.warmup:]
    total = sum(timed)
    value = len(timed) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded divergence-free velocity, smooth scalar)",
        "config": {"workload": f"TVD convection-diffusion {args.n}^3 periodic, van Leer, D=1e-4, Pe 5, CFL 0.5, "
                               "Jacobi-BiCGStab2 to 1e-10 relative", "cells": args.n ** 3},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{len(timed)} full implicit steps of the {args.n}^3 workload (CPU oracle: "
                                   "assembly, CSR build, BiCGStab2, copy back), OpenMP on all host threads",
                         "why_port": REF_CANNOT_RUN},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iterations_per_step": statistics.mean(iters),
        "parallelism": "one CPU run on rank 0's host (all its cores)",
        "value_scope": "one CPU run: the host's steps/s, not multiplied by n_gpus",
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
def run_dare(args):
    import torch

    import dare_b200 as D
    from dare_b200 import workloads as W
    from dare_b200.replicas import Replicas

    ranks = Replicas("nccl")
    rank, world, local = ranks.rank, ranks.world, ranks.local
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"

    n = args.n
    case = W.tvd_convection_diffusion(n=n, seed=args.seed, device=dev)
    ctx = D.Context(local)
    grid = D.Grid(ctx, case["n"], case["size"], 2, case["periodic"])
    field = D.Field(grid, 2)
    phi0 = case["phi0"].reshape(-1).cpu().numpy()
    field.upload(phi0, 0)
    field.upload(phi0, 1)
    system = D.MatrixSystem(grid)
    vel = [D.DeviceArray.from_tensor(case["face_vel"][d]) for d in range(3)]
    asm = D.Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(vel), limiter="VANLEER")
    solver = D.BiCGStab2(dict(_STEP_SOLVER))

    for _ in range(args.warmup):
        D.timestep(system, field, asm, solver)
    ctx.synchronize()

    barrier, max_over_ranks = ranks.barrier, ranks.max

    # the headline: the product path (iterations replayed from CUDA graphs,
    # no per-kernel events), exactly K steps between two barriers
    clocks = ClockSampler(local)
    launches0 = ctx.launch_count
    iters = []
    barrier()
    ctx.synchronize()
    clocks.mark()
    ctx.timer_start()
    for _ in range(args.steps):
        rep = D.timestep(system, field, asm, solver)
        iters.append(rep["iters"])
        if not rep["converged"]:
            raise RuntimeError(f"solve did not converge: {rep}")
    ms = ctx.timer_stop()
    barrier()
    clk = clocks.stop()
    launches = ctx.launch_count - launches0
    ms = max_over_ranks(ms)
    value = world * args.steps / (ms * 1e-3)

    # per-kernel durations: a separate, untimed pass of the same steps with a
    # CUDA event around every kernel (launched directly on the context's
    # stream); every iteration that ran is counted, the last one included
    ctx.set_profiling(True)
    ctx.reset_kernel_stats()
    prof_iters, true_res = [], None
    checked = D.BiCGStab2(dict(_SOLVER))       # the same solve, plus ||b - A x|| at its exit
    for _ in range(args.profile_steps):
        prep = D.timestep(system, field, asm, checked)
        prof_iters.append(prep["iters"])
        true_res = {"true_res_rel": prep["true_res_abs"] / prep["b_norm"], "res_rel": prep["res_abs"] / prep["b_norm"],
                    "of": "the last untimed profiling step"}
    ctx.synchronize()
    kstats = {}
    for name in BYTES_PER_CELL:
        tot, cnt = ctx.kernel_stats(name)
        if cnt:
            kstats[name] = {"ms_total": tot, "launches": cnt, "ms_avg": tot / cnt}
    ctx.set_profiling(False)
    dom = max(kstats, key=lambda k: kstats[k]["ms_total"]) if kstats else None
    peak, peak_kind = measured_peak_hbm()
    roofline = None
    if dom:
        algo = BYTES_PER_CELL[dom] * n ** 3
        achieved = algo / (kstats[dom]["ms_avg"] * 1e-3) / 1e9
        traffic, traffic_src = ncu_traffic(dom, n)
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                    "traffic_source": traffic_src, "algorithmic_bytes": algo,
                    "timing": f"CUDA events around each kernel over {args.profile_steps} untimed steps "
                              f"({sum(prof_iters)} iterations, every one counted)"}
        roofline["kernels"] = {k: {**v, "GBps": BYTES_PER_CELL[k] * n ** 3 / (v["ms_avg"] * 1e-3) / 1e9}
                               for k, v in kstats.items()}

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        # the field lives in pinned host memory: every step uploads it (both
        # time levels from it) and downloads the result.  The product entry
        # point pipelines one step's download with the next step's upload in
        # slices; the plain loop of single calls is timed beside it.
        host = torch.empty(grid.num_cells_ghosted, dtype=torch.float64, pin_memory=True).numpy()
        field.download(0, out=host)
        barrier()
        ctx.synchronize()
        ctx.timer_start()
        reps = D.timesteps_host(system, field, asm, solver, args.steps, host)
        ems = max_over_ranks(ctx.timer_stop())
        barrier()
        if not all(r["converged"] for r in reps):
            raise RuntimeError("a host-resident step did not converge")
        field.download(0, out=host)
        barrier()
        ctx.synchronize()
        ctx.timer_start()
        for _ in range(args.steps):
            field.upload(host, 0)
            field.copy_to_old()
            D.timestep(system, field, asm, solver)
            field.download(0, out=host)
        sms = max_over_ranks(ctx.timer_stop())
        barrier()
        nbytes = grid.num_cells_ghosted * 8
        e2e = {"value": world * args.steps / (ems * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes,
               "api": "dare_timesteps_host: each step's input from pinned host memory, its result back to it; "
                      "one step's download pipelined with the next step's upload in 16 slices",
               "unpipelined": {"value": world * args.steps / (sms * 1e-3),
                               "api": "per step dare_field_upload, dare_field_copy_to_old, dare_timestep, "
                                      "dare_field_download"}}

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        hcase = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in case.items() if k != "face_vel"}
        hcase["face_vel"] = [a.cpu().numpy() for a in case["face_vel"]]
        times, citers, cores, cpu_phi = cpu_steps(hcase, args.cpu_steps, n)
        cpu = {"value": len(times) / sum(times), "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{len(times)} full implicit steps of the same {n}^3 workload from the same initial "
                         f"field (CPU oracle, OpenMP), iterations {citers}", "why_port": REF_CANNOT_RUN}
        # parity at the full size: the same steps on the GPU from the same
        # initial field, final fields compared (internal and ghost cells)
        field.upload(phi0, 0)
        field.upload(phi0, 1)
        giters = [D.timestep(system, field, asm, solver)["iters"] for _ in range(args.cpu_steps)]
        gpu_phi = field.download(0)
        diff = gpu_phi - cpu_phi
        parity = {"steps": args.cpu_steps, "rel_l2": float(np.linalg.norm(diff) / np.linalg.norm(cpu_phi)),
                  "max_abs": float(np.abs(diff).max()), "iters_gpu": giters, "iters_cpu": citers,
                  "bar": "rel_l2 < 1e-9 (solutions at the same 1e-10 relative residual)"}

    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        # the other configurations of the workload family, each measured here
        # on the same device (one warm-up, then timed)
        configs = {"gauss64": measure_gauss64(D, ctx, args.seed),
                   "hetero512": measure_hetero(D, ctx, 512 if n >= 256 else 2 * n, args.seed),
                   "batched4096": measure_batched(D, ctx, 4096 if n >= 256 else 64, args.seed,
                                                  cpu_sample=16)}

    slabs = None
    if rank == 0 and world == 1 and not args.no_slabs:
        slabs = slab_comparison(D, ctx, system, field, asm, case, phi0, args)

    learned = None
    if rank == 0 and world == 1 and not args.no_learned:
        learned = learned_comparison(D, ctx, system, field, asm, n, args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded divergence-free velocity, smooth scalar in [0,1])",
            "config": {"workload": f"TVD convection-diffusion {n}^3 periodic, van Leer, D=1e-4, Pe 5, CFL 0.5, "
                                   "Jacobi-BiCGStab2 to 1e-10 relative",
                       "cells": n ** 3},
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (system ~3.6 GB per GPU)",
            "parity": parity,
            "time_to_residual_ms": ms / args.steps, "iterations_per_step": statistics.mean(iters),
            "cell_updates_per_s": value * n ** 3,
            "solver": "plain FP64 Jacobi-BiCGStab2 (value, e2e; iterations replayed from CUDA graphs; no true "
                      "residual at the exit, as the reference's solve); learned-preconditioned solve in 'learned'",
            "final_residual": true_res,
            "learned": learned,
            "slabs": slabs,
            "configs": configs,
            "gpu_launches": launches, "clocks": clk, "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def slab_comparison(D, ctx, system, field, asm, case, phi0, args, num_slabs=2, steps=2):
    """The same steps on slabs of i-planes (both on this device, run one after
    the other, planes exchanged by device copies) against the single grid
    from the same initial field: time per step and the final fields."""
    import torch
    field.upload(phi0, 0)
    field.upload(phi0, 1)
    single_iters = [D.timestep(system, field, asm, D.BiCGStab2(dict(_SOLVER)))["iters"] for _ in range(steps)]
    ref = field.download(0)
    sl = D.Slabs(system, num_slabs, 2)
    n0 = case["n"][0]
    keep, slab_asm = [], []
    for i0, i1 in sl.ranges:
        fx = case["face_vel"][0]
        fx = torch.cat([fx[i0:n0], fx[0:1]]) if (case["periodic"][0] and i1 == n0) else fx[i0:i1 + 1]
        arrs = [D.DeviceArray.from_tensor(fx), D.DeviceArray.from_tensor(case["face_vel"][1][i0:i1]),
                D.DeviceArray.from_tensor(case["face_vel"][2][i0:i1])]
        keep += arrs
        slab_asm.append(D.Assembly(dt=case["dt"], D=case["D"], face_vel=tuple(arrs), limiter="VANLEER"))
    solver = D.BiCGStab2(dict(_SOLVER))
    field.upload(phi0, 0)
    field.upload(phi0, 1)
    sl.scatter(field)
    sl.timestep(slab_asm, solver)          # captures the slab graphs
    sl.scatter(field)
    ctx.synchronize()
    ctx.timer_start()
    iters = [sl.timestep(slab_asm, solver)["iters"] for _ in range(steps)]
    ms = ctx.timer_stop()
    sl.gather(field)
    got = field.download(0)
    g = system.grid
    inner = lambda a: a.reshape(g.ghosted_shape)[2:-2, 2:-2, 2:-2]
    rel = float(np.linalg.norm(inner(got) - inner(ref)) / np.linalg.norm(inner(ref)))
    del sl
    return {"slabs": num_slabs, "steps": steps, "ms_per_step": ms / steps, "iters": iters,
            "iters_single_grid": single_iters, "rel_l2_vs_single_grid": rel,
            "setup": "all slabs on this one B200, launched one after the other; boundary planes cross by "
                     "device-to-device copies; the multi-GPU form (NCCL send/recv, all-reduce) is unmeasured "
                     "on hardware"}


_SOLVER = {"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1}
# The time-step loops' solver: the reference's BiCGStab2::Solve computes no
# true residual ||b - A x|| at its common exit (MatrixSystem/BiCGStab2.inl:
# 571-582), only at the tau = 0 exit (:407-424), which this solver keeps.
_STEP_SOLVER = dict(_SOLVER, compute_true_residual=0)


def _timed_solve(ctx, system, field, asm, fn, reps=2):
    """Assemble from the field and solve; the last of `reps` runs is reported
    (the first captures graphs and sizes workspaces)."""
    out = None
    for _ in range(reps):
        system.build(field, asm)
        ctx.synchronize()
        ctx.timer_start()
        rep = fn()
        ms = ctx.timer_stop()
        out = {"ms": ms, "iters": rep["iters"], "inner_iters": rep["inner_iters"],
               "refinements": rep["refinements"], "fallback_used": rep["fallback_used"],
               "converged": rep["converged"], "res_rel": rep["true_res_abs"] / rep["b_norm"]}
    return out


def learned_comparison(D, ctx, system, field, asm, n, args):
    """Time-to-1e-10 of one implicit step: plain FP64 Jacobi-BiCGStab2, the
    FP32-inner / FP64-refinement Jacobi solve, and the learned-preconditioned
    mixed-precision BiCGStab2 with the coarse-correction network
    N(u) = u + P U(R u).  The network is trained here, on the GPU, on the
    plain solver's (residual, error) pairs of 128^3 operators of the training
    distribution (constant or log-normal D, Pe in [1, 10], CFL 0.5), then
    evaluated on held-out 128^3 operators and, with the same weights, on this
    workload."""
    from dare_b200 import training
    out = {}
    t0 = time.perf_counter()
    m = 128
    net128 = D.LearnedPreconditioner(ctx, (m, m, m), seed=args.seed + 1, coarse=True)
    reps = training.train(net128, ctx, m, operators=args.learn_operators, steps_per_operator=args.learn_steps,
                          params=net128.train_params(steps=2, batch=4, lr=3e-4), seed=args.seed + 1000)
    out["training"] = {"grid": f"{m}^3 operators, network on {m // 2}^3 (coarse-correction form)",
                       "operators": args.learn_operators, "implicit_steps": len(reps),
                       "pairs": sum(r["pairs_added"] for r in reps), "adam_steps": sum(r["steps"] for r in reps),
                       "loss_first": reps[0]["loss_first"],
                       "loss_last_mean16": float(np.mean([r["loss_last"] for r in reps[-16:]])),
                       "wall_s": time.perf_counter() - t0}
    plain = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1})
    refine = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 5000, "tol_relative": 1},
                         precision="FP32_REFINE")
    ident128 = D.LearnedPreconditioner(ctx, (m, m, m), seed=args.seed + 1, coarse=True)
    held = []
    for seed in (args.seed + 9001, args.seed + 9002, args.seed + 9003, args.seed + 9004):
        op = training.Operator(ctx, training.sample_case(m, seed, "cuda:0"))
        row = {"peclet": op.case["peclet"], "heterogeneous_D": "cell_D" in op.case}
        for name, fn in (("plain_fp64", lambda: plain.solve(op.system)),
                         ("fp32_refine_jacobi", lambda: refine.solve(op.system)),
                         ("learned_untrained", lambda: ident128.solve(op.system, plain)),
                         ("learned", lambda: net128.solve(op.system, plain))):
            row[name] = _timed_solve(ctx, op.system, op.field, op.asm, fn)
        row["trained_beats_identity"] = row["learned"]["inner_iters"] < row["learned_untrained"]["inner_iters"]
        held.append(row)
        del op
    out["held_out_128"] = held
    out["trained_beats_identity_on_every_held_out"] = all(r["trained_beats_identity"] for r in held)
    net = D.LearnedPreconditioner(ctx, (n, n, n), seed=args.seed + 1, coarse=True)
    net.set_weights(net128.get_weights())
    res = {"grid": f"{n}^3 (this workload; network on {n // 2}^3, weights trained with {m}^3 operators)"}
    for name, fn in (("plain_fp64", lambda: plain.solve(system)),
                     ("fp32_refine_jacobi", lambda: refine.solve(system)),
                     ("learned", lambda: net.solve(system, plain))):
        res[name] = _timed_solve(ctx, system, field, asm, fn)
    res["learned_speedup_vs_plain"] = res["plain_fp64"]["ms"] / res["learned"]["ms"]
    res["learned_speedup_vs_fp32_refine"] = res["fp32_refine_jacobi"]["ms"] / res["learned"]["ms"]
    # one network application at this size (CUDA events, 20 applies)
    import torch
    u = torch.randn(n ** 3, device="cuda", dtype=torch.float32)
    z = torch.empty_like(u)
    net.apply(u.data_ptr(), z.data_ptr())
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(20):
        net.apply(u.data_ptr(), z.data_ptr())
    res["network_apply_ms"] = ctx.timer_stop() / 20
    out["bench_workload"] = res
    out["target_3x_met"] = res["learned_speedup_vs_plain"] >= 3.0
    return out


# ----------------------------------------------------------------------------
# the other configurations (reported beside the headline, not as it)
# ----------------------------------------------------------------------------
def _gpu_setup_field(D, ctx, case):
    grid = D.Grid(ctx, case["n"], case["size"], 2, case["periodic"])
    field = D.Field(grid, 2)
    return grid, field


def measure_gauss64(D, ctx, seed=0, warmup=1):
    """64^3 transient diffusion (Gaussian bump, Dirichlet x, Neumann elsewhere):
    10 implicit steps on the GPU against the oracle's loop from the same field."""
    from dare_b200 import workloads as W
    from oracle import oracle as O
    from tests.helpers import oracle_timeloop
    case = W.gaussian_diffusion(n=64, seed=seed, steps=10)
    grid, field = _gpu_setup_field(D, ctx, case)
    system = D.MatrixSystem(grid)
    for face, (kind, val) in case["bc"].items():
        system.set_bc(face, kind, val)
    asm = D.Assembly(dt=case["dt"], D=case["D"])
    solver = D.BiCGStab2(dict(_STEP_SOLVER))
    phi0 = np.ascontiguousarray(case["phi0"].reshape(-1))

    def trajectory():
        field.upload(phi0, 0)
        field.upload(phi0, 1)
        its = []
        ctx.synchronize()
        ctx.timer_start()
        for _ in range(case["steps"]):
            its.append(D.timestep(system, field, asm, solver)["iters"])
        return ctx.timer_stop(), its

    for _ in range(max(1, warmup)):
        trajectory()
    ms, its = trajectory()
    got = field.download(0)
    t0 = time.perf_counter()
    hist, oits = oracle_timeloop(case, case["steps"])
    cpu_s = time.perf_counter() - t0
    err = float(np.linalg.norm(got - hist[-1]) / np.linalg.norm(hist[-1]))
    port = {"value": case["steps"] / cpu_s, "unit": "steps/s", "cores": O.num_threads(), "kind": "port",
            "sample": "the whole 10-step loop, CPU oracle (OpenMP)"}
    out = {"workload": "gaussian diffusion 64^3, 10 implicit steps, Jacobi-BiCGStab2 1e-10",
           "metric": "implicit steps/s", "value": case["steps"] / (ms * 1e-3), "ms_total": ms,
           "iterations": its, "oracle_iterations": oits, "rel_l2_vs_oracle": err, "cpu_baseline": port}
    from oracle import ref as R
    if R.available():
        # the reference's own assembly and BiCGStab2 (its headers compiled
        # against single-rank MPI / Kokkos / Tpetra / Belos stand-ins), the
        # same loop; this workload needs no face fields, so the reference's
        # code runs it as stated
        from tests.helpers import ref_timeloop
        rhist, rits, rsec = ref_timeloop(case, case["steps"])
        out["cpu_port"] = port
        out["cpu_baseline"] = {"value": case["steps"] / rsec, "unit": "steps/s", "cores": O.num_threads(),
                               "kind": "reference",
                               "sample": "the whole 10-step loop, the reference's own assembly (per-cell MatrixBlock "
                                         "objects, OpenMP over cells) and BiCGStab2 (OpenMP vector kernels)"}
        out["reference_iterations"] = rits
        out["rel_l2_vs_reference"] = float(np.linalg.norm(got - rhist[-1]) / np.linalg.norm(rhist[-1]))
    return out


def run_gauss64(args):
    import dare_b200 as D
    print(json.dumps(measure_gauss64(D, D.Context(0), args.seed, args.warmup)), flush=True)
    return 0


def measure_hetero(D, ctx, n=512, seed=0, warmup=1, steps=2):
    """Heterogeneous-D TVD operator (log-normal D, box-filtered): FP64 plain vs
    FP32-inner / FP64-refinement per step, error of the latter vs the former."""
    import torch

    from dare_b200 import workloads as W
    dev = f"cuda:{torch.cuda.current_device()}"
    case = W.heterogeneous(n=n, seed=seed, device=dev)
    grid, field = _gpu_setup_field(D, ctx, case)
    phi0 = case["phi0"].reshape(-1).cpu().numpy()
    field.upload(phi0, 0)
    field.upload(phi0, 1)
    cell_D = case["cell_D"].contiguous()
    faceD = [D.DeviceArray.from_tensor(torch.empty(grid.face_shape(d), dtype=torch.float64, device=dev))
             for d in range(3)]
    D.face_average(grid, cell_D.data_ptr(), faceD)
    vel = [D.DeviceArray.from_tensor(case["face_vel"][d]) for d in range(3)]
    dt = case["dt"]
    del case, cell_D, phi0
    torch.cuda.empty_cache()
    system = D.MatrixSystem(grid)
    asm = D.Assembly(dt=dt, face_D=tuple(faceD), face_vel=tuple(vel))
    p64 = D.BiCGStab2(dict(_SOLVER))
    p32 = D.BiCGStab2(dict(_SOLVER), precision="FP32_REFINE")
    rows = []
    for step in range(warmup + steps):
        system.build(field, asm)
        ctx.synchronize()
        ctx.timer_start()
        r64 = p64.solve(system)
        t64 = ctx.timer_stop()
        x64 = system.solution()
        system.build(field, asm)
        ctx.synchronize()
        ctx.timer_start()
        r32 = p32.solve(system)
        t32 = ctx.timer_stop()
        x32 = system.solution()
        err = float(np.linalg.norm(x32 - x64) / np.linalg.norm(x64))
        del x64, x32
        system.copy_to(field)
        field.exchange_halo()
        field.copy_to_old()
        if step >= warmup:
            rows.append({"fp64_ms": t64, "fp64_iters": r64["iters"], "refine_ms": t32,
                         "refinements": r32["refinements"], "inner_iters": r32["inner_iters"],
                         "fallback": r32["fallback_used"], "rel_l2_vs_fp64": err,
                         "true_res_rel": r32["true_res_abs"] / r32["b_norm"]})
    # per-kernel CUDA events of the FP32 inner iterations: one more, untimed solve
    system.build(field, asm)
    ctx.set_profiling(True)
    ctx.reset_kernel_stats()
    p32.solve(system)
    ctx.synchronize()
    fp32_kernels = {}
    for name, bpc in (("fp32_step1", 44), ("fp32_step2", 44), ("fp32_step3", 44), ("fp32_step4", 52),
                      ("fp32_step5", 48)):
        tot, cnt = ctx.kernel_stats(name)
        if cnt:
            fp32_kernels[name] = {"launches": cnt, "ms_avg": tot / cnt, "bytes_per_cell": bpc,
                                  "GBps": bpc * n ** 3 / (tot / cnt * 1e-3) / 1e9}
    ctx.set_profiling(False)
    return {"workload": f"heterogeneous-D TVD convection-diffusion {n}^3 periodic, Pe 5 at median D",
            "fp32_kernels": fp32_kernels,
            "steps": rows,
            "fp64_ms_mean": statistics.mean(r["fp64_ms"] for r in rows),
            "refine_ms_mean": statistics.mean(r["refine_ms"] for r in rows)}


def run_hetero(args):
    import dare_b200 as D
    ctx = D.Context(0)
    print(json.dumps(measure_hetero(D, ctx, args.n, args.seed, args.warmup, args.steps)), flush=True)
    return 0


def run_unet(args):
    """The learned preconditioner's network alone: `--steps` timed applies of
    N at n^3 (seeded random weights) after `--warmup` untimed ones, and one
    training step (forward + backward + Adam, batch 4) when n <= 128."""
    import torch

    import dare_b200 as D
    n = args.n
    ctx = D.Context(0)
    net = D.LearnedPreconditioner(ctx, (n, n, n), seed=args.seed)
    rng = np.random.default_rng(args.seed)
    net.set_weights(rng.normal(0.0, 0.02, net.num_params).astype(np.float32))
    gen = torch.Generator(device="cuda").manual_seed(args.seed)
    u = torch.randn(n ** 3, device="cuda", generator=gen)
    z = torch.empty_like(u)
    for _ in range(max(1, args.warmup)):
        net.apply(u.data_ptr(), z.data_ptr())
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(args.steps):
        net.apply(u.data_ptr(), z.data_ptr())
    ms = ctx.timer_stop() / args.steps
    layers = D.LearnedPreconditioner.LAYERS
    flops = sum(2 * 27 * cin * cout * (n >> lev) ** 3 for _, lev, cin, cout in layers)
    out = {"workload": f"learned preconditioner apply z = u + U(u), {n}^3", "apply_ms": ms,
           "cells_per_s": n ** 3 / (ms * 1e-3), "useful_tflops": flops / (ms * 1e-3) / 1e12,
           "launch": {name: net.launch_info(i, 0) for i, (name, _, _, _) in enumerate(layers)}}
    if n <= 128:
        r = torch.randn(4, n ** 3, device="cuda", generator=gen)
        e = torch.randn(4, n ** 3, device="cuda", generator=gen)
        p = net.train_params()
        net.train_step(r.data_ptr(), e.data_ptr(), 4, p)
        ctx.synchronize()
        ctx.timer_start()
        net.train_step(r.data_ptr(), e.data_ptr(), 4, p)
        out["train_step_batch4_ms"] = ctx.timer_stop()
    print(json.dumps(out), flush=True)
    return 0


def measure_batched(D, ctx, count=4096, seed=0, warmup=3, steps=10, autotune=True, cpu_sample=64):
    """`count` independent diffusion boxes (sides 16-64), one implicit step
    each, one persistent launch; the CPU oracle on a bounded sample, scaled
    by cells."""
    from dare_b200 import workloads as W
    from oracle import oracle as O
    inst = W.batched_diffusion(count=count, seed=seed)
    cells = int(sum(np.prod(i["n"]) for i in inst))
    bt = D.Batch(ctx, inst)
    solver = D.BiCGStab2({"Convergence Tolerance": 1e-10, "Maximum Iterations": 10000, "tol_relative": 1})
    tuning = bt.autotune(solver) if autotune else None
    for _ in range(warmup):
        bt.zero_fields()
        bt.solve(solver, reports=False)
    times = []
    for _ in range(steps):
        bt.zero_fields()
        ctx.synchronize()
        ctx.timer_start()
        bt.solve(solver, reports=False)
        times.append(ctx.timer_stop())
    bt.zero_fields()
    reps = bt.solve(solver)
    its = [r["iters"] for r in reps]
    rng = np.random.default_rng(1)
    sample = rng.choice(len(inst), size=min(cpu_sample, len(inst)), replace=False)
    t0 = time.perf_counter()
    scells = 0
    for q in sample:
        ins = inst[q]
        g = O.make_grid(3, ins["n"], ins["size"], 2, (0, 0, 0))
        z = np.zeros(int(np.prod(O.ghosted_shape(g))))
        diag, rhs, mask = O.assemble(O.AssemblyDesc(g, dt=ins["dt"], D=ins["D"], bc=ins["bc"]), z, z)
        rp, cols, vals = O.export_csr(g, diag, mask)
        O.bicgstab2(rp, cols, vals, rhs, np.zeros(len(rhs)), 1e-10 * np.linalg.norm(rhs), 10000)
        scells += int(np.prod(ins["n"]))
    cpu_s = (time.perf_counter() - t0) * cells / scells
    ms = statistics.median(times)
    return {"workload": f"{len(inst)} diffusion boxes, sides 16-64, one implicit step each, "
                        "Jacobi-BiCGStab2 1e-10, one persistent launch",
            "cells": cells, "ms_per_batch": ms, "ms_all": times, "cell_steps_per_s": cells / (ms * 1e-3),
            "converged": sum(r["converged"] for r in reps), "iters_min": min(its), "iters_max": max(its),
            "iters_mean": statistics.mean(its), "tuning": tuning,
            "cpu_baseline": {"value_s_per_batch": cpu_s, "cores": O.num_threads(), "kind": "port",
                             "sample": f"{len(sample)} instances, scaled by cells"}}


def run_batched(args):
    import dare_b200 as D
    ctx = D.Context(0)
    print(json.dumps(measure_batched(D, ctx, args.batch, args.seed, args.warmup, args.steps,
                                     not args.no_autotune)), flush=True)
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "gauss64":
        return run_gauss64(args)
    if args.workload == "hetero":
        return run_hetero(args)
    if args.workload == "unet":
        return run_unet(args)
    if args.workload == "batched":
        return run_batched(args)
    return run_dare(args)


if __name__ == "__main__":
    sys.exit(main())
