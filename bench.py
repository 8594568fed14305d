"""Richards timesteps/s at 13.1M cells (512x512x50 heterogeneous box):
mixed-precision GPU solver against the plain FP64 GPU form, with the HBM
roofline of the dominant kernel and the reference CPU build beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --profile [--size NX,NY,NZ] --steps 1 --warmup 3

--profile runs only the mixed solve and brackets its timed steps with
cudaProfilerStart/Stop, for `ncu --profile-from-start off`; its line is a
profiling run, not a bench value.

A step is one implicit timestep (a full KINSOL Newton-Krylov solve) of the
workload, dt = 0.05 h.  Under torchrun (N > 1) every rank solves its own
replica of the workload (the path does not shard on this build: "replicas
only"); value = timesteps of all ranks / max wall time over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Richards steps/s @13M cells: mixed vs FP64 on B200 at ≤1e-8 rel err; HBM %"
NX, NY, NZ = 512, 512, 50
# The mixed-precision form the headline runs: FP64 Newton/Arnoldi, FP32
# multigrid arithmetic on the symmetrically diagonal-scaled operator stored in
# FP16 ("mixed16"); the all-FP32 multigrid ("mixed") is timed beside it.
HEADLINE = "mixed16"
# DRAM bytes (read + write) per cell of one k_rb_sweep2 launch of the headline
# form, from the ncu capture summarised in
# profiles/k_rb_sweep2_hetero_384x384x50_mixed16.md
RB_SWEEP_DRAM_BYTES_PER_CELL = 10.51


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(
            ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
             "--format=csv,noheader,nounits", "-lms", "200"],
            stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference CPU arm
# ---------------------------------------------------------------------------
def _workloads():
    from parflow_b200 import configs
    from parflow_b200.problem import BC_OVERLAND, BC_OVERLAND_DIFF

    return {
        # the bench line: heterogeneous box, 13.1M cells
        "hetero": {
            "build": lambda nx, ny, nz, nsteps: configs.hetero(nx=nx, ny=ny, nz=nz, nsteps=nsteps),
            "dims": (NX, NY, NZ), "sample": (128, 128, 50),
            "label": "hetero 512x512x50 (13.1M cells)",
            "config": {"dt_h": 0.05, "sigma_lnK": 1.5, "corr_cells": [32, 32, 4]}},
        # config 1: hillslope with kinematic overland flow, terrain-following grid
        "overland": {
            "build": lambda nx, ny, nz, nsteps: configs.overland(nx=nx, ny=ny, nz=nz, nsteps=nsteps),
            "dims": (256, 256, 20), "sample": (64, 64, 20),
            "label": "overland hillslope 256x256x20 (1.31M cells), kinematic overland flow, "
                     "terrain-following grid, rain 2 h on / 2 h off",
            "config": {"dt_h": 0.25, "dx_m": 10.0, "dz_m": 0.2, "mannings": 5.5e-5}},
        # config 1 with the OverlandFlow patch type (overlandflow_eval.c)
        "overland_flow": {
            "build": lambda nx, ny, nz, nsteps: configs.overland(nx=nx, ny=ny, nz=nz, nsteps=nsteps,
                                                                kind=BC_OVERLAND),
            "dims": (256, 256, 20), "sample": (64, 64, 20),
            "label": "overland hillslope 256x256x20 (1.31M cells), OverlandFlow overland flow, "
                     "terrain-following grid, rain 2 h on / 2 h off",
            "config": {"dt_h": 0.25, "dx_m": 10.0, "dz_m": 0.2, "mannings": 5.5e-5}},
        # config 1 with diffusive-wave routing (overlandflow_eval_diffusive.c)
        "overland_diff": {
            "build": lambda nx, ny, nz, nsteps: configs.overland(nx=nx, ny=ny, nz=nz, nsteps=nsteps,
                                                                kind=BC_OVERLAND_DIFF),
            "dims": (256, 256, 20), "sample": (64, 64, 20),
            "label": "overland hillslope 256x256x20 (1.31M cells), diffusive-wave overland flow, "
                     "terrain-following grid, rain 2 h on / 2 h off",
            "config": {"dt_h": 0.25, "dx_m": 10.0, "dz_m": 0.2, "mannings": 5.5e-5}},
    }


def _config(wl: dict, world: int) -> dict:
    """The workload's config as both arms print it (same keys, same values)."""
    cells = int(np.prod(wl["dims"]))
    return dict({"workload": wl["label"]}, **wl["config"],
                solver="KINSOL line search, EtaConstant 1e-5, GMRES(25), MGSemi V(1,1)",
                l2=f"inputs larger than L2 (every vector {cells * 8 / 1e6:.0f} MB, "
                   "working set several GB)",
                parallelism=f"replicas x{world}")


def reference_steps(workload: str, first: int, count: int, exe: str = "parflow_omp",
                    dump: bool = False):
    """Run the unmodified reference build (oracle/_ref) on the full workload
    for first + count timesteps from its initial condition and time steps
    first+1 .. first+count (per-step ends from the reference's KINSOL log).
    Returns (timesteps/s, the run's record)."""
    from oracle import refrun

    wl = _workloads()[workload]
    nx, ny, nz = wl["dims"]
    prob = wl["build"](nx, ny, nz, first + count)
    res = refrun.run(prob, first + count, exe=exe, dump=dump)
    return refrun.steps_per_second(res, first, count), res


def reference_arm(args, rank, world):
    """The reference's own CPU implementation on the same workload, at full
    size: the OpenMP build on every host thread runs warmup + steps
    timesteps and the last `steps` are timed; then the sequential build on
    one core times its second step.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return
    from oracle import refrun

    # the reference has no ensemble driver or adjoint: those use the headline workload
    wl_name = args.workload if args.workload in _workloads() else "hetero"
    wl = _workloads()[wl_name]
    nx, ny, nz = wl["dims"]
    k, w = max(1, args.steps), max(0, args.warmup)
    exe = "parflow_omp" if refrun.binary("parflow_omp") else "parflow"
    if refrun.binary(exe) is None:
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference build missing under oracle/_ref (built by "
                                         "oracle/ref.mk where the ParFlow sources are)"}),
              flush=True)
        return
    value, res = reference_steps(wl_name, w, k, exe=exe)
    counts = res["counts"]
    timed = counts[w:w + k]
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "timesteps/s",
           "n_gpus": args.gpus, "steps": k, "warmup": w,
           "ms_per_step": 1e3 / value, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": _config(wl, world),
           "cpu_baseline": {"value": value, "unit": "timesteps/s", "cores": res["threads"],
                            "kind": "reference",
                            "sample": f"the full workload ({nx}x{ny}x{nz}): {w + k} timesteps "
                                      f"from the initial condition with the unmodified "
                                      f"{exe} build, steps {w + 1}-{w + k} timed from the "
                                      f"reference's per-step KINSOL log",
                            "cpu": refrun.cpu_model()},
           "e2e": {"value": value, "unit": "timesteps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "wall_s": res["wall"], "kinsol_s": res["timing"].get("KINSol"),
           "newton_iters_per_step": float(timed[:, 0].mean()),
           "gmres_iters_per_step": float(timed[:, 1].mean()),
           "cell_newton_updates_per_s": nx * ny * nz * float(timed[:, 0].sum()) /
                                        (k / value)}
    if args.ref_seq_steps > 0 and refrun.binary("parflow"):
        sv, sres = reference_steps(wl_name, args.ref_seq_steps - 1, 1, exe="parflow")
        out["seq_1core"] = {"value": sv, "unit": "timesteps/s", "cores": 1,
                            "sample": f"step {args.ref_seq_steps} of the full workload from "
                                      f"its initial condition, sequential build, one core",
                            "wall_s": sres["wall"]}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# replicas: every rank solves its own copy; the job's time is the slowest rank
# ---------------------------------------------------------------------------
def max_over_ranks(ms: float, dist=None, device: str = "cuda") -> float:
    """Device-timed milliseconds of this rank -> the maximum over all ranks
    (one all-reduce of a scalar; NCCL on the GPU box, gloo in the tests)."""
    if dist is None:
        return ms
    import torch

    tt = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def job_throughput(steps: int, world: int, ms_max: float) -> float:
    """Whole-job timesteps/s: every rank's steps over the slowest rank's time."""
    return steps * world / (ms_max * 1e-3)


def compare_with_reference(prob, plan, ic, res, device: int) -> dict:
    """Max relative pressure difference (max |p - p_ref| / max |p_ref|) of
    every GPU form against the reference's pressures after each of the
    steps the reference run dumped, from the same initial condition, and
    whether the per-step Newton and GMRES counts equal the reference's."""
    from parflow_b200.solver import RichardsGPU

    ref_p = res["press"]
    out = {}
    for precision in ("fp64", "mixed", HEADLINE):
        g = RichardsGPU(prob, precision=precision, device=device)
        g.set_pressure(ic)
        errs, same = [], True
        for n in range(ref_p.shape[0]):
            t, dt = plan[n]
            g.set_time(t)
            st = g.advance(1, dt)[0]
            p = g.get_pressure()
            errs.append(float(np.abs(p - ref_p[n]).max() / np.abs(ref_p[n]).max()))
            same = same and (st.nonlin_iters == int(res["counts"][n, 0]) and
                             st.lin_iters == int(res["counts"][n, 1]))
        g.close()
        key = {"fp64": "fp64", "mixed": "mixed_fp32_mg", HEADLINE: "mixed"}[precision]
        out[key + "_max_rel_pressure_err"] = max(errs)
        out[key + "_per_step"] = errs
        out[key + "_counts_equal"] = bool(same)
    out["reference_counts"] = res["counts"][:, :2].tolist()
    return out


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def gpu_arm(args, rank, world, local_rank):
    import torch

    from parflow_b200 import configs
    from parflow_b200.solver import RichardsGPU, pad

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        dist = dist_mod
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    wl = _workloads()[args.workload]
    nx, ny, nz = args.size if args.profile else wl["dims"]
    prob = wl["build"](nx, ny, nz, args.warmup + args.steps + 2)
    cells = prob.ncells
    plan = prob.time_plan()
    ic = prob.initial_pressure()

    def timed_run(precision):
        s = RichardsGPU(prob, precision=precision, device=local_rank)
        s.set_pressure(ic)
        stream = torch.cuda.ExternalStream(s.stream())
        stats = []
        pressures = []
        for i in range(args.warmup):
            t, dt = plan[i]
            s.set_time(t)
            stats.extend(s.advance(1, dt))
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = s.kernel_launches()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        clocks = ClockSampler(local_rank)
        clocks.start()
        if args.profile:
            torch.cuda.profiler.start()
        e0.record(stream)
        for i in range(args.warmup, args.warmup + args.steps):
            t, dt = plan[i]
            s.set_time(t)
            stats.extend(s.advance(1, dt))
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        if args.profile:
            torch.cuda.profiler.stop()
        ck = clocks.stop()
        ms = e0.elapsed_time(e1)
        launches = s.kernel_launches() - launches0
        ms = max_over_ranks(ms, dist)
        p_final = s.get_pressure()
        return s, ms, stats[args.warmup:], launches, ck, p_final

    if args.profile:
        smx, msmx, stmx, launches, clocks, _ = timed_run(HEADLINE)
        smx.close()
        if rank == 0:
            print(json.dumps({"profile_run": True, "size": [nx, ny, nz], "steps": args.steps,
                              "ms_per_step": msmx / args.steps, "gpu_launches": int(launches),
                              "newton_iters": sum(x.nonlin_iters for x in stmx),
                              "gmres_iters": sum(x.lin_iters for x in stmx)}), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    # plain FP64 form first, then the all-FP32 multigrid, then the headline
    # mixed form, on the same steps
    s64, ms64, st64, _, _, p64 = timed_run("fp64")
    s64.close()
    s32, ms32, _, _, _, p32 = timed_run("mixed")
    s32.close()
    # the FP64 form with the mixed forms' kept preconditioned basis (x = Z y
    # instead of M^{-1} (V y)): separates that saving from the precision's
    os.environ["PFGPU_PC_BASIS"] = "2"
    s64z, ms64z, st64z, _, _, p64z = timed_run("fp64")
    s64z.close()
    del os.environ["PFGPU_PC_BASIS"]
    rel_err64z = float(np.abs(p64z - p64).max() / np.abs(p64).max())
    smx, msmx, stmx, launches, clocks, pmx = timed_run(HEADLINE)
    rel_err = float(np.abs(pmx - p64).max() / np.abs(p64).max())
    rel_err32 = float(np.abs(p32 - p64).max() / np.abs(p64).max())

    # roofline of the dominant kernel: k_rb_sweep, one red/black colour sweep
    # (27% of a timestep's GPU time in the launch list); timed on the finest
    # level, 13.1M cells, 12 algorithmic bytes per cell of the level (the
    # FP16 scaled operator 6 B; this colour's b 2 B, the other colour's x
    # read 2 B and this colour's x written 2 B: FP32 values of half the cells)
    kern = {}
    for name in ("colour_sweep", "rb_smooth", "matvec", "residual", "jacobian", "vcycle",
                 "mg_setup"):
        kms, kbytes = smx.time_kernel(name, reps=20)
        kern[name] = (kms, kbytes)
    dom = "colour_sweep"
    dms, dbytes = kern[dom]
    peak, peak_kind = peaks()
    achieved = dbytes / (dms * 1e-3) / 1e9
    traffic = None if RB_SWEEP_DRAM_BYTES_PER_CELL is None else \
        RB_SWEEP_DRAM_BYTES_PER_CELL * cells

    # end to end through the C ABI with host buffers: one pfgpu_newton_solve_sat
    # per step (p_old, s_old, p in; p and the saturation at it out), the call
    # a ParFlow nonlinear-solver module makes with its host vectors
    # (at the start of a step the old pressure / saturation equal the current
    # ones, so the caller passes each host buffer as both input and output)
    e2e_steps = max(3, min(args.steps, 10))
    shape_p = tuple(n + 2 for n in prob.shape)
    p_host = torch.from_numpy(pad(ic)).pin_memory()
    s_host = torch.from_numpy(pad(smx.saturation(ic))).pin_memory()
    import ctypes as C

    from parflow_b200 import lib as L

    lib = smx.lib
    st = L.Stats()

    def e2e_step(i):
        t, dt = plan[i]
        smx.set_time(t)
        pp, sp = C.c_void_p(p_host.data_ptr()), C.c_void_p(s_host.data_ptr())
        rc = lib.pfgpu_newton_solve_sat(smx.h, pp, sp, dt, pp, sp, C.byref(st))
        L.check(rc, "newton_solve_sat")

    e2e_step(0)  # warm
    stream = torch.cuda.ExternalStream(smx.stream())
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(1, 1 + e2e_steps):
        e2e_step(i)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    nbytes = int(np.prod(shape_p)) * 8
    h2d = 2 * nbytes   # p (= p_old), s_old
    d2h = 2 * nbytes   # p, s
    e2e_ms = max_over_ranks(e2e_ms, dist)

    # the reference build on the full workload: the CPU baseline (its second
    # timestep, timed from its KINSOL log) and the pressures after steps 1
    # and 2, against which every GPU form is checked from the same initial
    # condition (max relative difference, Newton and GMRES counts per step)
    cpu, vs_ref = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            v, res = reference_steps(args.workload, 1, 1, dump=True)
            cpu = {"value": v, "unit": "timesteps/s", "cores": res["threads"],
                   "kind": "reference",
                   "sample": f"the full workload ({nx}x{ny}x{nz}), unmodified {res['binary']} "
                             "build: 2 timesteps from the initial condition with pressure "
                             "output, step 2 timed from the reference's per-step KINSOL log",
                   "cpu": __import__("oracle.refrun", fromlist=["cpu_model"]).cpu_model()}
            vs_ref = compare_with_reference(prob, plan, ic, res, local_rank)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": "timesteps/s", "cores": 0, "kind": "reference",
                   "sample": f"failed: {e}"}

    if rank == 0:
        steps_mx = job_throughput(args.steps, world, msmx)
        steps_64 = job_throughput(args.steps, world, ms64)
        newton = sum(x.nonlin_iters for x in stmx)
        out = {
            "metric": METRIC, "value": steps_mx, "unit": "timesteps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": msmx / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 Newton/Arnoldi; f32 multigrid arithmetic on a diagonal-scaled f16 "
                     "operator; f32 Jacobian storage",
            "data": "synthetic",
            "precision": HEADLINE,
            "config": _config(wl, world),
            "fp64_steps_per_s": steps_64,
            "mixed_speedup_vs_fp64": steps_mx / steps_64,
            "mixed_vs_fp64_max_rel_pressure_err": rel_err,
            "mixed_fp32_mg_steps_per_s": job_throughput(args.steps, world, ms32),
            "mixed_fp32_mg_vs_fp64_max_rel_pressure_err": rel_err32,
            "fp64_kept_basis_steps_per_s": job_throughput(args.steps, world, ms64z),
            "fp64_kept_basis_vs_fp64_max_rel_pressure_err": rel_err64z,
            "solve": "one CUDA graph launch per Newton solve (device-side KINSOL/SPGMR "
                     "control); mixed forms keep the preconditioned Krylov basis (x = Z y)",
            "newton_iters_per_step": newton / max(1, len(stmx)),
            "gmres_iters_per_step": sum(x.lin_iters for x in stmx) / max(1, len(stmx)),
            "cell_newton_updates_per_s": cells * newton * world / (msmx * 1e-3),
            "roofline": {"bound": "hbm",
                         "kernel": "k_rb_sweep2: one red/black colour sweep, finest level "
                                   "(scaled f16 operator, colour-split f32 b and x)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "bytes_per_launch": dbytes, "ms_per_launch": dms},
            "kernels": {k: {"ms": v[0], "alg_bytes": v[1],
                            "gbs": (v[1] / (v[0] * 1e-3) / 1e9) if v[1] else None}
                        for k, v in kern.items()},
            "cpu_baseline": cpu,
            "vs_reference_steps_1_2": vs_ref,
            "e2e": {"value": world / (e2e_ms * 1e-3), "unit": "timesteps/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "pfgpu_newton_solve_sat with pinned host buffers"},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    smx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Ensemble workload (config 3): 48 members of uneven size, advanced together
# ---------------------------------------------------------------------------
def ensemble_arm(args, rank, world, local_rank):
    """Member-timesteps/s of the 48-member ensemble, every member resident on
    the GPU and all advanced concurrently (pfgpu_ensemble_advance) with the
    stencil launches' block shapes picked by the autotuner (pfgpu_autotune,
    untimed, once per member size), against the same members on the built-in
    block-shape heuristic and advanced one after another."""
    import torch

    from parflow_b200 import configs
    from parflow_b200.solver import RichardsGPU, ensemble_advance

    torch.cuda.set_device(local_rank)
    # the configuration's 10 timesteps per member (fewer with a smaller
    # --steps), timed from the initial state again after the warm-up steps
    # (graph capture, autotuning)
    warm = min(max(args.warmup, 1), 3)
    nsteps = max(1, min(args.steps, 10))
    probs = configs.ensemble(48, nsteps=10)
    cells = [p.ncells for p in probs]

    shapes = {}

    def fresh(tuned=True):
        ms = []
        for p in probs:
            g = RichardsGPU(p, precision=HEADLINE, device=local_rank)
            g.set_pressure(p.initial_pressure())
            g.set_time(p.start_time + p.dt)
            if tuned:
                shapes[p.shape] = g.autotune()
            ms.append(g)
        return ms

    def restart(ms):
        for g, p in zip(ms, probs):
            g.set_pressure(p.initial_pressure())
            g.set_time(p.start_time + p.dt)

    def timed(ms, nsteps, concurrent):
        streams = [torch.cuda.ExternalStream(g.stream()) for g in ms]
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in ms]
        ends = [torch.cuda.Event(enable_timing=True) for _ in ms]
        for e, st in zip(starts, streams):
            e.record(st)
        if concurrent:
            stats = ensemble_advance(ms, nsteps)
        else:
            stats = [g.advance(nsteps) for g in ms]
        for e, st in zip(ends, streams):
            e.record(st)
        torch.cuda.synchronize()
        t0 = starts[0]
        ms_total = max(t0.elapsed_time(e) for e in ends)
        return ms_total, stats

    conc = fresh()
    ensemble_advance(conc, warm)
    restart(conc)
    t_conc, st_conc = timed(conc, nsteps, True)
    for g in conc:
        g.close()
    heur = fresh(tuned=False)
    ensemble_advance(heur, warm)
    restart(heur)
    t_heur, _ = timed(heur, nsteps, True)
    for g in heur:
        g.close()
    seq = fresh()
    ensemble_advance(seq, warm)
    restart(seq)
    t_seq, st_seq = timed(seq, nsteps, False)
    for g in seq:
        g.close()
    newton = sum(s.nonlin_iters for m in st_conc for s in m)
    cell_updates = sum(c * sum(s.nonlin_iters for s in m) for c, m in zip(cells, st_conc))
    member_steps = len(probs) * nsteps
    if rank == 0:
        print(json.dumps({
            "metric": "ensemble member-timesteps/s (48 uneven members, mixed precision)",
            "precision": HEADLINE,
            "value": member_steps * world / (t_conc * 1e-3), "unit": "member-timesteps/s",
            "n_gpus": world, "steps": nsteps, "warmup": warm,
            "ms_per_step": t_conc / nsteps, "higher_is_better": True, "scaling": "weak",
            "dtype": "f64 Newton/Arnoldi; f32 multigrid arithmetic on a diagonal-scaled f16 "
                     "operator; f32 Jacobian storage",
            "data": "synthetic",
            "config": {"workload": "ensemble of 48 boxes, nx=ny in {64,96,128,192}, "
                                   "nz in {16,24,32,40}, 24.3M cells total",
                       "cells": sum(cells), "dt_h": 0.1},
            "mode": ("one CUDA graph launch per ensemble timestep (every member's Newton solve "
                     "with its own device-side control)"
                     if os.environ.get("PFGPU_ENSEMBLE_GRAPH", "1") != "0" else
                     "host thread per member"),
            "sequential_member_timesteps_per_s": member_steps / (t_seq * 1e-3),
            "concurrency_speedup": t_seq / t_conc,
            "heuristic_shapes_member_timesteps_per_s": member_steps / (t_heur * 1e-3),
            "autotune_speedup": t_heur / t_conc,
            "tile_shapes": {"x".join(map(str, k[::-1])): v for k, v in sorted(shapes.items())},
            "newton_iters_total": newton,
            "cell_newton_updates_per_s": cell_updates * world / (t_conc * 1e-3),
        }), flush=True)


# ---------------------------------------------------------------------------
# Adjoint workload (config 4): gradient of a misfit w.r.t. ln K, alpha, n
# ---------------------------------------------------------------------------
def adjoint_arm(args, rank, world, local_rank):
    """Forward run (20 FP64 steps, 128x128x32, trajectory recorded) plus the
    discrete-adjoint gradient of sum (p - p_obs)^2 over 256 observation cells
    at steps 5/10/15/20, timed on the device; then a central-difference check
    of the gradient with the same forward model (ResidualTol 1e-13)."""
    import torch

    from parflow_b200 import configs
    from parflow_b200.problem import SolverSettings
    from parflow_b200.solver import RichardsGPU

    torch.cuda.set_device(local_rank)
    nsteps, obs_steps = 20, [5, 10, 15, 20]
    solver = SolverSettings(residual_tol=1e-13, step_tol=1e-30)
    prob = configs.box(nx=128, ny=128, nz=32, nsteps=nsteps, dt=0.1, seed=4, solver=solver)
    shape = prob.shape
    lnk0 = np.log(prob.perm)
    prob.vg_alpha = np.full(shape, 2.0)
    prob.vg_n = np.full(shape, 3.0)
    rng = np.random.default_rng(40)
    cells = rng.choice(prob.ncells, size=256, replace=False)
    plan = prob.time_plan()[:nsteps]
    g = RichardsGPU(prob, precision="fp64", device=local_rank)
    stream = torch.cuda.ExternalStream(g.stream())

    def forward(lnk, alpha, vg_n, record=False):
        prob.perm = np.exp(lnk)
        prob.vg_alpha, prob.vg_n = alpha, vg_n
        g.update_fields()
        g.set_pressure(prob.initial_pressure())
        if record:
            g.adjoint_record(nsteps)
        ps = {}
        for n, (t, dt) in enumerate(plan, start=1):
            g.set_time(t)
            g.advance(1, dt)
            if n in obs_steps:
                ps[n] = g.get_pressure().ravel()[cells]
        return ps

    alpha0, n0 = prob.vg_alpha.copy(), prob.vg_n.copy()
    truth = forward(lnk0 + 0.3 * rng.standard_normal(shape), alpha0, n0)
    obs = np.stack([truth[n] + 0.01 * rng.standard_normal(len(cells)) for n in obs_steps])

    def misfit(ps):
        return sum(float(np.sum((ps[n] - obs[k]) ** 2)) for k, n in enumerate(obs_steps))

    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    forward(lnk0, alpha0, n0, record=True)
    e1.record(stream)
    m, g_lnk, g_a, g_n = g.adjoint_gradient(obs_steps, cells, obs, tol=1e-12)
    e2.record(stream)
    e2.synchronize()
    t_fwd, t_adj = e0.elapsed_time(e1), e1.elapsed_time(e2)
    grads = {"lnk": g_lnk, "alpha": g_a, "n": g_n}

    # central differences with the same forward model: the largest-gradient
    # cells and random cells of each field, and random directions
    # central differences at two steps: h, and h/5 whose truncation error is
    # 25x smaller (the misfit can have a kink where a cell's pressure crosses
    # zero during the run; there the two differences disagree with each other)
    h, h2 = 1e-5, 2e-6
    errs, checks = [], []

    def central(which, c, step):
        fields = {"lnk": lnk0.copy(), "alpha": alpha0.copy(), "n": n0.copy()}
        fields[which].ravel()[c] += step
        jp = misfit(forward(fields["lnk"], fields["alpha"], fields["n"]))
        fields[which].ravel()[c] -= 2 * step
        jm = misfit(forward(fields["lnk"], fields["alpha"], fields["n"]))
        return (jp - jm) / (2 * step)

    for which in ("lnk", "alpha", "n"):
        ga = np.abs(grads[which]).ravel()
        floor = 1e-6 * float(ga.max())  # relative error floor for near-zero entries
        order = np.argsort(-ga)
        # the four largest entries and four random ones among the top 10% of
        # the nonzero entries, excluding those four
        pool = order[4:max(12, int(np.count_nonzero(ga > floor)) // 10)]
        picks = list(order[:4]) + list(rng.choice(pool, min(4, len(pool)), replace=False))
        for c in picks:
            fd, fd2 = central(which, c, h), central(which, c, h2)
            ad = float(grads[which].ravel()[c])
            e1 = abs(ad - fd) / max(abs(fd), floor)
            e2 = abs(ad - fd2) / max(abs(fd2), floor)
            errs.append(min(e1, e2))
            checks.append({"field": which, "cell": int(c), "adjoint": ad, "fd_h": fd,
                           "fd_h5": fd2, "rel_to_max_grad": abs(ad) / float(ga.max()),
                           "rel_err_h": e1, "rel_err_h5": e2,
                           "fd_step_spread": abs(fd - fd2) / max(abs(fd2), floor)})
    for _ in range(2):
        d = {k: rng.standard_normal(shape) for k in grads}
        ad = sum(float(np.sum(grads[k] * d[k])) for k in grads)
        jp = misfit(forward(lnk0 + h * d["lnk"], alpha0 + h * d["alpha"], n0 + h * d["n"]))
        jm = misfit(forward(lnk0 - h * d["lnk"], alpha0 - h * d["alpha"], n0 - h * d["n"]))
        fd = (jp - jm) / (2 * h)
        errs.append(abs(ad - fd) / abs(fd))
        checks.append({"field": "random direction", "adjoint": ad, "fd": fd,
                       "rel_err": errs[-1]})
    g.close()
    if rank == 0:
        print(json.dumps({
            "metric": "adjoint gradient (ln K, alpha, n) of a 20-step misfit, 128x128x32",
            "value": 1e3 / (t_fwd + t_adj), "unit": "gradients/s", "n_gpus": world,
            "steps": nsteps, "warmup": 0, "ms_per_step": (t_fwd + t_adj) / nsteps,
            "higher_is_better": True, "scaling": "weak", "dtype": "f64", "data": "synthetic",
            "config": {"workload": "box 128x128x32 (524k cells), config-0 physics, 20 steps "
                                   "dt 0.1 h, 256 observation cells at steps 5/10/15/20",
                       "residual_tol": 1e-13, "adjoint_gmres_tol": 1e-12},
            "forward_ms": t_fwd, "adjoint_ms": t_adj, "adjoint_over_forward": t_adj / t_fwd,
            "misfit": m, "fd_checks": len(errs), "fd_max_rel_err": max(errs),
            "fd_median_rel_err": float(np.median(errs)), "fd_steps": [h, h2],
            "fd_error_rule": "per check the smaller of the errors against the two central "
                             "differences",
            "fd_check_list": checks,
        }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the reference CPU baseline and the check against its pressures")
    ap.add_argument("--ref-seq-steps", type=int, default=2,
                    help="reference arm: also time step N of the sequential one-core build "
                         "(0: skip)")
    ap.add_argument("--workload", default="hetero",
                    choices=["hetero", "overland", "overland_flow", "overland_diff", "ensemble",
                             "adjoint"],
                    help="hetero: the 512x512x50 bench line; overland / overland_flow / "
                         "overland_diff: the 256x256x20 overland hillslope with "
                         "OverlandKinematic / OverlandFlow / OverlandDiffusive routing; "
                         "ensemble: the 48-member set; adjoint: the gradient workload")
    ap.add_argument("--profile", action="store_true",
                    help="mixed solve only, timed steps bracketed by cudaProfilerStart/Stop")
    ap.add_argument("--size", default=f"{NX},{NY},{NZ}",
                    help="grid NX,NY,NZ (profiling runs only; the bench line is 512,512,50)")
    args = ap.parse_args()
    args.size = tuple(int(v) for v in args.size.split(","))
    if not args.profile and args.size != (NX, NY, NZ):
        ap.error("--size is for --profile runs; the bench workloads have fixed sizes")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.workload == "ensemble":
        ensemble_arm(args, rank, world, local_rank)
        return
    if args.workload == "adjoint":
        adjoint_arm(args, rank, world, local_rank)
        return
    gpu_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
