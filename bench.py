"""Benchmark of the single-GPU MHD integration hot path (one JSON line on stdout).

Workload: one RK3 step (3 x [periodic halo fill + substep + swap]) of the
8-field MHD system at 512^3 interior, FP64, seeded synthetic fields of the
benchmark workloads (lnrho, s ~ U(-1e-5, 1e-5), uu ~ N(0, 1e-3^2),
aa ~ N(0, 1e-4^2)), nu = eta = 5e-3, cs = 1, gamma = 5/3, dt = 1e-3.

  python bench.py [--gpus N --steps K --warmup W] [--n 512] [--impl reference]

* value       cell-updates/s of the whole job (N ranks x n^3 / max-over-ranks
              step time), device-resident inputs, CUDA events on the library's
              stream; the 17.8 GB state exceeds L2, so no flush is needed.
* e2e         the same metric through the C ABI with host buffers: every step
              copies the whole mesh from pinned host memory, runs
              acDeviceIntegrateStep and reads two diagnostics (max and rms of uu)
              back to the host.  The copy of a step's mesh is staged on a second
              stream while the previous step integrates (acDeviceLoadMeshStaged,
              acDeviceCommitStagedMesh); `serial` is the same with acDeviceLoadMesh
              in sequence.
* roofline    the solve kernel: algorithmic bytes (512 B per cell per RK3 step
              in FP64 = 5 reads + 3 writes of 8 fields) / its CUDA-event time,
              against the measured HBM copy bandwidth.
* cpu_baseline  the reference's own host model (oracle/_ref) on the host cores,
              a bounded sample (one RK3 step at 128^3), rank 0 at N=1.
* ensemble    64 independent FP32-compensated members of sizes {32,48,64,96}^3,
              graph-captured step in the autotuner's mode (persistent work list or
              per-member tiled launches as graph branches); against the members
              advanced one by one, a Device per member through acDeviceIntegrateStep.
* fp32comp    the same workload with FP32 fields and a compensated FP32 hi/lo RK3
              state (AC_precision = 1): cell-updates/s, speed-up over FP64, and
              the per-field relative L-inf against the FP64 path after 100 steps
              from the same initial mesh (rank 0 at N=1).
* cfl1024     the 1024^3 FP32-compensated run with adaptive CFL timesteps from the
              on-device maxima (20 steps, ~149 GB), with the FP64 run on the same
              dt sequence for its diagnostics (rank 0 at N=1).
* adjoint     the 64^3 discrete-adjoint gradient through 200 steps: backward /
              forward time (rank 0 at N=1).

--impl reference times that CPU implementation alone, one bounded sample per
step (rank 0; other ranks exit without work).  Multi-GPU runs are replicas:
each rank integrates its own mesh (weak scaling, no data-path collective).
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s per RK3 step at 512^3 (FP64)"
UNIT = "cell-updates/s"
# Minimum HBM bytes per cell per RK3 step: 8 fields x (5 reads + 3 writes) of
# the state; the FP32-compensated state is a (hi, lo) pair of 4-byte words.
BYTES_PER_CELL_STEP = {"fp64": 512, "fp32comp": 512}
# The CPU samples are one RK3 step at 128^3 (the reference's own host model
# takes ~1.6 s per step on 16 cores; 512^3 would take minutes per step).
REF_SAMPLE_N = 128


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32comp", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-cfl1024", action="store_true",
                    help="skip the 1024^3 adaptive-CFL leg (about 149 GB of device memory)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--workload", default="step512",
                    choices=["step512", "cfl1024", "adjoint64"],
                    help="step512: the FP64 RK3 step (default line); cfl1024: 1024^3 "
                         "FP32-compensated run with adaptive CFL timesteps; adjoint64: "
                         "gradient of the final energy through 200 steps at 64^3")
    ap.add_argument("--accuracy-steps", type=int, default=100)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- helpers

def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name: str):
    """dram bytes per launch recorded in profiles/<name> (a `traffic_bytes_per_launch:` line)."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def profile_limiter(name: str):
    """The `limiter:` line of profiles/<name>: what ncu showed bounding the kernel."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("limiter:"):
            return line.split(":", 1)[1].strip()
    return None


def cpu_reference_sample(n: int, steps: int = 1):
    """Times the reference's host model (oracle/_ref, else the port) on an n^3
    sample.  Inputs and parameters come from the oracle side, so this leg maps
    no library of the product."""
    from oracle import oracle  # checker only: the CPU baseline leg
    kind = "reference" if oracle.available("reference") else "port"
    f = oracle.seeded_mesh(n, 2)
    p = oracle.box_params(n)
    t0 = time.perf_counter()
    oracle.integrate(f, p, 1e-3, steps, kind)
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": n ** 3 * steps / dt, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{steps} RK3 step(s) of the reference host model "
                      f"(src/utils/modelsolver.cc acHostIntegrateStep, long double, OpenMP) "
                      f"on a {n}^3 periodic box, same physics and seeded distributions; "
                      f"rate per cell",
            "seconds": dt}


# ---------------------------------------------------------------- reference arm

def workload_config(n: int, world: int) -> dict:
    """The `config` of both arms' lines."""
    return {"workload": f"MHD RK3 step, {n}^3 interior + 3-cell halos, 8 fields, FP64, "
                        f"periodic, dt=1e-3",
            "n": n, "parallelism": f"replicas x{world}",
            "l2": f"state {2 * 8 * (n + 6) ** 3 * 8 / 1e9:.1f} GB > 126 MB L2; no flush needed"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    for _ in range(args.warmup):
        cpu_reference_sample(REF_SAMPLE_N)
    vals, secs = [], []
    for _ in range(args.steps):
        s = cpu_reference_sample(REF_SAMPLE_N)
        vals.append(s["value"])
        secs.append(s["seconds"])
    v = statistics.median(vals)
    ms = statistics.median(secs) * 1e3  # measured at the sample size, not scaled
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f80",
        "data": "synthetic",
        "config": dict(workload_config(args.n, world), cpu_sample_n=REF_SAMPLE_N,
                       cpu_sample=f"each step: one RK3 step of a {REF_SAMPLE_N}^3 box; "
                                  f"ms_per_step is that step's time"),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": s["cores"], "kind": s["kind"],
                         "sample": s["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm

def run_gpu(args):
    import numpy as np
    import torch

    import astaroth_b200 as ab
    from astaroth_b200 import capi
    from astaroth_b200 import dist as adist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    adist.init("nccl")

    n = args.n
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    dt = 1e-3
    host = ab.seeded_mesh(info, 2 + rank)
    dev = ab.Device(info, device_id=local)
    dev.load_mesh(host)
    dev.synchronize()
    stream = torch.cuda.ExternalStream(dev.stream_handle(0), device=torch.device("cuda", local))

    barrier = adist.barrier

    for _ in range(args.warmup):
        dev.integrate_step(dt)
    dev.synchronize()

    # ---- timed region: K graph-launched RK3 steps
    launches0 = dev.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            dev.integrate_step(dt)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    launches = dev.launch_count() - launches0
    t_ms = ev0.elapsed_time(ev1) / args.steps
    t_max = adist.max_over_ranks(t_ms)
    clocks = clk.summary()

    # ---- per-kernel times of the solve kernel (same stream, plain launches)
    solve_ms, bc_ms = [], []
    for _ in range(2):
        for s in range(3):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(stream)
            dev.periodic_boundconds()
            e[1].record(stream)
            dev.integrate_substep(s, dt)
            e[2].record(stream)
            dev.swap_buffers()
            e[2].synchronize()
            bc_ms.append(e[0].elapsed_time(e[1]))
            solve_ms.append(e[1].elapsed_time(e[2]))
    solve_step_ms = sum(solve_ms[-3:])
    cells = n ** 3
    alg_bytes_step = BYTES_PER_CELL_STEP["fp64"] * cells
    peak, peak_kind = peaks()
    achieved = alg_bytes_step / (solve_step_ms * 1e-3) / 1e9
    traffic = profile_traffic("solve_lead_fp64_256.md")

    # ---- e2e through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty(host.shape, dtype=torch.float64, pin_memory=True)
        pinned.numpy()[...] = host
        hmesh = ab.device.mesh_struct(pinned.numpy(), info)
        lib = capi.load()
        out = capi.C.c_double()
        rt_max, rt_rms = capi.RTYPES["RTYPE_MAX"], capi.RTYPES["RTYPE_RMS"]

        def e2e_step():
            lib.acDeviceLoadMesh(dev.handle, 0, hmesh)
            lib.acDeviceIntegrateStep(dev.handle, 0, dt)
            lib.acDeviceReduceVec(dev.handle, 0, rt_max, 1, 2, 3, capi.C.byref(out))
            a = out.value
            lib.acDeviceReduceVec(dev.handle, 0, rt_rms, 1, 2, 3, capi.C.byref(out))
            return a, out.value

        def e2e_step_pipelined():
            # this step's input was staged during the previous step; stage the
            # next one on stream 1 while stream 0 integrates this one
            lib.acDeviceCommitStagedMesh(dev.handle, 0)
            lib.acDeviceLoadMeshStaged(dev.handle, 1, hmesh)
            lib.acDeviceIntegrateStep(dev.handle, 0, dt)
            lib.acDeviceReduceVec(dev.handle, 0, rt_max, 1, 2, 3, capi.C.byref(out))
            a = out.value
            lib.acDeviceReduceVec(dev.handle, 0, rt_rms, 1, 2, 3, capi.C.byref(out))
            return a, out.value

        ke = max(2, min(args.steps, 5))
        e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            e2e_step()
        ts = adist.max_over_ranks((time.perf_counter() - t0) / ke)
        lib.acDeviceLoadMeshStaged(dev.handle, 1, hmesh)  # the first step's input
        e2e_step_pipelined()
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            e2e_step_pipelined()
        te = adist.max_over_ranks((time.perf_counter() - t0) / ke)
        dev.synchronize()
        e2e = {"value": world * cells / te, "unit": UNIT,
               "h2d_bytes_per_step": int(host.nbytes), "d2h_bytes_per_step": 16,
               "ms_per_step": te * 1e3,
               "how": "every step: the whole 512^3 mesh from pinned host memory "
                      "(acDeviceLoadMeshStaged on stream 1, overlapping the previous step; "
                      "acDeviceCommitStagedMesh), acDeviceIntegrateStep, two reductions "
                      "read back; wall clock",
               "serial": {"value": world * cells / ts, "ms_per_step": ts * 1e3,
                          "how": "acDeviceLoadMesh, acDeviceIntegrateStep, two reductions, "
                                 "in sequence"}}

    fp32 = None
    if world == 1 and not args.no_fp32comp:
        fp32 = fp32comp_leg(args, ab, torch, host, dev, info)

    ens = None
    if not args.no_ensemble:
        ens = ensemble_leg(args, torch, rank, world)

    dev.destroy()
    host = pinned = hmesh = None  # the host copies of the 512^3 mesh (17.8 GB) go first
    cfl = adj = None
    if rank == 0 and world == 1 and not args.no_cfl1024:
        try:
            cfl = cfl1024_leg()
        except Exception as exc:  # reported, never fatal to the main line
            cfl = {"error": str(exc)[:300]}
    if rank == 0 and world == 1 and not args.no_adjoint:
        try:
            adj = adjoint_leg(max(3, min(args.steps, 10)), max(1, min(args.warmup, 3)))
        except Exception as exc:
            adj = {"error": str(exc)[:300]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_sample(REF_SAMPLE_N)
            cpu.pop("seconds", None)
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"error": str(exc)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": world * cells / (t_max * 1e-3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded: lnrho,s ~ U(-1e-5,1e-5); uu ~ N(0,1e-3^2); "
                    "aa ~ N(0,1e-4^2))",
            "config": workload_config(n, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "solve (3 launches per RK3 step)",
                         "alg_bytes_per_launch": alg_bytes_step / 3,
                         "traffic_source": "profiles/solve_lead_fp64_256.md (ncu dram bytes at "
                                           "256^3 scaled by the cell count to 512^3)",
                         "bytes_per_cell_step": BYTES_PER_CELL_STEP["fp64"],
                         "peak_source": peak_kind, "solve_ms_per_step": solve_step_ms,
                         "boundconds_ms_per_step": sum(bc_ms[-3:]),
                         "limiter": profile_limiter("solve_lead_fp64_256.md")},
            "e2e": e2e, "gpu_launches": launches, "clocks": clocks, "cpu_baseline": cpu,
            "fp32comp": fp32, "ensemble": ens, "cfl1024": cfl, "adjoint": adj,
        }
        if fp32 and "ms_per_step" in fp32:
            fp32["speedup_vs_fp64"] = t_max / fp32["ms_per_step"]
        print(json.dumps(line), flush=True)
    adist.barrier()
    adist.destroy()


def timed_steps(dev, torch, stream, steps, dt):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        dev.integrate_step(dt)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def fp32comp_leg(args, ab, torch, host, dev64, info64):
    """FP32-compensated run of the same workload, and its error against FP64."""
    import numpy as np
    n, dt = args.n, 1e-3
    info = ab.make_info(n, precision=1, **ab.CONFIG_PARAMS)
    dev = ab.Device(info, device_id=torch.cuda.current_device())
    stream = torch.cuda.ExternalStream(dev.stream_handle(0))
    dev.load_mesh(host)
    for _ in range(args.warmup):
        dev.integrate_step(dt)
    dev.synchronize()
    l0 = dev.launch_count()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms = timed_steps(dev, torch, stream, args.steps, dt)
    launches = dev.launch_count() - l0
    solve = []
    for s in range(3):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        dev.periodic_boundconds()
        e[0].record(stream)
        dev.integrate_substep(s, dt)
        e[1].record(stream)
        dev.swap_buffers()
        e[1].synchronize()
        solve.append(e[0].elapsed_time(e[1]))
    peak, _ = peaks()
    achieved = BYTES_PER_CELL_STEP["fp32comp"] * n ** 3 / (sum(solve) * 1e-3) / 1e9
    out = {"value": n ** 3 / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
           "gpu_launches": launches, "clocks": clk.summary(),
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak,
                        "bytes_per_cell_step": BYTES_PER_CELL_STEP["fp32comp"],
                        "solve_ms_per_step": sum(solve)}}
    if args.accuracy_steps > 0:
        # both paths from the same initial mesh, compared field by field
        dev.load_mesh(host)
        dev64.load_mesh(host)
        for _ in range(args.accuracy_steps):
            dev.integrate_step(dt)
            dev64.integrate_step(dt)
        lib = ab.capi.load()
        C = ab.capi.C
        shape = ab.empty_mesh(info64).shape[1:]
        fa = np.zeros(shape)
        fb = np.zeros(shape)
        errs, errs2 = [], []
        for q in range(8):
            # one field at a time: an AcMesh whose only buffer is field q
            sa, sb = ab.capi.AcMesh(), ab.capi.AcMesh()
            sa.info, sb.info = info64, info
            sa.vertex_buffer[q] = fa.ctypes.data_as(C.POINTER(C.c_double))
            sb.vertex_buffer[q] = fb.ctypes.data_as(C.POINTER(C.c_double))
            lib.acDeviceStoreVertexBuffer(dev64.handle, 0, q, C.byref(sa))
            lib.acDeviceStoreVertexBuffer(dev.handle, 0, q, C.byref(sb))
            ia = fa[3:-3, 3:-3, 3:-3]
            ib = fb[3:-3, 3:-3, 3:-3]
            den = float(np.abs(ia).max()) or 1.0
            errs.append(float(np.abs(ib - ia).max()) / den)
            den2 = float(np.sqrt(np.sum(ia * ia))) or 1.0
            errs2.append(float(np.sqrt(np.sum((ib - ia) ** 2))) / den2)
        out["rel_linf_vs_fp64"] = {"steps": args.accuracy_steps, "per_field": errs,
                                   "max": max(errs)}
        out["rel_l2_vs_fp64"] = {"steps": args.accuracy_steps, "per_field": errs2,
                                 "max": max(errs2)}
    dev.destroy()
    return out


def ensemble_leg(args, torch, rank, world):
    """The 64-member FP32-compensated ensemble (N in {32, 48, 64, 96}, nu and
    eta log-uniform on [1e-3, 1e-2], seeds 100..163, dt = 1e-3): members are
    sharded across ranks (no data-path collective); each rank advances its
    members with the graph-captured persistent step and, for comparison, with
    sequential per-member plain launches."""
    from astaroth_b200 import dist as adist
    from astaroth_b200.ensemble import Ensemble, ensemble_members

    members = ensemble_members(64)
    costs = [abs(ab_cells(i)) for i, _ in members]
    mine = adist.shard(costs, rank, world)
    total_cells = sum(costs)
    e = Ensemble([members[m][0] for m in mine], device_id=torch.cuda.current_device())
    e.load_seeded([members[m][1] for m in mine])
    e.set_timesteps(1e-3)
    tiles, tune_ms = e.autotune(use_cache=False)
    stream = torch.cuda.ExternalStream(e.stream_handle())

    def timed(step, k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        adist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(k):
            step()
        e1.record(stream)
        e1.synchronize()
        return adist.max_over_ranks(e0.elapsed_time(e1) / k)

    # a step is a few ms: time at least 20, with the clock sampler (a
    # subprocess whose start-up would stall launches) running before warm-up
    k = max(args.steps, 20)
    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(args.warmup):
            e.integrate_step()
        e.synchronize()
        l0 = e.launch_count()
        ms = timed(e.integrate_step, k)
        launches = (e.launch_count() - l0) // k
    for _ in range(args.warmup):
        e.integrate_step_sequential()
    l1 = e.launch_count()
    ms_plain = timed(e.integrate_step_sequential, k)
    launches_plain = (e.launch_count() - l1) // k
    # the one-by-one arm: one single-mesh Device per member, each stepped with
    # acDeviceIntegrateStep (its default tiled kernel, its own streams)
    ms_seq, launches_seq = device_loop_ms(torch, [members[m] for m in mine], k, args.warmup)
    ms_seq = adist.max_over_ranks(ms_seq)
    # both step modes with the tuned work-list tiles, for the record
    modes = {}
    for mode in (0, 1):
        try:
            e.set_tiles(*tiles[:4], mode=mode)
        except Exception:
            continue
        for _ in range(args.warmup):
            e.integrate_step()
        e.synchronize()
        modes[mode] = timed(e.integrate_step, k)
    e.set_tiles(*tiles)
    e.destroy()
    peak, _ = peaks()
    achieved = BYTES_PER_CELL_STEP["fp32comp"] * total_cells / world / (ms * 1e-3) / 1e9
    return {"workload": "64 members, N in {32,48,64,96}, nu/eta log-U[1e-3,1e-2], "
                        "seeds 100..163, FP32 compensated, dt=1e-3",
            "members": len(members), "cells": total_cells, "value": total_cells / (ms * 1e-3),
            "unit": UNIT, "ms_per_step": ms, "steps": k, "gpu_launches_per_step": launches,
            "sequential": {"value": total_cells / (ms_seq * 1e-3), "ms_per_step": ms_seq,
                           "gpu_launches_per_step": launches_seq,
                           "how": "one single-mesh Device per member, acDeviceIntegrateStep "
                                  "on each in turn (default tiled kernel, the Devices' own "
                                  "streams); CUDA events joined over all member streams"},
            "speedup_vs_sequential": ms_seq / ms,
            "plain_sequential": {"ms_per_step": ms_plain, "gpu_launches_per_step": launches_plain,
                                 "how": "acEnsembleIntegrateStepSequential: per-member plain "
                                        "(untiled) launches in one stream"},
            "tiles": list(tiles),
            "ms_per_step_by_mode": {"persistent": modes.get(0),
                                    "tiled_per_member_graph": modes.get(1)},
            "autotune_solve_ms": tune_ms, "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "bytes_per_cell_step": BYTES_PER_CELL_STEP["fp32comp"],
                         "note": "whole step incl. halo fills"},
            "scaling": "strong (64 members split across ranks)"}


def device_loop_ms(torch, members, k, warmup):
    """ms per RK3 step of the members advanced one by one: a Device per member,
    acDeviceIntegrateStep on each in turn.  The Devices run on their own
    streams; the timing joins them with CUDA events on one stream."""
    import astaroth_b200 as ab
    devs = []
    try:
        for info, seed in members:
            d = ab.Device(info, device_id=torch.cuda.current_device())
            d.load_mesh(ab.seeded_mesh(info, seed))
            devs.append(d)
        streams = [torch.cuda.ExternalStream(d.stream_handle(0)) for d in devs]
        for _ in range(warmup):
            for d in devs:
                d.integrate_step(1e-3)
        torch.cuda.synchronize()
        main = torch.cuda.current_stream()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = sum(d.launch_count() for d in devs)
        e0.record(main)
        for st in streams:
            st.wait_event(e0)
        for _ in range(k):
            for d in devs:
                d.integrate_step(1e-3)
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        e1.record(main)
        e1.synchronize()
        launches = (sum(d.launch_count() for d in devs) - l0) // k
        return e0.elapsed_time(e1) / k, launches
    finally:
        for d in devs:
            d.destroy()


def ab_cells(info):
    from astaroth_b200.device import dims
    nx, ny, nz = dims(info)
    return nx * ny * nz


def load_fields_by_parts(ab, dev, info, seed):
    """Loads the seeded initial condition with a solenoidal velocity one part at
    a time (uu as three fields together, then each other field), so the host
    holds at most three fields."""
    import numpy as np
    from astaroth_b200 import capi
    C = capi.C
    lib = capi.load()
    nx, ny, nz = ab.device.dims(info)
    shape = (nz + 6, ny + 6, nx + 6)

    def mesh_of(bufs):
        m = capi.AcMesh()
        m.info = info
        for q, b in bufs.items():
            m.vertex_buffer[q] = b.ctypes.data_as(C.POINTER(C.c_double))
        return m

    bufs = {q: np.empty(shape) for q in (1, 2, 3)}
    m = mesh_of(bufs)
    if lib.acHostMeshSolenoidalModes(C.byref(m), seed, 64, 8, 1e-2) != 0:
        raise RuntimeError("acHostMeshSolenoidalModes failed")
    for q in bufs:
        if lib.acDeviceLoadVertexBuffer(dev.handle, 0, m, q) != 0:
            raise RuntimeError("acDeviceLoadVertexBuffer failed")
    del bufs, m
    for q in (0, 4, 5, 6, 7):
        bufs = {q: np.empty(shape)}
        m = mesh_of(bufs)
        if lib.acHostMeshRandomizeSeeded(C.byref(m), seed, 1e-5, 1e-3, 1e-4) != 0:
            raise RuntimeError("acHostMeshRandomizeSeeded failed")
        if lib.acDeviceLoadVertexBuffer(dev.handle, 0, m, q) != 0:
            raise RuntimeError("acDeviceLoadVertexBuffer failed")
        del bufs, m
    dev.synchronize()


def diagnostics(dev):
    out = {}
    for q, name in enumerate(("lnrho", "uux", "uuy", "uuz", "ax", "ay", "az", "entropy")):
        out[name] = [dev.reduce_scal("RTYPE_MAX", q), dev.reduce_scal("RTYPE_MIN", q),
                     dev.reduce_scal("RTYPE_RMS", q)]
    out["uu_rms"] = [dev.reduce_vec("RTYPE_RMS", 1, 2, 3)]
    out["aa_rms"] = [dev.reduce_vec("RTYPE_RMS", 4, 5, 6)]
    return out


# Diffusive Courant factor of the 1024^3 run.  The timestep bound of the
# reference (samples/standalone_mpi/main.cc:430-440, mhdsolver.ac:551-583) is
# cdtv * dsmin^2 / max(nu, eta, gamma chi), with no dimension or stencil factor
# and without the bulk viscosity zeta.  The fastest decaying mode of the
# 6th-order Laplacian in 3-D has eigenvalue -18.13 / dx^2, and the longitudinal
# velocity diffuses with (4/3) nu + zeta = 0.0167, so RK3 (stable for
# dt * |lambda| <= 2.51 on the negative real axis) needs cdtv <= 0.0415 at
# nu = 5e-3.  cdtv = 0.3 (config/astaroth.conf:46) gives dt * |lambda| = 18 at
# 1024^3, where the diffusive bound is the smaller one, and the run overflows
# in a few steps (in the reference's formula as in this one).
CFL1024_CDTV = 0.04


def cfl1024_leg(n: int = 1024, steps: int = 20) -> dict:
    """The 1024^3 FP32-compensated run with adaptive CFL timesteps: u a solenoidal
    sum of 64 Fourier modes (|k| <= 8, amplitude 1e-2), aa ~ N(0, 1e-4^2), lnrho
    and s ~ U(-1e-5, 1e-5), seed 3; 20 RK3 steps whose dt comes from the
    on-device CFL maxima (Courant factors cdt = 0.4 and cdtv = CFL1024_CDTV).
    The same run in FP64 with the same dt sequence checks the diagnostics (max,
    min, rms of every field).  About 149 GB on the device, one run at a time."""
    import torch
    import astaroth_b200 as ab

    dev_id = torch.cuda.current_device()
    res = {}
    dts = []
    for prec in (1, 0):
        info = ab.make_info(n, precision=prec, cdtv=CFL1024_CDTV, **ab.CONFIG_PARAMS)
        dev = ab.Device(info, device_id=dev_id)
        t0 = time.perf_counter()
        load_fields_by_parts(ab, dev, info, 3)
        t_load = time.perf_counter() - t0
        stream = torch.cuda.ExternalStream(dev.stream_handle(0))
        free_b, total_b = torch.cuda.mem_get_info()
        if prec == 1:
            dev.calc_timestep()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        l0 = dev.launch_count()
        with ClockSampler(dev_id) as clk:
            ev0.record(stream)
            for s in range(steps):
                if prec == 1:
                    dt = dev.timestep()  # from the maxima of the last substep 2
                    dts.append(dt)
                else:
                    dt = dts[s]
                dev.integrate_step(dt)
            ev1.record(stream)
            ev1.synchronize()
        ms = ev0.elapsed_time(ev1) / steps
        res[prec] = {"ms_per_step": ms, "value": n ** 3 / (ms * 1e-3),
                     "gpu_launches": dev.launch_count() - l0, "clocks": clk.summary(),
                     "device_bytes_used": total_b - free_b, "load_s": t_load,
                     "diagnostics": diagnostics(dev)}
        dev.destroy()
        del dev
        torch.cuda.synchronize()
    d32, d64 = res[1]["diagnostics"], res[0]["diagnostics"]
    rel = {k: max(abs(a - b) / max(abs(b), 1e-300) for a, b in zip(d32[k], d64[k]))
           for k in d32}
    peak, _ = peaks()
    achieved = BYTES_PER_CELL_STEP["fp32comp"] * n ** 3 / (res[1]["ms_per_step"] * 1e-3) / 1e9
    return {"metric": f"cell-updates/s per RK3 step at {n}^3 (FP32-compensated, adaptive CFL)",
            "value": res[1]["value"], "unit": UNIT, "steps": steps,
            "ms_per_step": res[1]["ms_per_step"], "dtype": "f32 (compensated hi/lo)",
            "data": "synthetic (seed 3: solenoidal uu of 64 modes, |k|<=8, amplitude 1e-2; "
                    "aa ~ N(0,1e-4^2); lnrho, s ~ U(-1e-5,1e-5))",
            "workload": f"{n}^3 FP32-compensated, {steps} RK3 steps, dt from the on-device CFL "
                        f"maxima each step (cdt=0.4, cdtv={CFL1024_CDTV})",
            "dt": dts, "gpu_launches": res[1]["gpu_launches"], "clocks": res[1]["clocks"],
            "device_bytes_used": res[1]["device_bytes_used"], "load_s": res[1]["load_s"],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "note": "whole step incl. halo fills and "
                                                          "the per-step host read of dt"},
            "fp64_same_dts": {"ms_per_step": res[0]["ms_per_step"], "value": res[0]["value"],
                              "device_bytes_used": res[0]["device_bytes_used"],
                              "clocks": res[0]["clocks"]},
            "diagnostics_fp32comp": d32, "diagnostics_fp64": d64,
            "diagnostics_rel_diff_vs_fp64": rel,
            "diagnostics_max_rel_diff": max(rel.values())}


def run_cfl1024(args):
    """--workload cfl1024: the 1024^3 leg alone, as its own line."""
    import torch
    torch.cuda.set_device(0)
    d = cfl1024_leg(args.n if args.n != 512 else 1024)
    line = {k: d[k] for k in ("metric", "value", "unit", "steps", "ms_per_step", "dtype",
                              "data")}
    line.update({"n_gpus": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak",
                 "vs_baseline": None, "config": {"workload": d["workload"]}})
    line.update({k: v for k, v in d.items() if k not in line})
    print(json.dumps(line), flush=True)


def adjoint_leg(steps_timed: int, warmup: int) -> dict:
    """Gradient of J = E_kin + E_mag after 200 FP64 RK3 steps at 64^3 (dt = 1e-3,
    seed 4, checkpoints every 20 steps) with respect to the initial fields and
    nu, eta, through the torch.autograd wrapper over the C ABI: forward time,
    backward time (recompute + reverse sweep) and their ratio, CUDA events on
    torch's current stream with a device synchronisation on both sides."""
    import torch
    import astaroth_b200 as ab
    from astaroth_b200 import autograd as AG

    n, steps, every, dt = 64, 200, 20, 1e-3
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = torch.from_numpy(ab.seeded_mesh(info, 4)).cuda()
    dev = ab.Device(info, device_id=torch.cuda.current_device())
    fwd, bwd = [], []
    l0 = dev.launch_count()
    peak_bytes = 0
    for it in range(warmup + steps_timed):
        x0 = f.clone().requires_grad_(True)
        nu = torch.tensor(5e-3, dtype=torch.float64, device="cuda", requires_grad=True)
        eta = torch.tensor(5e-3, dtype=torch.float64, device="cuda", requires_grad=True)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        fN = AG.integrate(x0, nu, eta, dev, steps, dt, checkpoint_every=every)
        J = AG.energy(fN, info)
        e[1].record()
        J.backward()
        e[2].record()
        torch.cuda.synchronize()
        peak_bytes = max(peak_bytes, torch.cuda.max_memory_allocated())
        if it >= warmup:
            fwd.append(e[0].elapsed_time(e[1]))
            bwd.append(e[1].elapsed_time(e[2]))
    launches = dev.launch_count() - l0
    dev.destroy()
    tf, tb = statistics.median(fwd), statistics.median(bwd)
    return {"metric": "adjoint cost: backward (recompute + reverse sweep) / forward time",
            "value": tb / tf, "unit": "x", "higher_is_better": False, "dtype": "f64",
            "workload": f"{n}^3, {steps} RK3 steps, dt={dt}, checkpoints every {every} steps, "
                        f"J = E_kin + E_mag at the final time; gradients w.r.t. the 8 initial "
                        f"fields and nu, eta",
            "samples": steps_timed, "forward_ms": tf, "backward_ms": tb,
            "forward_ms_per_step": tf / steps, "backward_ms_per_step": tb / steps,
            "peak_torch_bytes": peak_bytes, "gpu_launches": launches}


def run_adjoint64(args):
    """--workload adjoint64: the adjoint leg alone, as its own line."""
    import torch
    torch.cuda.set_device(0)
    d = adjoint_leg(args.steps, args.warmup)
    line = {"metric": d["metric"], "value": d["value"], "unit": "x", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seed 4, benchmark distributions)",
            "config": {"workload": d["workload"], "n": 64}}
    line.update({k: v for k, v in d.items() if k not in line})
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "cfl1024":
        run_cfl1024(args)
        return
    if args.workload == "adjoint64":
        run_adjoint64(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
