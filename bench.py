"""Benchmark of the RKDG shallow-water step (element-DOF updates per second per RK stage).

Default workload: the manufactured-solution p=2 case at scale -- 512x512 quads -> 524,288 jittered
triangles, Dunavant degree 4 / 3-point Gauss-Legendre, LLF, SSP-RK3 -- on the FP32-bulk path, with
the FP64 plain path timed on the same workload and the L2 errors of both against the analytic
solution reported after the run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision fp32|fp64]

One process per GPU (torchrun for N > 1); each rank advances its own replica of the workload
(the step does not shard: replicas only). Rank 0 prints one JSON line.
--impl reference times the CPU implementation of the same step (the oracle port: the reference
itself cannot be built here) on the host cores, rank 0 only.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "element-DOF updates/s per RK stage, FP32+MLP vs FP64 plain on B200 at equal L2"
UNIT = "element-DOF/s"
# compulsory HBM bytes per element-DOF and RK stage for p=2 SSP-RK3 (state in, q0 on 2 of 3 stages,
# state out, per-element geometry and per-edge data, each array touched once): FP32 45 B, FP64 87 B
# compulsory HBM bytes per element-DOF per RK stage (each array touched once): stage states read
# (1 + the fraction of stages that also read q_0) and written, FP64 in both precisions; element
# geometry and bathymetry (FP32 in the FP32 path) and the edge records. p = 2 SSP-RK3, p = 1 SSP-RK2.
ALG_BYTES_PER_UNIT = {("fp32", 2): 77.0, ("fp64", 2): 87.0, ("fp32", 1): 82.0, ("fp64", 1): 99.0}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--nq", type=int, default=512, help="quads per side of the workload mesh")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU baseline sample")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self._t.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n, backend=None):
    """One process per GPU from the torchrun environment; NCCL on GPUs (gloo when no GPU is visible, which
    is how the rank logic is tested on a CPU host)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def dist_max(x, world):
    """Max over ranks (every rank takes this collective in the same order)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch

    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def job_value(units_per_step, steps, world, max_ms):
    """Whole-job throughput of N replicas: all ranks' units over the slowest rank's time."""
    return units_per_step * steps * world / (max_ms / 1e3)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(precision):
    """DRAM bytes per stage-kernel launch from the committed ncu summary of this workload, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")) as f:
            d = json.load(f)
        return d.get(precision)
    except Exception:
        return None


def cpu_baseline(nq, seconds, precision_note):
    """The oracle (FP64 CPU restatement) on the host cores, on a bounded sample of the workload."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    from dgswemv2_b200 import configs
    from tests.oracle_ctypes import Oracle

    cores = os.cpu_count() or 1
    O = Oracle(os.path.join(ROOT, "oracle", "build", "liboracle.so"))
    # size the sample so one RK step takes well under the budget: start from a quarter-size mesh
    sub = max(32, nq // 4)
    mesh, cfg = configs.config2(nq=sub)
    P = O.problem(cfg, mesh, n_threads=cores)
    P.step(1)  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        P.step(1)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 1000:
            break
    units = mesh.n_elems * 6 * 3 * n
    return {"value": units / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "oracle (FP64 C++ restatement of the reference step) on the same discretisation at %dx%d quads "
                      "(%d triangles), %d SSP-RK3 steps in %.1f s, %d OpenMP threads" % (sub, sub, mesh.n_elems, n, el,
                                                                                        cores)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    from dgswemv2_b200 import configs
    from tests.oracle_ctypes import Oracle

    cores = os.cpu_count() or 1
    O = Oracle(os.path.join(ROOT, "oracle", "build", "liboracle.so"))
    # each step is one SSP-RK3 step on a bounded sample of the workload: the mesh is scaled so that
    # warm-up + timed steps take about two minutes on this host
    budget = 120.0
    nq = args.nq
    while True:
        mesh, cfg = configs.config2(nq=nq)
        P = O.problem(cfg, mesh, n_threads=cores)
        t0 = time.perf_counter()
        P.step(1)
        t1 = time.perf_counter() - t0
        if t1 * (args.steps + args.warmup) <= budget or nq <= 16:
            break
        nq = max(16, int(nq / math.sqrt(t1 * (args.steps + args.warmup) / budget * 1.2)))
    P.step(max(0, args.warmup - 1))
    t0 = time.perf_counter()
    P.step(args.steps)
    el = time.perf_counter() - t0
    units = mesh.n_elems * 6 * 3 * args.steps
    v = units / el
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "manufactured solution p=2, SSP-RK3, jittered triangles (%dx%d quads, %d triangles)" % (
            nq, nq, mesh.n_elems), "p": 2, "rk": "SSP(3,3)", "precision": "fp64"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": "oracle FP64 C++ restatement of the reference step (the reference needs Eigen, "
                                   "yaml-cpp and METIS, absent here), %dx%d quads, %d OpenMP threads" % (nq, nq, cores)},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def time_steps(P, K):
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    P.step_serial(K)
    wall = time.perf_counter() - t0
    ms, launches = P.last_step_timing()
    return ms, launches, wall


def limiter_workload(dev, steps=400, warmup=5):
    """The metric's "FP32 + MLP vs FP64 plain" on the limited workload it concerns: config 3 (Thacker bowl,
    131,072 triangles, p = 1, wetting/drying + Cockburn-Shu limiter). FP32 bulk with the learned
    indicator gating the limiter (confidence 0.9, committed weights) against the FP64 path with the
    plain limiter, plus FP32 with the plain limiter; device time of graph-replayed steps, L2 error
    against the analytic solution after the same number of steps."""
    from dgswemv2_b200 import Problem, configs, indicator

    W = indicator.load_weights()
    out = {"workload": "config 3: Thacker bowl, 131072 triangles, p=1, SSP-RK2, wetting/drying + limiter",
           "steps": steps + warmup}
    for name, prec, mode in (("fp32_mlp", "fp32", 1), ("fp32_plain", "fp32", 0), ("fp64_plain", "fp64", 0)):
        mesh, cfg = configs.config3(precision=prec)
        P = Problem(cfg, mesh, device=dev)
        if mode:
            P.set_indicator(W, confidence=0.9, mode=mode)
        P.step_serial(warmup)
        ms, _, _ = time_steps(P, steps)
        units = P.ne * P.nd * cfg.rk_nstages * steps
        out[name] = {"value": units / (ms / 1e3), "ms_per_step": ms / steps, "l2_error": P.compute_residual_L2()}
        if mode:
            c = P.indicator_stats()
            out[name]["sent_fraction"] = c[1] / max(1, c[0])
        del P
    out["speedup_fp32_mlp_over_fp64_plain"] = out["fp32_mlp"]["value"] / out["fp64_plain"]["value"]
    out["l2_ratio_fp32_mlp_over_fp64_plain"] = out["fp32_mlp"]["l2_error"] / out["fp64_plain"]["l2_error"]
    return out


def run_ours(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup(args.gpus)
    from dgswemv2_b200 import Problem, configs

    dev = local
    torch.cuda.set_device(dev)
    mesh, cfg = configs.config2(nq=args.nq, precision=args.precision)
    # tile size chosen by the library's autotuner (both sizes timed on this workload at create)
    P = Problem(cfg, mesh, device=dev, tile=-1)
    ne, nd, ns = P.ne, P.nd, cfg.rk_nstages
    units_per_step = ne * nd * ns

    # warm-up (includes CUDA-graph capture)
    P.step_serial(args.warmup)
    barrier(world)
    with ClockSampler(dev) as clk:
        ms, launches, wall = time_steps(P, args.steps)
        barrier(world)
    ms = dist_max(ms, world)
    value = job_value(units_per_step, args.steps, world, ms)

    # the FP64 plain path on the same workload (the comparator of the FP32 path)
    fp64 = None
    if args.precision == "fp32":
        mesh64, cfg64 = configs.config2(nq=args.nq, precision="fp64")
        P64 = Problem(cfg64, mesh64, device=dev, tile=-1)
        P64.step_serial(args.warmup)
        barrier(world)
        ms64, _, _ = time_steps(P64, args.steps)
        barrier(world)
        ms64 = dist_max(ms64, world)
        fp64 = {"value": job_value(units_per_step, args.steps, world, ms64), "ms_per_step": ms64 / args.steps,
                "tile_autotuned": P64.info.tile}
        l2_32, l2_64 = P.compute_residual_L2(), P64.compute_residual_L2()
        fp64["l2_error_fp64"] = l2_64
        fp64["l2_error_fp32"] = l2_32
        fp64["l2_ratio_fp32_over_fp64"] = l2_32 / l2_64
        del P64

    # end to end through the C ABI host API: H2D of the state from pinned memory, one RK step,
    # D2H of the new state, every step
    ke = max(3, min(args.steps, 40))
    host = torch.empty((ne, 3, nd), dtype=torch.float64).pin_memory()
    host.numpy()[:] = P.get_state()
    hq = host.numpy()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(ke):
        P.set_state(hq)
        P.step_serial(1)
        P.get_state(out=hq)
    torch.cuda.synchronize()
    e2e_s = dist_max(time.perf_counter() - t0, world)
    barrier(world)
    e2e = {"value": units_per_step * ke * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(hq.nbytes),
           "d2h_bytes_per_step": int(hq.nbytes), "steps": ke}

    peak, peak_kind = load_peaks()
    stage_ms = ms / (args.steps * ns)
    alg = ALG_BYTES_PER_UNIT[(args.precision, cfg.p)] * ne * nd
    achieved = alg / (stage_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": load_traffic(args.precision), "peak_kind": peak_kind,
                "kernel": "rkdg_stage_kernel<2,%s,...>" % ("float" if args.precision == "fp32" else "double"),
                "stage_kernel_ms": stage_ms, "algorithmic_bytes_per_launch": alg}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": "manufactured solution p=2 at scale: %dx%d quads -> %d jittered triangles, Dunavant "
                               "deg 4 / 3-pt Gauss-Legendre, LLF, SSP-RK3" % (args.nq, args.nq, ne),
                   "elements": ne, "p": 2, "rk": "SSP(3,3)", "precision": args.precision,
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "tile_fp32_autotuned": P.info.tile,
                   "l2_cache": "no flush: the per-step working set (%d MB of stage states, bathymetry and mesh "
                               "arrays) exceeds the 126 MB L2" % int(P.info.device_bytes / 2 ** 20)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "e2e": e2e,
        "roofline": roofline,
    }
    if fp64:
        out["fp64_plain"] = fp64
        out["speedup_fp32_over_fp64"] = value / fp64["value"]
    if args.precision == "fp32":
        out["limiter_workload"] = limiter_workload(dev)
        barrier(world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(args.nq, args.cpu_seconds, args.precision)
        except Exception as e:  # the CPU leg must not hide the GPU number
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                   "sample": "failed: %s" % e}
    if rank == 0:
        print(json.dumps(out))
    del P
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
