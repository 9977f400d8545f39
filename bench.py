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
# compulsory HBM bytes per element-DOF per RK stage (each array touched once), p = 2 SSP-RK3 and p = 1
# SSP-RK2, keyed (precision, p, stage increments): element geometry and bathymetry (FP32 in the FP32 path)
# and the edge records, plus the stage states. FP64 stage states: q_s read, q_{s+1} written, q_0 read by
# the stages after the first. FP32 stage increments: the carried state's leading FP32 part q0f (4 B) and the
# increment d_s (4 B) read, d_{s+1} (4 B) written; the last stage also reads the trailing part q0lo (4 B)
# and writes both parts of the new carried state (8 B).
ALG_BYTES_PER_UNIT = {("fp32", 2, 0): 77.0, ("fp64", 2, 0): 87.0, ("fp32", 1, 0): 82.0, ("fp64", 1, 0): 99.0,
                      ("fp32", 2, 1): 53.0}


def workload_name(nq, ne):
    return ("manufactured solution p=2 at scale: %dx%d quads -> %d jittered triangles, Dunavant deg 4 / "
            "3-pt Gauss-Legendre, LLF, SSP-RK3" % (nq, nq, ne))


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
    """SM clock, power and throttle reasons sampled while the timed region runs: NVML polled every 2 ms
    from a thread (a short timed region still gets samples), else nvidia-smi at its 100 ms minimum."""

    NVML_REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
                    ("sw_power_cap", 0x4))
    SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []  # (sm_mhz, max_mhz, power_w, set of reasons)
        self.proc = None
        self.nv = None
        self._stop = threading.Event()
        self._t = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.device)
        try:
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _sample_nvml(self):
        nv, h = self.nv
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
        try:
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.samples.append((float(sm), float(smax), pw, {n for n, bit in self.NVML_REASONS if r & bit}))

    def _poll(self):
        while not self._stop.is_set():
            try:
                self._sample_nvml()
            except Exception:
                return
            time.sleep(0.002)

    def _read_smi(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm, smax, pw = float(parts[1]), float(parts[2]), float(parts[3])
            except ValueError:
                continue
            self.samples.append((sm, smax, pw, {n for n, v in zip(names, parts[5:9]) if v.lower().startswith("active")}))

    def __enter__(self):
        try:
            self.nv = self._nvml_handle()
            self._sample_nvml()
            self._t = threading.Thread(target=self._poll, daemon=True)
        except Exception:
            self.nv = None
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.SMI_FIELDS,
                     "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE,
                    stderr=subprocess.DEVNULL, text=True)
                self._t = threading.Thread(target=self._read_smi, daemon=True)
            except Exception:
                self.proc = None
        if self._t:
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.nv:
            self._t.join(timeout=2)
            try:
                self._sample_nvml()
            except Exception:
                pass
        elif self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self._t.join(timeout=2)

    def summary(self):
        sm = [x[0] for x in self.samples]
        reasons = set()
        for x in self.samples:
            reasons |= x[3]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": self.samples[-1][1] if self.samples else None, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max((x[2] for x in self.samples), default=None),
                "source": "nvml 2 ms" if self.nv else "nvidia-smi 100 ms"}


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


def load_traffic(key):
    """DRAM bytes per stage-kernel launch (read + write, mean over the stages of one step) from the
    committed ncu summary of this workload, if any; key "fp32_increments", "fp32" or "fp64"."""
    try:
        with open(os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")) as f:
            d = json.load(f)
        return d.get(key)
    except Exception:
        return None


def oracle_rate(nq, seconds, threads):
    """FP64 oracle steps of the config-2 discretisation on an nq x nq mesh for about `seconds`:
    (element-DOF/s, steps, elapsed s, triangles)."""
    from dgswemv2_b200 import configs
    from tests.oracle_ctypes import Oracle

    O = Oracle(os.path.join(ROOT, "oracle", "build", "liboracle.so"))
    mesh, cfg = configs.config2(nq=nq)
    P = O.problem(cfg, mesh, n_threads=threads)
    P.step(1)  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        P.step(1)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 1000:
            break
    return mesh.n_elems * 6 * 3 * n / el, n, el, mesh.n_elems


def cpu_baseline(nq, seconds):
    """The oracle (FP64 C++ restatement of the reference step) on the host cores, on bounded samples of the
    workload: all host threads (OpenMP) on a quarter-size mesh, and one thread (the reference's serial
    driver) on an eighth-size mesh."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    cores = os.cpu_count() or 1
    sub = max(32, nq // 4)
    v, n, el, ne = oracle_rate(sub, seconds, cores)
    sub1 = max(16, nq // 8)
    v1, n1, el1, ne1 = oracle_rate(sub1, seconds / 2, 1)
    return {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "oracle (FP64 C++ restatement of the reference step) on the same discretisation at %dx%d quads "
                      "(%d triangles), %d SSP-RK3 steps in %.1f s, %d OpenMP threads" % (sub, sub, ne, n, el, cores),
            "serial": {"value": v1, "unit": UNIT, "cores": 1,
                       "sample": "the same oracle on one thread (as the reference's serial driver runs), %dx%d quads "
                                 "(%d triangles), %d steps in %.1f s" % (sub1, sub1, ne1, n1, el1)}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    from dgswemv2_b200 import configs
    from tests.oracle_ctypes import Oracle

    cores = os.cpu_count() or 1
    O = Oracle(os.path.join(ROOT, "oracle", "build", "liboracle.so"))
    # each step is one SSP-RK3 step of the workload; when warm-up + timed steps would take more than
    # about two minutes on this host, the mesh is scaled down and the line says so
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
    sample = ("oracle FP64 C++ restatement of the reference step (the reference needs Eigen, yaml-cpp and METIS, "
              "absent here), %dx%d quads, %d OpenMP threads" % (nq, nq, cores))
    if nq != args.nq:
        sample += "; mesh scaled down from %dx%d to keep %d steps within %d s" % (args.nq, args.nq,
                                                                                  args.steps + args.warmup, budget)
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(nq, mesh.n_elems), "elements": mesh.n_elems, "p": 2, "rk": "SSP(3,3)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def autotuned(P):
    """The autotuner's choice and its timed candidates (tile, occupancy, tile order, ms per step; each the
    faster of the capped and the run-time-stride kernel where the mesh fits the caps)."""
    return {"tile": P.info.tile, "occupancy": P.info.occupancy, "tile_order": P.info.tile_order,
            "smem_capped": P.info.smem_capped, "candidates": [list(c) for c in P.tuning()]}


def time_steps(P, K):
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    P.step_serial(K)
    wall = time.perf_counter() - t0
    ms, launches = P.last_step_timing()
    return ms, launches, wall


def e2e_leg(P, steps, world):
    """The metric through the host API every step: set_state from pinned host memory, one RK step,
    get_state back into the same pinned buffer (wall clock, max over ranks)."""
    import torch

    ne, nd, ns = P.ne, P.nd, P.cfg.rk_nstages
    host = torch.empty((ne, 3, nd), dtype=torch.float64).pin_memory()
    hq = host.numpy()
    hq[:] = P.get_state()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        P.set_state(hq)
        P.step_serial(1)
        P.get_state(out=hq)
    torch.cuda.synchronize()
    el = dist_max(time.perf_counter() - t0, world)
    barrier(world)
    return {"value": ne * nd * ns * steps * world / el, "unit": UNIT, "h2d_bytes_per_step": int(hq.nbytes),
            "d2h_bytes_per_step": int(hq.nbytes), "steps": steps}


def limiter_workload(dev, steps=400, warmup=5, nq=256, dt=0.25, name="config 3: Thacker bowl, 131072 triangles"):
    """The metric's "FP32 + MLP vs FP64 plain" on the limited workloads it concerns: the Thacker bowl (p = 1,
    wetting/drying + Cockburn-Shu limiter). FP32 bulk with the learned indicator gating the limiter
    (confidence 0.9, committed weights) against the FP64 path with the plain limiter, plus FP32 with the
    plain limiter; device time of graph-replayed steps, L2 error against the analytic solution after the
    same number of steps."""
    from dgswemv2_b200 import Problem, configs, indicator

    W = indicator.load_weights()
    out = {"workload": name + ", p=1, SSP-RK2, wetting/drying + limiter", "steps": steps + warmup}
    for key, prec, mode in (("fp32_mlp", "fp32", 1), ("fp32_plain", "fp32", 0), ("fp64_plain", "fp64", 0)):
        mesh, cfg = configs.config3(nq=nq, dt=dt, precision=prec)
        P = Problem(cfg, mesh, device=dev)
        if mode:
            P.set_indicator(W, confidence=0.9, mode=mode)
        P.step_serial(warmup)
        ms, _, _ = time_steps(P, steps)
        units = P.ne * P.nd * cfg.rk_nstages * steps
        out[key] = {"value": units / (ms / 1e3), "ms_per_step": ms / steps, "l2_error": P.compute_residual_L2()}
        if mode:
            c = P.indicator_stats()
            out[key]["sent_fraction"] = c[1] / max(1, c[0])
        del P
    out["speedup_fp32_mlp_over_fp64_plain"] = out["fp32_mlp"]["value"] / out["fp64_plain"]["value"]
    out["l2_ratio_fp32_mlp_over_fp64_plain"] = out["fp32_mlp"]["l2_error"] / out["fp64_plain"]["l2_error"]
    return out


def ensemble_workload(dev, steps=20, warmup=3):
    """Config 5: 256 p = 1 members of 64^2 to 200^2 quads with wetting/drying, FP32 bulk, one autotuned
    stage-kernel launch per RK stage for all members, graph-replayed steps."""
    from dgswemv2_b200 import configs, ensemble

    meshes, cfgs = configs.config5(precision="fp32")
    t0 = time.perf_counter()
    E = ensemble(cfgs[0], meshes, [c.fn_params for c in cfgs], device=dev)
    create_s = time.perf_counter() - t0
    E.step_serial(warmup)
    ms, launches, _ = time_steps(E, steps)
    m0 = E.mass()
    return {"workload": "config 5: ensemble of 256 p=1 members (64^2-200^2 quads, %d triangles), wetting/drying, "
                        "FP32 bulk" % E.ne, "steps": steps, "value": E.ne * E.nd * E.cfg.rk_nstages * steps / (ms / 1e3),
            "ms_per_step": ms / steps, "autotuned": autotuned(E),
            "kernel_launches_per_step": launches / steps, "create_seconds": create_s, "mass": m0}


def run_ours(args):
    import torch

    world, rank, local = dist_setup(args.gpus)
    from dgswemv2_b200 import Problem, configs

    dev = local
    torch.cuda.set_device(dev)
    mesh, cfg = configs.config2(nq=args.nq, precision=args.precision)
    # tile size, register budget and tile order chosen by the library's autotuner (all timed at create)
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
    # the stage kernel's own duration: the same number of steps again, each stage-kernel launch bracketed
    # by CUDA events on the handle's stream (stages launched one by one)
    kms, klaunches = P.step_timed(args.steps)
    stage_ms = dist_max(kms / max(1, klaunches), world)
    e2e = e2e_leg(P, max(3, min(args.steps, 40)), world)

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
        k64, n64 = P64.step_timed(args.steps)
        fp64 = {"value": job_value(units_per_step, args.steps, world, ms64), "ms_per_step": ms64 / args.steps,
                "autotuned": autotuned(P64), "stage_kernel_ms": dist_max(k64 / max(1, n64), world)}
        fp64["stage_kernel_frac_of_hbm"] = (ALG_BYTES_PER_UNIT[("fp64", cfg.p, 0)] * ne * nd /
                                            (fp64["stage_kernel_ms"] / 1e3) / 1e9 / load_peaks()[0])
        fp64["e2e"] = e2e_leg(P64, max(3, min(args.steps, 40)), world)
        # both paths advanced the same steps: warm-up, timed, kernel-timed and e2e
        l2_32, l2_64 = P.compute_residual_L2(), P64.compute_residual_L2()
        fp64["l2_error_fp64"] = l2_64
        fp64["l2_error_fp32"] = l2_32
        fp64["l2_ratio_fp32_over_fp64"] = l2_32 / l2_64
        del P64

    peak, peak_kind = load_peaks()
    alg = ALG_BYTES_PER_UNIT[(args.precision, cfg.p, P.info.stage_increments)] * ne * nd
    achieved = alg / (stage_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": load_traffic(args.precision + ("_increments" if P.info.stage_increments else "")),
                "peak_kind": peak_kind,
                "kernel": "rkdg_stage_kernel<2,%s,...>" % ("float" if args.precision == "fp32" else "double"),
                "stage_kernel_ms": stage_ms, "stage_kernel_launches_timed": int(klaunches),
                "stage_states": "FP32 increments from a two-part FP32 carried state" if P.info.stage_increments else "FP64",
                "step_ms_over_stages": ms / (args.steps * ns), "algorithmic_bytes_per_launch": alg}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": workload_name(args.nq, ne), "elements": ne, "p": 2, "rk": "SSP(3,3)",
                   "l2_cache": "no flush: each step moves %d MB of stage states, bathymetry and mesh arrays "
                            "(algorithmic bytes), more than the 126 MB L2" % int(alg * ns / 1e6)},
        "precision": args.precision, "parallelism": "replicas" if world > 1 else "single GPU",
        "autotuned": autotuned(P),
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
        out["limiter_workload_config4"] = limiter_workload(dev, steps=50, nq=1024, dt=0.06,
                                                           name="config 4: Thacker bowl, 2097152 triangles")
        barrier(world)
        out["ensemble_workload"] = ensemble_workload(dev)
        barrier(world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(args.nq, args.cpu_seconds)
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
