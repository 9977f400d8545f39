"""Device throughput of the RK step on the named configurations, in FP32 bulk and FP64:

    python -m dgswemv2_b200.throughput [config2 config3 ...] [--steps N]

config1: manufactured sine, 800 triangles, p = 1, SSP-RK2 (fits in L2: a latency figure, not a roofline one)
config2: manufactured sine, 524,288 jittered triangles, p = 2, SSP-RK3
config3: Thacker bowl, 131,072 triangles, p = 1, SSP-RK2, wetting/drying + Cockburn-Shu limiter
config3_nolim: the same without the limiter
config4: Thacker bowl, 2,097,152 triangles, p = 1, SSP-RK2, wetting/drying + limiter
tidal_p1 / tidal_p2: 100 km x 25 km tidal channel, 524,288 triangles, M2 + K1 tide, river flow, Manning
  friction, forcing ramp (p = 1 SSP-RK2 dt = 0.5 s / p = 2 SSP-RK3 dt = 0.25 s)
levee_p1: the same channel cut across by a levee (256 levee interfaces), p = 1, SSP-RK2, dt = 0.5 s
Prints one JSON line per (configuration, precision): device ms per step after warm-up (CUDA events on
the handle's stream around graph-replayed steps), element-DOF updates per second per RK stage, the
L2 error against the analytic solution at the end, and the host wall time of the handle's creation
(topology, tiling, projections, uploads, initial state).

Options for measuring single kernels (for instance under a profiler): --no-graphs launches every stage
separately, --warmup sets the untimed steps, --tile fixes the tile size (default: the library's default,
-1: the autotuner), --indicator 1 gates the limiter with the committed learned indicator (2: shadow
mode), --trouble evaluates the KXRCF trouble indicator in each limiter pass, --postprocess computes the
writers' output values once after the steps, --fp64-stages keeps the FP32 path's intermediate stage states
in FP64 instead of FP32 increments.
"""
import argparse
import json
import time

from . import Problem, configs


def build(name, precision):
    if name == "config1":
        return configs.config1(precision=precision)
    if name == "config2":
        return configs.config2(precision=precision)
    if name == "config3":
        return configs.config3(precision=precision)
    if name == "config3_nolim":
        return configs.config3(precision=precision, limiter=False)
    if name == "config4":
        return configs.config3(nq=1024, dt=0.06, precision=precision)
    big = dict(nx=1024, ny=256, length=1.0e5, width=2.5e4, precision=precision)
    if name == "tidal_p1":
        return configs.tidal_channel(p=1, rk=(2, 2), dt=0.5, friction="manning", cf=0.0005, **big)
    if name == "tidal_p2":
        return configs.tidal_channel(p=2, rk=(3, 3), dt=0.25, friction="manning", cf=0.0005, **big)
    if name == "levee_p1":
        return configs.levee_channel(p=1, rk=(2, 2), dt=0.5, **big)
    raise ValueError(name)


def measure(name, precision, steps, warmup=5, graphs=True, tile=0, indicator=0, trouble=False, postprocess=False,
            fp64_stages=False):
    mesh, cfg = build(name, precision)
    t0 = time.perf_counter()
    P = Problem(cfg, mesh, use_graphs=graphs, tile=tile, fp64_stages=fp64_stages)
    create_s = time.perf_counter() - t0
    if indicator:
        from . import indicator as ind

        P.set_indicator(ind.load_weights(), confidence=0.9, mode=indicator)
    if trouble:
        P.set_trouble(True)
    P.step_serial(warmup)
    P.step_serial(steps)
    ms, launches = P.last_step_timing()
    per_step = ms / steps
    if postprocess:
        P.postprocess()
    return {
        "config": name, "precision": precision, "elements": P.ne, "p": cfg.p, "stages": cfg.rk_nstages,
        "tile": P.info.tile, "steps": steps, "ms_per_step": per_step,
        "element_dof_per_s_per_stage": P.ne * P.nd * cfg.rk_nstages / (per_step * 1e-3),
        "kernel_launches_per_step": launches / steps, "l2_error": P.compute_residual_L2(),
        "create_seconds": create_s, "occupancy": P.info.occupancy, "tile_order": P.info.tile_order,
        "graphs": graphs, "indicator": indicator, "stage_increments": P.info.stage_increments,
        "smem_capped": P.info.smem_capped,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("configs", nargs="*", default=["config1", "config2", "config3", "config3_nolim", "config4", "tidal_p1",
                                                   "tidal_p2", "levee_p1"])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--precisions", default="fp32,fp64")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--indicator", type=int, default=0, choices=[0, 1, 2])
    ap.add_argument("--trouble", action="store_true")
    ap.add_argument("--postprocess", action="store_true")
    ap.add_argument("--fp64-stages", action="store_true")
    a = ap.parse_args()
    for name in a.configs:
        for prec in a.precisions.split(","):
            print(json.dumps(measure(name, prec, a.steps, a.warmup, graphs=not a.no_graphs, tile=a.tile,
                                     indicator=a.indicator, trouble=a.trouble, postprocess=a.postprocess,
                                     fp64_stages=a.fp64_stages)), flush=True)


if __name__ == "__main__":
    main()
