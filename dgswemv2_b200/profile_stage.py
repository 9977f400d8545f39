"""Small driver for profiling the RK stage kernel, two steps without CUDA graphs (each stage is a
separate launch, so `ncu -k regex:rkdg_stage_kernel -s <n> -c <m>` selects stages of step 2):

    python -m dgswemv2_b200.profile_stage fp32 [nq] [workload]

workload "manufactured" (default): config 2, p = 2 manufactured solution on nq x nq jittered quads
(nq = 512: 524,288 triangles), SSP-RK3; "bowl": config 3, Thacker bowl on nq x nq quads (nq = 256:
131,072 triangles), p = 1, SSP-RK2, wetting/drying and the slope limiter (stage kernel, then limiter
kernel, per stage); "tidal_p1" / "tidal_p2": the tidal channel of 524,288 triangles with tide and
river-flow boundaries, Manning friction and a ramp (nq is ignored).
"""
import sys

from . import Problem, configs


def main():
    prec = sys.argv[1] if len(sys.argv) > 1 else "fp32"
    workload = sys.argv[3] if len(sys.argv) > 3 else "manufactured"
    if workload.startswith("tidal"):
        from . import throughput
        mesh, cfg = throughput.build(workload, prec)
    elif workload == "bowl":
        nq = int(sys.argv[2]) if len(sys.argv) > 2 else 256
        mesh, cfg = configs.config3(nq=nq, precision=prec)
    else:
        nq = int(sys.argv[2]) if len(sys.argv) > 2 else 512
        mesh, cfg = configs.config2(nq=nq, precision=prec)
    P = Problem(cfg, mesh, use_graphs=False)
    P.step_serial(2)
    P.synchronize()
    print("ok", prec, workload, P.ne)


if __name__ == "__main__":
    main()
