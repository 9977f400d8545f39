"""Small driver for profiling the RK stage kernel: config 2 (p = 2 manufactured solution on 512 x 512
jittered quads, 524,288 triangles, SSP-RK3) in one precision, two steps without CUDA graphs (each stage
is a separate launch, so `ncu -k regex:rkdg_stage_kernel -s 3 -c 1` selects the first stage of step 2).

    python -m dgswemv2_b200.profile_stage fp32 [nq]
"""
import sys

from . import Problem, configs


def main():
    prec = sys.argv[1] if len(sys.argv) > 1 else "fp32"
    nq = int(sys.argv[2]) if len(sys.argv) > 2 else 512
    mesh, cfg = configs.config2(nq=nq, precision=prec)
    P = Problem(cfg, mesh, use_graphs=False)
    P.step_serial(2)
    P.synchronize()
    print("ok", prec, P.ne)


if __name__ == "__main__":
    main()
