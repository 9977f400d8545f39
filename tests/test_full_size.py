"""Parity at the named configurations' full size and length (GPU against the FP64 oracle on the same
mesh, initial condition and step count; the oracle runs on all host cores).

- config 2: 512 x 512 quads -> 524,288 jittered triangles, p = 2, SSP-RK3, dt = 0.5 s, 20 steps:
  FP64 GPU state within 1e-12 of each variable in the L2 sense (pointwise within 2e-12 of its largest
  value), L2 errors equal to 1e-12; the FP32-bulk path's L2
  error within 1.05x of the FP64 oracle's.
- config 3: the Thacker bowl at 256 x 256 quads -> 131,072 triangles, p = 1, SSP-RK2, wetting/drying and
  the Cockburn-Shu limiter, dt = 0.25 s for two periods (5,383 steps): FP64 GPU against the oracle (wet
  counts within 0.5 %, state within 1e-8 of each variable's scale, L2 within 1e-6), and the L2 error
  against Thacker's solution of the FP32-bulk path and of FP32 with the learned indicator gating the
  limiter, each within 1.05x of the FP64 oracle's (Simulation::ComputeL2Residual,
  source/simulation/serial/simulation.hpp:85-93).
- config 5 members over the configuration's whole size range (64^2 to 200^2 quads): in one ensemble
  handle, each member equals its own single run to 1e-12 (FP64) with identical wet flags, for 100 steps.
"""
import os

import numpy as np
import pytest

from dgswemv2_b200 import Problem, configs, ensemble, indicator

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 8


def rel_err(a, b):
    out = 0.0
    for v in range(3):
        scale = max(np.max(np.abs(b[:, v, :])), 1e-300)
        out = max(out, np.max(np.abs(a[:, v, :] - b[:, v, :])) / scale)
    return out


def test_config2_full_size_fp64_and_fp32(oracle):
    mesh, cfg = configs.config2()
    assert mesh.n_elems == 524288
    O = oracle.problem(cfg, mesh, n_threads=THREADS)
    P = Problem(cfg, mesh)
    assert rel_err(P.get_state(), O.get_state()) <= 1e-13
    P.step_serial(20)
    O.step(20)
    qg, qo = P.get_state(), O.get_state()
    diag = {"max_rel_per_variable": [float(np.abs(qg[:, v] - qo[:, v]).max() / np.abs(qo[:, v]).max()) for v in range(3)],
            "l2_rel_per_variable": [float(np.linalg.norm(qg[:, v] - qo[:, v]) / np.linalg.norm(qo[:, v])) for v in range(3)]}
    # each variable within 1e-12 relative in the L2 sense; the largest pointwise difference within 2e-12 of
    # the variable's largest value (measured 1.2e-12 in qy, whose largest value at t = 10 s is 1 % of its
    # amplitude)
    assert max(diag["l2_rel_per_variable"]) <= 1e-12, diag
    assert max(diag["max_rel_per_variable"]) <= 2e-12, diag
    lo = O.l2_error()
    assert abs(P.compute_residual_L2() - lo) <= 1e-12 * lo
    del P
    m32, c32 = configs.config2(precision="fp32")
    P32 = Problem(c32, m32)
    P32.step_serial(20)
    assert P32.compute_residual_L2() <= 1.05 * lo


@pytest.mark.slow
def test_config3_two_periods(oracle):
    mesh, cfg = configs.config3()
    assert mesh.n_elems == 131072
    nsteps = int(round(2 * configs.thacker_period() / cfg.dt))  # t = 1345.75 s, two periods of 672.9 s
    assert nsteps == 5383
    O = oracle.problem(cfg, mesh, n_threads=THREADS)
    O.step(nsteps)
    lo = O.l2_error()
    P = Problem(cfg, mesh)
    P.step_serial(nsteps)
    wg, wo = P.get_wet(), O.get_wet()
    assert abs(int(wg.sum()) - int(wo.sum())) <= 0.005 * mesh.n_elems
    assert rel_err(P.get_state(), O.get_state()) <= 1e-8
    assert abs(P.compute_residual_L2() - lo) <= 1e-6 * lo
    del P
    W = indicator.load_weights()
    for gated in (False, True):
        m32, c32 = configs.config3(precision="fp32")
        P32 = Problem(c32, m32)
        if gated:
            P32.set_indicator(W, confidence=0.9, mode=1)
        P32.step_serial(nsteps)
        l32 = P32.compute_residual_L2()
        assert l32 <= 1.05 * lo, (gated, l32, lo)
        del P32


def test_config5_members_across_the_size_range():
    sizes = (64, 112, 156, 200)
    meshes, cfgs = [], []
    for k, n in enumerate(sizes):
        m, c = configs.ensemble_member(n, 1000 + k, precision="fp64")
        meshes.append(m)
        cfgs.append(c)
    assert meshes[0].n_elems == 8192 and meshes[-1].n_elems == 80000
    E = ensemble(cfgs[0], meshes, [c.fn_params for c in cfgs], tile=0)
    E.step_serial(100)
    q, w = E.get_state(), E.get_wet()
    for k, (m, c) in enumerate(zip(meshes, cfgs)):
        first, n = E.member_range(k)
        assert n == m.n_elems
        P = Problem(c, m)
        P.step_serial(100)
        assert rel_err(q[first:first + n], P.get_state()) <= 1e-12, k
        assert np.array_equal(w[first:first + n], P.get_wet()), k
