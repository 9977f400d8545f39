"""Analytic checks with an evaluator independent of the product (tests/analytic.py: numpy and scipy only).

CPU:
- the numpy Dubiner basis equals the reference's own table (test/test_basis_dubiner_2d.cpp, 66 modes at
  15 points) to 1e-13, which pins the basis the L2 errors below are evaluated with;
- function_sets.h (compiled into the library and the oracle) gives the configuration's manufactured
  solution and Thacker's bowl to 1e-13, and its source terms equal the residual of the shallow-water
  equations on the numpy solution (centred finite differences, 1e-6 of the source scale);
- Thacker's formula solves the frictionless shallow-water equations over the bowl (finite-difference
  residual 1e-6 of the momentum-flux scale).
GPU (FP64):
- h-refinement of the manufactured solution at p = 1 (SSP-RK2) and p = 2 (SSP-RK3): the numpy L2 error of
  the GPU state falls at an observed order >= p + 0.5 on the finest pair of meshes, and the library's own
  L2 error equals the numpy one to 1e-6 (different quadrature rules);
- the Thacker bowl with wetting/drying and the limiter: the error at a quarter period falls with each
  refinement of the mesh.
The reference sweeps mesh size, order and time step the same way in scripts/correctness/auto_runner_serial.sh.
"""
import json
import math
import os

import numpy as np
import pytest

from dgswemv2_b200 import Problem, configs
from dgswemv2_b200.types import FN_MANUFACTURED_SINE, FN_THACKER_BOWL

from . import analytic

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_numpy_dubiner_basis_equals_the_reference_table():
    with open(os.path.join(GOLD, "dubiner_2d.json")) as f:
        d = json.load(f)
    pts = np.asarray(d["points"])
    phi = analytic.dubiner_phi(d["p"], pts[:, 0], pts[:, 1])
    ref = np.asarray(d["phi"])
    assert phi.shape == ref.shape == (66, 15)
    assert np.abs(phi - ref).max() <= 1e-13 * np.abs(ref).max()


def test_collapsed_rule_is_exact_to_degree_14():
    z1, z2, w = analytic.collapsed_rule(8)
    for px in range(8):
        for py in range(8 - px):
            # int over the master triangle (area 2) of ((1 + z1)/2)^px ((1 + z2)/2)^py = 4 px! py! / (px + py + 2)!
            exact = 4.0 * math.factorial(px) * math.factorial(py) / math.factorial(px + py + 2)
            got = float(np.sum(((1 + z1) / 2) ** px * ((1 + z2) / 2) ** py * w))
            assert abs(got - exact) <= 1e-14, (px, py)


def swe_residual(sol, t, x, y, bath, g, ds, dt):
    """Residual of the shallow-water equations (frictionless, depth h = ze + b) by centred differences of
    step ds in space and dt in time:
    [ze_t + qx_x + qy_y, qx_t + (qx^2/h)_x + (qx qy/h)_y + g h ze_x, qy_t + (qx qy/h)_x + (qy^2/h)_y + g h ze_y]."""
    def at(xx, yy, tt):
        ze, qx, qy = sol(tt, xx, yy)
        return ze, qx, qy, ze + bath(xx, yy)

    _, _, _, h = at(x, y, t)
    q_t = (sol(t + dt, x, y) - sol(t - dt, x, y)) / (2 * dt)
    zxp, qxxp, qyxp, hxp = at(x + ds, y, t)
    zxm, qxxm, qyxm, hxm = at(x - ds, y, t)
    zyp, qxyp, qyyp, hyp = at(x, y + ds, t)
    zym, qxym, qyym, hym = at(x, y - ds, t)
    d = 2 * ds
    r0 = q_t[0] + (qxxp - qxxm) / d + (qyyp - qyym) / d
    r1 = q_t[1] + (qxxp ** 2 / hxp - qxxm ** 2 / hxm) / d + (qxyp * qyyp / hyp - qxym * qyym / hym) / d + \
        g * h * (zxp - zxm) / d
    r2 = q_t[2] + (qxxp * qyxp / hxp - qxxm * qyxm / hxm) / d + (qyyp ** 2 / hyp - qyym ** 2 / hym) / d + \
        g * h * (zyp - zym) / d
    return np.stack([r0, r1, r2])


def test_function_set_manufactured_solution_and_sources(oracle):
    M = analytic.Manufactured()
    params = configs.sine_params()
    rng = np.random.default_rng(3)
    x = rng.uniform(0, M.L, 400)
    y = rng.uniform(0, M.L, 400)
    for t in (0.0, 137.0, 1000.0, 4321.0):
        true_h = oracle.fn_eval(FN_MANUFACTURED_SINE, params, t, 0, x, y)
        true_n = M(t, x, y).T
        assert np.abs(true_h - true_n).max() <= 1e-13 * max(M.A, M.B)
        src_h = oracle.fn_eval(FN_MANUFACTURED_SINE, params, t, 1, x, y)
        res = swe_residual(M, t, x, y, M.bath, M.g, ds=1.0, dt=1e-3).T
        scale = np.abs(res[:, 1:]).max() + 1e-30
        assert np.abs(src_h[:, 0]).max() <= 1e-15  # continuity holds without a source
        assert np.abs(res[:, 0]).max() <= 1e-6 * M.A * M.w
        assert np.abs(src_h[:, 1:] - res[:, 1:]).max() <= 1e-6 * max(scale, M.g * M.H * M.A * M.k), t


def test_function_set_thacker_bowl(oracle):
    T = analytic.Thacker()
    params = configs.thacker_params()
    rng = np.random.default_rng(4)
    x = rng.uniform(-4000, 4000, 500)
    y = rng.uniform(-4000, 4000, 500)
    assert np.abs(oracle.fn_eval(FN_THACKER_BOWL, params, 0.0, 2, x, y) - T.bath(x, y)).max() <= 1e-12
    period = 2 * math.pi / T.w
    assert abs(period - configs.thacker_period()) <= 1e-9
    for t in (0.0, 0.1 * period, 0.37 * period, 0.5 * period, 0.9 * period):
        h = oracle.fn_eval(FN_THACKER_BOWL, params, t, 0, x, y)
        n = T(t, x, y).T
        assert np.abs(h - n).max() <= 1e-12 * 20.0, t
        # the formula solves the equations where the water column is well away from the shoreline
        xs = rng.uniform(-1500, 1500, 200)
        ys = rng.uniform(-1500, 1500, 200)
        ze, qx, qy = T(t, xs, ys)
        assert np.all(ze + T.bath(xs, ys) > 1.0)
        res = swe_residual(T, t, xs, ys, T.bath, T.g, ds=0.5, dt=1e-2)
        mom = T.g * (ze + T.bath(xs, ys)) * T.h0 / T.a  # momentum-flux gradient scale
        assert np.abs(res[0]).max() <= 1e-5 * max(np.abs(qx).max(), 1.0) / T.a, t
        assert np.abs(res[1:]).max() <= 1e-6 * mom.max(), t


def l2_pair(P, mesh, true, order):
    """(numpy L2 error of the GPU state, the library's L2 error)."""
    q = P.get_state()
    t = P.time()[0]
    return analytic.l2_error(q, mesh.node_xyz, mesh.elem_nodes, order, true, t), P.compute_residual_L2()


@pytest.mark.gpu
@pytest.mark.parametrize("p,rk", [(1, (2, 2)), (2, (3, 3))])
def test_manufactured_h_convergence(p, rk):
    """nq x nq quads (nq = 8, 16, 32, 64; jitter 0.1) on the config-1 square, to t = 200 s with dt = 0.05 s.
    The time step is small because the reference's SSP-RK stage times all equal the step's start time
    (the crk/drk recurrence of explicit_ssp_rk_stepper.cpp:262-277 gives zero offsets for these tables),
    so a time-dependent source enters at first order in dt: at dt = 4 s to t = 2000 s that error, about
    8 in this L2 norm, hides the p = 2 spatial error from 32^2 quads on."""
    M = analytic.Manufactured()
    errs = []
    for nq in (8, 16, 32, 64):
        mesh, cfg = configs.manufactured(nq, p=p, rk=rk, dt=0.05, jitter=0.1, seed=5)
        P = Problem(cfg, mesh)
        P.step_serial(4000)
        assert abs(P.time()[0] - 200.0) <= 1e-9
        e_np, e_lib = l2_pair(P, mesh, M, p)
        assert abs(e_np - e_lib) <= 1e-6 * e_lib, (nq, e_np, e_lib)
        errs.append(e_np)
    orders = [math.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
    assert all(o > 0.8 * p for o in orders), (errs, orders)
    assert orders[-1] >= p + 0.5, (errs, orders)


@pytest.mark.gpu
def test_thacker_bowl_error_falls_with_refinement():
    """The config-3 bowl (wetting/drying, limiter, p = 1, SSP-RK2) at 32^2, 64^2 and 128^2 quads, a quarter
    period (168 s) with dt = 1, 0.5, 0.25 s: the numpy L2 error against Thacker's solution falls with each
    refinement (the wet/dry front limits the order) and equals the library's own L2 error to 1e-3."""
    T = analytic.Thacker()
    period = configs.thacker_period()
    errs = []
    for nq, dt in ((32, 1.0), (64, 0.5), (128, 0.25)):
        mesh, cfg = configs.config3(nq=nq, dt=dt)
        P = Problem(cfg, mesh)
        n = int(round(0.25 * period / dt))
        P.step_serial(n)
        e_np, e_lib = l2_pair(P, mesh, T, 1)
        assert abs(e_np - e_lib) <= 1e-3 * e_lib, (nq, e_np, e_lib)
        errs.append(e_np)
    assert errs[0] > errs[1] > errs[2], errs
    assert errs[0] / errs[2] > 2.0, errs
