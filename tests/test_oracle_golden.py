"""Pin the CPU oracle against the known-answer vectors of the reference's own unit tests
(tests/golden/*.json, extracted from test/*.cpp by tests/golden/make_golden.py)."""
import json
import math
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
EPS = np.finfo(np.float64).eps


def almost_equal(a, b, factor=100.0):
    """source/utilities/almost_equal.hpp:16-22: relative |a-b| < factor*eps (absolute near zero)."""
    m = max(abs(a), abs(b))
    if m < EPS * factor:
        return True
    return abs(a - b) < m * EPS * factor


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def test_llf_flux_golden(oracle):
    d = load("llf_flux.json")
    assert len(d["cases"]) == 3
    for c in d["cases"]:
        F = oracle.llf_flux(d["gravity"], c["q_in"], c["q_ex"], c["bath"], c["sp"], c["normal"])
        for got, exp in zip(F, c["F_expected"]):
            assert almost_equal(exp, got, d["tolerance_factor"]), (c["config"], got, exp)


def test_dubiner_golden(oracle):
    d = load("dubiner_2d.json")
    phi, d1, d2 = oracle.dubiner(d["p"], d["points"])
    nd = (d["p"] + 1) * (d["p"] + 2) // 2
    assert nd == len(d["phi"]) == 66
    for dof in range(nd):
        for pt in range(len(d["points"])):
            assert almost_equal(d["phi"][dof][pt], phi[dof, pt], d["phi_tolerance_factor"]), (dof, pt)
            assert almost_equal(d["dphi"][dof][2 * pt], d1[dof, pt], d["dphi_tolerance_factor"]), (dof, pt)
            assert almost_equal(d["dphi"][dof][2 * pt + 1], d2[dof, pt], d["dphi_tolerance_factor"]), (dof, pt)


def test_element_integrals_golden(oracle):
    d = load("element_triangle.json")
    integ, ip, ix, iy = oracle.element_integrals(d["p"], d["vertices"], d["f_terms"])
    tol = d["tolerance_factor"]
    assert almost_equal(d["IntegrationPhi_true"][0], integ, tol)
    for dof in range(66):
        assert almost_equal(d["IntegrationPhi_true"][dof], ip[dof], tol), ("phi", dof, ip[dof])
        assert almost_equal(d["IntegrationDPhiDX_true"][dof], ix[dof], tol), ("dx", dof, ix[dof])
        assert almost_equal(d["IntegrationDPhiDY_true"][dof], iy[dof], tol), ("dy", dof, iy[dof])


def test_wetting_drying_golden(oracle):
    d = load("wetting_drying.json")
    assert len(d["cases"]) == 5
    for c in d["cases"]:
        q, wet = oracle.wet_dry_single(d["vertices"], d["bath_vrtx"], d["h_o"], c["q_vrtx_in"], c["wet_in"])
        if c["expect_wet"] is not None:
            assert wet == c["expect_wet"], c["name"]
        for key, (val, tol) in c["expected"].items():
            var = "ze qx qy".split().index(key[:2])
            assert almost_equal(q[var, int(key[2])], val, tol), (c["name"], key, q[var, int(key[2])], val)


@pytest.mark.parametrize("degree", range(1, 20))
def test_dunavant_exactness(oracle, degree):
    """test/test_integ_dunavant_2d.cpp:11-37: int x^p over the master triangle, within 1e3 eps."""
    w, z1, z2 = oracle.triangle_rule(degree)
    p = degree
    exact = 1 / (p + 1) * ((1 - (-1.0) ** p) / (p + 2) + 2 * (-1.0) ** p)
    assert almost_equal(float(np.sum(z1 ** p * w)), exact, 1.0e3)


@pytest.mark.parametrize("degree", range(1, 20))
def test_gauss_legendre_exactness(oracle, degree):
    """test/test_integ_gausslegendre_1d.cpp:11-27: int (1 - x^p) over [-1,1]."""
    w, z = oracle.gl_rule(degree)
    p = degree
    exact = 2.0 - (1 - (-1.0) ** (p + 1)) / (p + 1)
    assert almost_equal(float(np.sum((1 - z ** p) * w)), exact, 1.0e3)
    assert len(w) == math.ceil((degree + 1) / 2)


def test_gauss_legendre_tabulated_points(oracle):
    """GL nodes of the reference table (integration_gausslegendre_1D.cpp:41-54) to double rounding."""
    w, z = oracle.gl_rule(3)
    assert z[1] == pytest.approx(0.577350269189625764509148780502, abs=2 * EPS)
    w, z = oracle.gl_rule(5)
    assert z[2] == pytest.approx(0.774596669241483377035853079956, abs=2 * EPS)
    assert w[1] == pytest.approx(0.888888888888888888888888888889, abs=2 * EPS)


@pytest.mark.parametrize("pair", [(1, 1), (2, 2), (3, 3), (4, 3), (5, 3), (6, 3), (7, 3), (5, 4), (6, 4), (7, 4), (8, 4)])
def test_rk_stepper_ode(oracle, pair):
    """test/test_rk_stepper.cpp:13-80: y'' + y = t/2, y(0)=0, y'(0)=1.5 -> sin t + t/2 at t ~ 5, within 1e-2.
    dt = 5e-4 instead of the reference's 5e-5 keeps the run short; forward Euler still meets the 1e-2 bound."""
    ns, order = pair
    a, b, drk = oracle.rk_table(ns, order)
    a = a.tolist()
    b = b.tolist()
    dt = 5e-4
    nsteps = int(5.0 / dt) + 1
    y0 = [[0.0, 0.0] for _ in range(ns + 1)]
    y0[0] = [0.0, 1.5]
    rhs = [[0.0, 0.0] for _ in range(ns)]
    t = 0.0
    for _ in range(nsteps):
        for st in range(ns):
            ts = t + dt * drk[st]
            rhs[st] = [y0[st][1], -y0[st][0] + 0.5 * ts]
            u = v = 0.0
            for s in range(st + 1):
                u += a[st][s] * y0[s][0] + dt * b[st][s] * rhs[s][0]
                v += a[st][s] * y0[s][1] + dt * b[st][s] * rhs[s][1]
            y0[st + 1] = [u, v]
        y0[0], y0[ns] = y0[ns], y0[0]
        t += dt
    assert abs(y0[0][0] - math.sin(t) - 0.5 * t) < 1e-2


def test_stage_times_follow_reference_recurrence(oracle):
    """The reference's crk/drk recurrence leaves every stage time at t for these tables
    (explicit_ssp_rk_stepper.cpp:262-277)."""
    for pair in [(2, 2), (3, 3)]:
        _, _, d = oracle.rk_table(*pair)
        assert np.all(d == 0.0)
