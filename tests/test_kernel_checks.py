"""The reference's known-answer vectors through the CUDA device code itself (the library's kernel
self-check entry points run the stage kernel's llf_flux, ISP::Internal fix-ups and wetting_drying):

- LLF: the three configurations of test/test_llf_flux.cpp:66-171 (tests/golden/llf_flux.json), FP64 within
  the reference's own tolerance (100 eps relative), FP32 within 2e-6 relative;
- wetting/drying: the five single-element cases of test/test_wetting_drying.cpp:15-380
  (tests/golden/wetting_drying.json), within each case's stated tolerance;
- ISP::Internal::ComputeFlux (rkdg_swe_is_internal.hpp:26-95, no reference unit test): random states on
  both sides with every wet/dry combination, against the oracle's restatement, FP64 within 1e-13 of the flux scale.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from dgswemv2_b200 import _lib

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
EPS = np.finfo(np.float64).eps


def almost_equal(a, b, factor=100.0):
    """source/utilities/almost_equal.hpp:16-22: relative |a-b| < factor*eps (absolute near zero)."""
    m = max(abs(a), abs(b))
    if m < EPS * factor:
        return True
    return abs(a - b) < m * EPS * factor


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def up(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def llf_gpu(precision, g, qi, qe, bath, sp, n):
    lib = _lib.load()
    qi, qe = np.ascontiguousarray(qi, np.float64), np.ascontiguousarray(qe, np.float64)
    bath, sp, n = (np.ascontiguousarray(x, np.float64) for x in (bath, sp, n))
    F = np.zeros_like(qi)
    _lib.check(lib.dgsw_check_llf_flux(precision, len(qi), g, dp(qi), dp(qe), dp(bath), dp(sp), dp(n), dp(F)))
    return F


def test_llf_golden_vectors_through_the_cuda_flux():
    with open(os.path.join(GOLD, "llf_flux.json")) as f:
        d = json.load(f)
    cases = d["cases"]
    assert len(cases) == 3
    qi = np.array([c["q_in"] for c in cases])
    qe = np.array([c["q_ex"] for c in cases])
    bath = np.array([c["bath"] for c in cases])
    sp = np.array([c["sp"] for c in cases])
    n = np.array([c["normal"] for c in cases])
    F64 = llf_gpu(_lib.DGSW_FP64, d["gravity"], qi, qe, bath, sp, n)
    F32 = llf_gpu(_lib.DGSW_FP32, d["gravity"], qi, qe, bath, sp, n)
    for k, c in enumerate(cases):
        for v in range(3):
            exp = c["F_expected"][v]
            assert almost_equal(exp, F64[k, v], d["tolerance_factor"]), (c["config"], v, F64[k, v], exp)
            assert abs(F32[k, v] - exp) <= 2e-6 * max(abs(x) for x in c["F_expected"]), (c["config"], v, F32[k, v])


def linear_to_modal(vals):
    """Vertex values of a linear field -> its p = 1 Dubiner modes (the inverse of T_basis_linear:
    vertex values a - b - c, a - b + c, a + 2b)."""
    v0, v1, v2 = vals
    return [(v0 + v1 + v2) / 3.0, (-v0 - v1 + 2.0 * v2) / 6.0, (-v0 + v1) / 2.0]


def modal_to_linear(m):
    a, b, c = m
    return [a - b - c, a - b + c, a + 2.0 * b]


def test_wetting_drying_golden_cases_through_the_cuda_kernel():
    with open(os.path.join(GOLD, "wetting_drying.json")) as f:
        d = json.load(f)
    cases = d["cases"]
    assert len(cases) == 5
    n = len(cases)
    q = np.array([[linear_to_modal(c["q_vrtx_in"][v]) for v in range(3)] for c in cases], np.float64)
    bath = np.array([d["bath_vrtx"]] * n, np.float64)
    wet_in = np.array([1 if c["wet_in"] else 0 for c in cases], np.uint8)
    qo = np.zeros_like(q)
    wet_out = np.zeros(n, np.uint8)
    went_dry = np.zeros(n, np.uint8)
    lib = _lib.load()
    _lib.check(lib.dgsw_check_wetting_drying(n, dp(q), dp(bath), d["h_o"], up(wet_in), dp(qo), up(wet_out),
                                             up(went_dry)))
    for k, c in enumerate(cases):
        if c["expect_wet"] is not None:
            assert bool(wet_out[k]) == c["expect_wet"], c["name"]
        vert = [modal_to_linear(qo[k, v]) for v in range(3)]
        for key, (val, tol) in c["expected"].items():
            var = "ze qx qy".split().index(key[:2])
            got = vert[var][int(key[2])]
            assert almost_equal(got, val, tol), (c["name"], key, got, val)
    # went_completely_dry (mean vertex depth at or below the 1e6 h_o eps threshold) holds in none of the
    # five cases: the driest has a mean depth of 0.003 m
    assert not went_dry.any()


def test_internal_flux_with_wet_dry_fixups_against_the_oracle(oracle):
    rng = np.random.default_rng(11)
    n = 4096
    g = 9.81
    bath_in = rng.uniform(0.5, 3.0, n)
    bath_ex = bath_in + rng.uniform(-0.2, 0.2, n)
    qi = np.stack([rng.uniform(-0.3, 0.5, n), rng.normal(0, 0.5, n), rng.normal(0, 0.5, n)], 1)
    qe = np.stack([rng.uniform(-0.3, 0.5, n), rng.normal(0, 0.5, n), rng.normal(0, 0.5, n)], 1)
    th = rng.uniform(0, 2 * np.pi, n)
    nrm = np.stack([np.cos(th), np.sin(th)], 1)
    sp = np.ones(n)
    wet_in = (rng.uniform(size=n) < 0.7).astype(np.uint8)
    wet_ex = (rng.uniform(size=n) < 0.7).astype(np.uint8)
    lib = _lib.load()
    Fi = np.zeros((n, 3))
    Fe = np.zeros((n, 3))
    _lib.check(lib.dgsw_check_internal_flux(_lib.DGSW_FP64, n, g, dp(qi), dp(qe), dp(bath_in), dp(bath_ex), dp(sp),
                                            dp(nrm), up(wet_in), up(wet_ex), dp(Fi), dp(Fe)))
    kinds = set()
    for k in range(n):
        ri, re_ = oracle.internal_flux(g, qi[k], qe[k], bath_in[k], bath_ex[k], 1.0, nrm[k], wet_in[k], wet_ex[k])
        scale = max(1e-300, np.abs(ri).max(), np.abs(re_).max())
        assert np.abs(Fi[k] - ri).max() <= 1e-13 * scale, (k, Fi[k], ri)
        assert np.abs(Fe[k] - re_).max() <= 1e-13 * scale, (k, Fe[k], re_)
        F = oracle.llf_flux(g, qi[k], qe[k], bath_in[k], 1.0, nrm[k])  # the flux before any fix-up
        if not (wet_in[k] and wet_ex[k]) and abs(F[0]) > 1e-12:
            kinds.add((int(wet_in[k]), int(wet_ex[k]), bool(F[0] > 0)))
    # every branch of the fix-up ran
    assert len(kinds) >= 6, kinds
