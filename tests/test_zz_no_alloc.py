"""dgsw_l2_error_static, the allocation-free L2 error (static device scratch, no handle), against the
handle's dgsw_rkdg_l2_error on the same FP64 state.

Tolerance: relative 1e-12, the FP64 tolerance of the parity tests; the two differ only in summation
order. This file is collected last so that the static entry point also runs after every other test
has used the device in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from dgswemv2_b200 import Problem, _lib, configs, meshgen
from dgswemv2_b200.types import FUNCTION

TOL = 1e-12
MAX_ELEMS = _lib.DGSW_L2_STATIC_MAX_ELEMS


def static_l2(p, ne, d_q, d_elem_nodes, d_node_xyz, fn_set, fn_params, t, stream=None):
    lib = _lib.load()
    out = C.c_double()
    prm = (C.c_double * 16)(*list(fn_params)[:16])
    _lib.check(lib.dgsw_l2_error_static(p, ne, C.c_void_p(d_q), C.c_void_p(d_elem_nodes), C.c_void_p(d_node_xyz),
                                        fn_set, prm, t, C.c_void_p(stream) if stream else None, C.byref(out)))
    return out.value


def test_rejects_bad_sizes_before_any_device_work():
    """Sizes beyond the static scratch, empty inputs and p outside 1..2 fail with a clear message; the
    checks come before any CUDA call (the dummy pointers are never read)."""
    lib = _lib.load()
    out = C.c_double()
    dummy = C.c_void_p(256)
    for p, ne, what in ((2, MAX_ELEMS + 1, b"static scratch"), (1, 0, b"outside 1.."), (3, 10, b"p must be")):
        rc = lib.dgsw_l2_error_static(p, ne, dummy, dummy, dummy, 2, None, 0.0, None, C.byref(out))
        assert rc == 1, (p, ne, rc)
        assert what in lib.dgsw_last_error(), lib.dgsw_last_error()
    rc = lib.dgsw_l2_error_static(2, 10, None, dummy, dummy, 2, None, 0.0, None, C.byref(out))
    assert rc == 1


def _device_mesh(mesh):
    import torch

    order = np.arange(mesh.n_elems) if mesh.elem_ids is None else np.argsort(mesh.elem_ids, kind="stable")
    en = torch.from_numpy(np.ascontiguousarray(mesh.elem_nodes[order], np.int32)).cuda()
    xyz = torch.from_numpy(np.ascontiguousarray(mesh.node_xyz, np.float64)).cuda()
    return en, xyz


def _compare_two_calls(mesh, cfg, steps_between):
    import torch

    P = Problem(cfg, mesh)
    dq = torch.empty((P.ne, 3, P.nd), dtype=torch.float64, device="cuda")
    en, xyz = _device_mesh(mesh)
    torch.cuda.synchronize()
    got = []
    for call in range(2):
        if call:
            P.step_serial(steps_between)
        P.get_state_device(dq.data_ptr())
        P.synchronize()
        t = P.time()[0]
        ref = P.compute_residual_L2()
        val = static_l2(cfg.p, P.ne, dq.data_ptr(), en.data_ptr(), xyz.data_ptr(), cfg.function_set, cfg.fn_params, t)
        assert np.isfinite(val) and ref > 0
        assert abs(val - ref) <= TOL * ref, (call, val, ref)
        got.append(val)
    P.close()
    return got


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 2])
def test_static_l2_matches_handle_on_two_calls_in_a_row(p):
    mesh, cfg = configs.manufactured(24, p=p, rk=(3, 3) if p == 2 else (2, 2), dt=1.0, jitter=0.2)
    v0, v1 = _compare_two_calls(mesh, cfg, steps_between=20)
    assert v0 != v1  # the second call saw the advanced state, not the first call's scratch


@pytest.mark.gpu
def test_static_l2_at_the_size_limit():
    """Exactly DGSW_L2_STATIC_MAX_ELEMS elements (1024 x 512 quads), p=2."""
    _, cfg = configs.manufactured(4, p=2, rk=(3, 3), dt=0.5)
    mesh = meshgen.quad_mesh(1024, 512, corners=((0, 0), (configs.L_MMS, 0), (configs.L_MMS, configs.L_MMS),
                                                 (0, configs.L_MMS)),
                             bc=(FUNCTION,) * 4, jitter=0.1, seed=3, bathymetry=meshgen.bath_flat(2.0))
    assert mesh.n_elems == MAX_ELEMS
    _compare_two_calls(mesh, cfg, steps_between=2)
