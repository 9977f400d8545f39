"""ctypes binding of libdgsw_rkdg.so (include/dgsw_rkdg.h).

The shared library is built in-tree (dgswemv2_b200/libdgsw_rkdg.so, see __graft_entry__.build()).
Loading fails loudly when it is missing: there is no CPU fallback for the RKDG step.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdgsw_rkdg.so")

DGSW_FP64, DGSW_FP32 = 0, 1
DGSW_TILE_AUTOTUNE = -1
DGSW_L2_STATIC_MAX_ELEMS = 1048576
DGSW_MLP_NPARAM = 5441
DGSW_MLP_NFEATURES = 18

STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "mesh error",
    3: "CUDA error",
    4: "NaN in solution",
    5: "unsupported",
    6: "no CUDA device",
    7: "I/O error",
}


class DgswError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (%d): %s" % (STATUS.get(status, "?"), status, message))
        self.status = status


class Config(C.Structure):
    _fields_ = [
        ("p", C.c_int32),
        ("rk_nstages", C.c_int32),
        ("rk_order", C.c_int32),
        ("dt", C.c_double),
        ("g", C.c_double),
        ("wetting_drying", C.c_int32),
        ("h_o", C.c_double),
        ("slope_limiting", C.c_int32),
        ("sl_M", C.c_double),
        ("sl_nu", C.c_double),
        ("function_source", C.c_int32),
        ("ic_type", C.c_int32),
        ("ic_const", C.c_double * 3),
        ("function_set", C.c_int32),
        ("fn_params", C.c_double * 16),
        ("spherical", C.c_int32),
        ("sp_lat0_deg", C.c_double),
        ("sp_R", C.c_double),
        ("bottom_friction", C.c_int32),
        ("friction_cf", C.c_double),
        ("ramp_duration", C.c_double),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("tile", C.c_int32),
        ("renumber", C.c_int32),
        ("use_graphs", C.c_int32),
        ("fp64_limiter", C.c_int32),
        ("occupancy", C.c_int32),
        ("tile_order", C.c_int32),
        ("fp64_stages", C.c_int32),
        ("reserved", C.c_int32 * 4),
    ]


class ForcingBlock(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("n_nodes", C.c_int32),
        ("n_constituents", C.c_int32),
        ("nodes", C.POINTER(C.c_int32)),
        ("frequency", C.POINTER(C.c_double)),
        ("forcing_fact", C.POINTER(C.c_double)),
        ("equilib_arg", C.POINTER(C.c_double)),
        ("amplitude", C.POINTER(C.c_double)),
        ("phase", C.POINTER(C.c_double)),
    ]


class Mesh(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("node_xyz", C.POINTER(C.c_double)),
        ("n_elems", C.c_int64),
        ("elem_nodes", C.POINTER(C.c_int32)),
        ("elem_ids", C.POINTER(C.c_uint32)),
        ("n_segments", C.c_int32),
        ("seg_type", C.POINTER(C.c_int32)),
        ("seg_offsets", C.POINTER(C.c_int64)),
        ("seg_nodes", C.POINTER(C.c_int32)),
        ("node_manning_n", C.POINTER(C.c_double)),
        ("n_forcing", C.c_int32),
        ("forcing", C.POINTER(ForcingBlock)),
        ("n_levee_pairs", C.c_int32),
        ("levee_nodes", C.POINTER(C.c_int32)),
        ("levee_data", C.POINTER(C.c_double)),
    ]


def forcing_blocks(mesh, block_type=None):
    """ctypes array of the mesh's forcing blocks (block_type: ForcingBlock struct class to fill) plus the
    numpy arrays it points into (keep them alive as long as the array is used)."""
    block_type = block_type or ForcingBlock
    blocks = list(getattr(mesh, "forcing", None) or [])
    keep = []
    arr = (block_type * max(len(blocks), 1))()
    for k, b in enumerate(blocks):
        nodes = np.ascontiguousarray(b.nodes, np.int32)
        fr = np.ascontiguousarray(b.frequency, np.float64)
        ff = np.ascontiguousarray(b.forcing_fact, np.float64)
        eq = np.ascontiguousarray(b.equilib_arg, np.float64)
        am = np.ascontiguousarray(b.amplitude, np.float64).reshape(len(fr), len(nodes))
        ph = np.ascontiguousarray(b.phase, np.float64).reshape(len(fr), len(nodes))
        keep += [nodes, fr, ff, eq, am, ph]
        arr[k].type = int(b.type)
        arr[k].n_nodes = len(nodes)
        arr[k].n_constituents = len(fr)
        arr[k].nodes = ptr(nodes, C.c_int32)
        arr[k].frequency = ptr(fr, C.c_double)
        arr[k].forcing_fact = ptr(ff, C.c_double)
        arr[k].equilib_arg = ptr(eq, C.c_double)
        arr[k].amplitude = ptr(am, C.c_double)
        arr[k].phase = ptr(ph, C.c_double)
    keep.append(arr)
    return (arr if blocks else None), len(blocks), keep


def levee_arrays(mesh):
    """(n, front/back node pairs, data) of the mesh's .bcis levee lines, as contiguous arrays or Nones."""
    pairs = getattr(mesh, "levee_pairs", None)
    if pairs is None or len(pairs) == 0:
        return 0, None, None
    pairs = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
    data = np.ascontiguousarray(mesh.levee_data, np.float64).reshape(-1, 3)
    if data.shape[0] != pairs.shape[0]:
        raise ValueError("levee_data needs one (H, C_sub, C_super) row per levee pair")
    return pairs.shape[0], pairs, data


class Info(C.Structure):
    _fields_ = [
        ("n_elems", C.c_int64),
        ("n_nodes", C.c_int64),
        ("n_interfaces", C.c_int64),
        ("n_boundaries", C.c_int64),
        ("n_tiles", C.c_int64),
        ("n_tile_edges", C.c_int64),
        ("p", C.c_int32),
        ("ndof", C.c_int32),
        ("ngp_volume", C.c_int32),
        ("ngp_edge", C.c_int32),
        ("nstages", C.c_int32),
        ("precision", C.c_int32),
        ("tile", C.c_int32),
        ("device_bytes", C.c_int64),
        ("state_bytes", C.c_int64),
        ("occupancy", C.c_int32),
        ("tile_order", C.c_int32),
        ("stage_increments", C.c_int32),
        ("smem_capped", C.c_int32),
    ]


# every symbol include/dgsw_rkdg.h declares, with its ctypes signature
SIGNATURES = {
    "dgsw_abi_version": (C.c_int32, []),
    "dgsw_last_error": (C.c_char_p, []),
    "dgsw_status_string": (C.c_char_p, [C.c_int32]),
    "dgsw_config_default": (None, [C.POINTER(Config)]),
    "dgsw_rkdg_create": (C.c_int32, [C.POINTER(Config), C.POINTER(Mesh), C.POINTER(C.c_void_p)]),
    "dgsw_rkdg_destroy": (C.c_int32, [C.c_void_p]),
    "dgsw_ensemble_create": (C.c_int32, [C.POINTER(Config), C.c_int32, C.POINTER(Mesh), C.POINTER(C.c_double),
                                         C.POINTER(C.c_void_p)]),
    "dgsw_ensemble_member_range": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "dgsw_rkdg_tuning": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "dgsw_rkdg_info": (C.c_int32, [C.c_void_p, C.POINTER(Info)]),
    "dgsw_rkdg_init_state": (C.c_int32, [C.c_void_p]),
    "dgsw_rkdg_set_state": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "dgsw_rkdg_get_state": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "dgsw_rkdg_set_wet": (C.c_int32, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "dgsw_rkdg_get_wet": (C.c_int32, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "dgsw_rkdg_get_bathymetry": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "dgsw_rkdg_postprocess": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]),
    "dgsw_rkdg_set_state_device": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "dgsw_rkdg_get_state_device": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "dgsw_rkdg_step": (C.c_int32, [C.c_void_p, C.c_int32]),
    "dgsw_rkdg_stage": (C.c_int32, [C.c_void_p]),
    "dgsw_rkdg_get_time": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "dgsw_rkdg_l2_error": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "dgsw_rkdg_mass": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double)]),
    "dgsw_l2_error_static": (C.c_int32, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                         C.POINTER(C.c_double), C.c_double, C.c_void_p, C.POINTER(C.c_double)]),
    "dgsw_rkdg_topology": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_uint8), C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "dgsw_mesh_topology": (C.c_int32, [C.POINTER(Mesh), C.POINTER(C.c_int32), C.POINTER(C.c_uint8),
                                       C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int32)]),
    "dgsw_rkdg_get_limited": (C.c_int32, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "dgsw_rkdg_set_trouble": (C.c_int32, [C.c_void_p, C.c_int32]),
    "dgsw_rkdg_get_trouble": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint8)]),
    "dgsw_rkdg_indicator_features": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dgsw_rkdg_stage_record": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "dgsw_rkdg_set_indicator": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float), C.c_double, C.c_int32]),
    "dgsw_rkdg_indicator_stats": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64), C.c_int32]),
    "dgsw_rkdg_set_indicator_features": (C.c_int32, [C.c_void_p, C.c_int32]),
    "dgsw_mlp_forward": (C.c_int32, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "dgsw_mlp_grad_work_floats": (C.c_int64, [C.c_int64]),
    "dgsw_mlp_grad": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p,
                                  C.c_int64, C.c_void_p, C.c_void_p]),
    "dgsw_mlp_adam": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_float, C.c_float,
                                  C.c_float, C.c_float, C.c_void_p]),
    "dgsw_check_llf_flux": (C.c_int32, [C.c_int32, C.c_int64, C.c_double] + [C.POINTER(C.c_double)] * 6),
    "dgsw_check_internal_flux": (C.c_int32, [C.c_int32, C.c_int64, C.c_double] + [C.POINTER(C.c_double)] * 6 +
                                 [C.POINTER(C.c_uint8)] * 2 + [C.POINTER(C.c_double)] * 2),
    "dgsw_check_wetting_drying": (C.c_int32, [C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                              C.POINTER(C.c_uint8), C.POINTER(C.c_double), C.POINTER(C.c_uint8),
                                              C.POINTER(C.c_uint8)]),
    "dgsw_rkdg_set_stream": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "dgsw_rkdg_synchronize": (C.c_int32, [C.c_void_p]),
    "dgsw_rkdg_last_step_timing": (C.c_int32, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "dgsw_rkdg_step_timed": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
}

_lib = None


def load():
    """Load the in-tree library (once). Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libdgsw_rkdg.so is not built (run __graft_entry__.build() or make -C dgswemv2_b200/csrc)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status):
    if status != 0:
        raise DgswError(status, load().dgsw_last_error().decode())


def ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None
