"""B200-native RKDG shallow-water step with dgswemv2's problem/stepper interface.

Python host side of the drop-in. `Problem` wraps one library handle and exposes the reference's
SWE::RKDG::Problem / Serial::Simulation operations (preprocessor_serial, step_serial, stage_serial,
compute_residual_L2); all arithmetic runs in libdgsw_rkdg.so on the GPU.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import DGSW_FP32, DGSW_FP64, DgswError  # noqa: F401
from .types import MeshArrays, ProblemConfig  # noqa: F401

__all__ = ["Problem", "ProblemConfig", "MeshArrays", "DgswError", "mesh_topology", "ensemble"]


def _make_config(cfg, device=0, tile=0, renumber=True, use_graphs=True, fp64_limiter=False, occupancy=0,
                 tile_order=0, fp64_stages=False):
    lib = _lib.load()
    c = _lib.Config()
    lib.dgsw_config_default(C.byref(c))
    c.p = cfg.p
    c.rk_nstages = cfg.rk_nstages
    c.rk_order = cfg.rk_order
    c.dt = cfg.dt
    c.g = cfg.g
    c.wetting_drying = int(cfg.wetting_drying)
    c.h_o = cfg.h_o
    c.slope_limiting = int(cfg.slope_limiting)
    c.sl_M = cfg.sl_M
    c.sl_nu = cfg.sl_nu
    c.function_source = int(cfg.function_source)
    c.ic_type = cfg.ic_type
    for i in range(3):
        c.ic_const[i] = cfg.ic_const[i]
    c.function_set = cfg.function_set
    for i, v in enumerate(list(cfg.fn_params)[:16]):
        c.fn_params[i] = v
    c.spherical = int(cfg.spherical)
    c.sp_lat0_deg = cfg.sp_lat0_deg
    c.sp_R = cfg.sp_R
    c.bottom_friction = int(getattr(cfg, "bottom_friction", 0))
    c.friction_cf = float(getattr(cfg, "friction_cf", 0.0))
    c.ramp_duration = float(getattr(cfg, "ramp_duration", 0.0))
    c.precision = DGSW_FP32 if cfg.precision == "fp32" else DGSW_FP64
    c.device = device
    c.tile = tile
    c.renumber = int(renumber)
    c.use_graphs = int(use_graphs)
    c.fp64_limiter = int(fp64_limiter)
    c.occupancy = int(occupancy)
    c.tile_order = int(tile_order)
    c.fp64_stages = int(fp64_stages)
    return c


def _mesh_struct(mesh):
    keep = [
        np.ascontiguousarray(mesh.node_xyz, np.float64),
        np.ascontiguousarray(mesh.elem_nodes, np.int32),
        None if mesh.elem_ids is None else np.ascontiguousarray(mesh.elem_ids, np.uint32),
        np.ascontiguousarray(mesh.seg_type, np.int32),
        np.ascontiguousarray(mesh.seg_offsets, np.int64),
        np.ascontiguousarray(mesh.seg_nodes, np.int32),
    ]
    m = _lib.Mesh()
    m.n_nodes = keep[0].shape[0]
    m.node_xyz = _lib.ptr(keep[0], C.c_double)
    m.n_elems = keep[1].shape[0]
    m.elem_nodes = _lib.ptr(keep[1], C.c_int32)
    m.elem_ids = _lib.ptr(keep[2], C.c_uint32)
    m.n_segments = keep[3].shape[0]
    m.seg_type = _lib.ptr(keep[3], C.c_int32)
    m.seg_offsets = _lib.ptr(keep[4], C.c_int64)
    m.seg_nodes = _lib.ptr(keep[5], C.c_int32)
    mann = getattr(mesh, "node_manning_n", None)
    if mann is not None:
        mann = np.ascontiguousarray(mann, np.float64)
        if mann.shape != (mesh.n_nodes,):
            raise ValueError("node_manning_n must hold one value per node")
        keep.append(mann)
        m.node_manning_n = _lib.ptr(mann, C.c_double)
    arr, nf, fkeep = _lib.forcing_blocks(mesh)
    keep.append(fkeep)
    m.n_forcing = nf
    m.forcing = arr
    nl, lp, ld = _lib.levee_arrays(mesh)
    if nl:
        keep += [lp, ld]
        m.n_levee_pairs = nl
        m.levee_nodes = _lib.ptr(lp, C.c_int32)
        m.levee_data = _lib.ptr(ld, C.c_double)
    return m, keep


def mesh_topology(mesh):
    """Host-only topology (MeshMetaData + interface/boundary creation), in ascending element-ID order:
    neighbours, boundary type per face, interfaces (in, ex, face_in, face_ex), boundaries (elem, face, type)."""
    lib = _lib.load()
    m, keep = _mesh_struct(mesh)
    ni, nb = C.c_int64(), C.c_int64()
    _lib.check(lib.dgsw_mesh_topology(C.byref(m), None, None, C.byref(ni), None, C.byref(nb), None))
    ne = mesh.n_elems
    nbr = np.empty((ne, 3), np.int32)
    bt = np.empty((ne, 3), np.uint8)
    intf = np.empty((ni.value, 4), np.int32)
    bnd = np.empty((nb.value, 3), np.int32)
    _lib.check(lib.dgsw_mesh_topology(C.byref(m), _lib.ptr(nbr, C.c_int32), _lib.ptr(bt, C.c_uint8), C.byref(ni),
                                      _lib.ptr(intf, C.c_int32), C.byref(nb), _lib.ptr(bnd, C.c_int32)))
    return nbr, bt, intf, bnd


def ensemble(cfg, meshes, member_params=None, device=0, tile=_lib.DGSW_TILE_AUTOTUNE, renumber=True,
             use_graphs=True, init=True, occupancy=0, tile_order=0, fp64_stages=False):
    """Ensemble batching (dgsw_ensemble_create): the members share `cfg` except their function-set
    parameters (member_params: one 16-value list per member, or None for cfg.fn_params). Returns a
    Problem whose state holds the members one after another (Problem.member_range)."""
    lib = _lib.load()
    P = Problem.__new__(Problem)
    P.cfg = cfg
    P._c = _make_config(cfg, device, tile, renumber, use_graphs, occupancy=occupancy, tile_order=tile_order,
                        fp64_stages=fp64_stages)
    arr = (_lib.Mesh * len(meshes))()
    P._keep = []
    for k, m in enumerate(meshes):
        arr[k], keep = _mesh_struct(m)
        P._keep.append(keep)
    prm = None
    if member_params is not None:
        prm = np.zeros((len(meshes), 16), np.float64)
        for k, v in enumerate(member_params):
            prm[k, :len(v)] = v
        P._keep.append(prm)
    h = C.c_void_p()
    _lib.check(lib.dgsw_ensemble_create(C.byref(P._c), len(meshes), arr, _lib.ptr(prm, C.c_double), C.byref(h)))
    P._h = h
    P.info = _lib.Info()
    _lib.check(lib.dgsw_rkdg_info(h, C.byref(P.info)))
    P.ne = P.info.n_elems
    P.nd = P.info.ndof
    if init:
        P.preprocessor_serial()
    return P


class Problem:
    """One RKDG problem on one GPU (SWE::RKDG::Problem + Serial::Simulation, rkdg_swe_problem.hpp:34-194,
    simulation.hpp:14-93)."""

    def __init__(self, cfg, mesh, device=0, tile=0, renumber=True, use_graphs=True, init=True, fp64_limiter=False,
                 occupancy=0, tile_order=0, fp64_stages=False):
        lib = _lib.load()
        self.cfg = cfg
        self._c = _make_config(cfg, device, tile, renumber, use_graphs, fp64_limiter, occupancy, tile_order,
                               fp64_stages)
        m, self._keep = _mesh_struct(mesh)
        h = C.c_void_p()
        _lib.check(lib.dgsw_rkdg_create(C.byref(self._c), C.byref(m), C.byref(h)))
        self._h = h
        self.info = _lib.Info()
        _lib.check(lib.dgsw_rkdg_info(h, C.byref(self.info)))
        self.ne = self.info.n_elems
        self.nd = self.info.ndof
        if init:
            self.preprocessor_serial()

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().dgsw_rkdg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # reference interface ---------------------------------------------------------------------
    def preprocessor_serial(self):
        """Problem::preprocessor_serial: initial projections, wet/dry and limiter initialisation."""
        _lib.check(_lib.load().dgsw_rkdg_init_state(self._h))

    def step_serial(self, nsteps=1):
        """Problem::step_serial, nsteps times."""
        _lib.check(_lib.load().dgsw_rkdg_step(self._h, int(nsteps)))

    def stage_serial(self):
        """Problem::stage_serial: one RK stage."""
        _lib.check(_lib.load().dgsw_rkdg_stage(self._h))

    def compute_residual_L2(self):
        """Simulation::ComputeL2Residual: sqrt of the summed per-element squared L2 error."""
        out = C.c_double()
        _lib.check(_lib.load().dgsw_rkdg_l2_error(self._h, C.byref(out)))
        return out.value

    # state access ----------------------------------------------------------------------------
    def get_state(self, out=None):
        """Modal state [ne][3][nd] in ascending element-ID order; `out`: a C-contiguous float64 array of that
        shape (for example pinned host memory) to write into instead of a new array."""
        if out is None:
            out = np.empty((self.ne, 3, self.nd), np.float64)
        elif out.dtype != np.float64 or out.shape != (self.ne, 3, self.nd) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (ne, 3, nd)")
        _lib.check(_lib.load().dgsw_rkdg_get_state(self._h, _lib.ptr(out, C.c_double)))
        return out

    def set_state(self, q):
        q = np.ascontiguousarray(q, np.float64)
        assert q.shape == (self.ne, 3, self.nd)
        _lib.check(_lib.load().dgsw_rkdg_set_state(self._h, _lib.ptr(q, C.c_double)))

    def postprocess(self):
        """Writer values (dgsw_rkdg_postprocess): point data [ne][3][ze, qx, qy, bath] at the vertices,
        cell data [ne][ze, qx, qy, bath] at the centroids, wet and went-completely-dry flags, in ascending
        element-ID order."""
        lib = _lib.load()
        pt = np.empty((self.ne, 3, 4), np.float64)
        cell = np.empty((self.ne, 4), np.float64)
        wet = np.empty(self.ne, np.uint8)
        wd = np.empty(self.ne, np.uint8)
        _lib.check(lib.dgsw_rkdg_postprocess(self._h, _lib.ptr(pt, C.c_double), _lib.ptr(cell, C.c_double),
                                             _lib.ptr(wet, C.c_uint8), _lib.ptr(wd, C.c_uint8)))
        return pt, cell, wet, wd

    def get_wet(self):
        w = np.empty(self.ne, np.uint8)
        _lib.check(_lib.load().dgsw_rkdg_get_wet(self._h, _lib.ptr(w, C.c_uint8)))
        return w

    def set_wet(self, w):
        w = np.ascontiguousarray(w, np.uint8)
        _lib.check(_lib.load().dgsw_rkdg_set_wet(self._h, _lib.ptr(w, C.c_uint8)))

    def get_limited(self):
        w = np.empty(self.ne, np.uint8)
        _lib.check(_lib.load().dgsw_rkdg_get_limited(self._h, _lib.ptr(w, C.c_uint8)))
        return w

    # learned troubled-cell indicator ---------------------------------------------------------
    def indicator_features(self, d_features, d_ok=0):
        """Features [ne][18] (FP32) and limiter-looks flags [ne] of the current state into device buffers."""
        _lib.check(_lib.load().dgsw_rkdg_indicator_features(self._h, C.c_void_p(d_features), C.c_void_p(d_ok or None)))

    def stage_record(self, d_features, d_labels):
        """One stage with the plain limiter, recording pre-limiter features and the limiter's decisions."""
        _lib.check(_lib.load().dgsw_rkdg_stage_record(self._h, C.c_void_p(d_features), C.c_void_p(d_labels)))

    def set_indicator(self, params, confidence=0.9, mode=1):
        """mode 0 plain limiter, 1 MLP-gated limiter, 2 plain limiter with the gate's misses counted."""
        prm = np.ascontiguousarray(params, np.float32)
        assert prm.size == _lib.DGSW_MLP_NPARAM
        _lib.check(_lib.load().dgsw_rkdg_set_indicator(self._h, _lib.ptr(prm, C.c_float), float(confidence), int(mode)))

    def set_indicator_features(self, feature_set):
        """0: the characteristic feature set (default); 1: raw modal coefficients and neighbour means."""
        _lib.check(_lib.load().dgsw_rkdg_set_indicator_features(self._h, int(feature_set)))

    def indicator_stats(self, reset=False):
        """(considered, sent to the limiter, limited, missed) cell counts since the last reset."""
        c = (C.c_int64 * 4)()
        _lib.check(_lib.load().dgsw_rkdg_indicator_stats(self._h, c, int(reset)))
        return tuple(int(v) for v in c)

    def set_trouble(self, enable=True):
        """Evaluate the reference's (unused) KXRCF trouble indicator in every limiter pass."""
        _lib.check(_lib.load().dgsw_rkdg_set_trouble(self._h, int(enable)))

    def get_trouble(self):
        """(I [ne], troubled flags [ne]) of the last limiter pass, ascending element ID."""
        I = np.empty(self.ne, np.float64)
        t = np.empty(self.ne, np.uint8)
        _lib.check(_lib.load().dgsw_rkdg_get_trouble(self._h, _lib.ptr(I, C.c_double), _lib.ptr(t, C.c_uint8)))
        return I, t

    def set_state_device(self, dptr):
        _lib.check(_lib.load().dgsw_rkdg_set_state_device(self._h, C.c_void_p(dptr)))

    def get_state_device(self, dptr):
        _lib.check(_lib.load().dgsw_rkdg_get_state_device(self._h, C.c_void_p(dptr)))

    def step_timed(self, nsteps):
        """nsteps steps with every stage-kernel launch timed by its own CUDA events (no step graphs):
        (summed stage-kernel milliseconds, number of stage-kernel launches)."""
        ms, n = C.c_double(), C.c_int64()
        _lib.check(_lib.load().dgsw_rkdg_step_timed(self._h, int(nsteps), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def time(self):
        t = C.c_double()
        st = C.c_int64()
        sg = C.c_int32()
        _lib.check(_lib.load().dgsw_rkdg_get_time(self._h, C.byref(t), C.byref(st), C.byref(sg)))
        return t.value, st.value, sg.value

    def mass(self):
        out = C.c_double()
        _lib.check(_lib.load().dgsw_rkdg_mass(self._h, C.byref(out)))
        return out.value

    def topology(self):
        lib = _lib.load()
        ni, nb = C.c_int64(), C.c_int64()
        _lib.check(lib.dgsw_rkdg_topology(self._h, None, None, C.byref(ni), None, C.byref(nb), None))
        nbr = np.empty((self.ne, 3), np.int32)
        bt = np.empty((self.ne, 3), np.uint8)
        intf = np.empty((ni.value, 4), np.int32)
        bnd = np.empty((nb.value, 3), np.int32)
        _lib.check(lib.dgsw_rkdg_topology(self._h, _lib.ptr(nbr, C.c_int32), _lib.ptr(bt, C.c_uint8), C.byref(ni),
                                          _lib.ptr(intf, C.c_int32), C.byref(nb), _lib.ptr(bnd, C.c_int32)))
        return nbr, bt, intf, bnd

    def member_range(self, member):
        """(first element, element count) of an ensemble member in the state order."""
        f, n = C.c_int64(), C.c_int64()
        _lib.check(_lib.load().dgsw_ensemble_member_range(self._h, int(member), C.byref(f), C.byref(n)))
        return f.value, n.value

    def tuning(self):
        """The autotuner's record: [(tile, occupancy, tile_order, device ms per step), ...] (empty if not tuned)."""
        cap = 8
        t, o, r = (C.c_int32 * cap)(), (C.c_int32 * cap)(), (C.c_int32 * cap)()
        ms = (C.c_double * cap)()
        n = C.c_int32()
        _lib.check(_lib.load().dgsw_rkdg_tuning(self._h, t, o, r, ms, C.byref(n)))
        return [(t[i], o[i], r[i], ms[i]) for i in range(n.value)]

    def synchronize(self):
        _lib.check(_lib.load().dgsw_rkdg_synchronize(self._h))

    def last_step_timing(self):
        ms = C.c_double()
        n = C.c_int64()
        _lib.check(_lib.load().dgsw_rkdg_last_step_timing(self._h, C.byref(ms), C.byref(n)))
        return ms.value, n.value
