"""ctypes binding of the CPU oracle (oracle/oracle.hpp). Test infrastructure only."""
import ctypes as C

import numpy as np

from dgswemv2_b200._lib import forcing_blocks, levee_arrays


class OrcConfig(C.Structure):
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
        ("n_threads", C.c_int32),
        ("bottom_friction", C.c_int32),
        ("friction_cf", C.c_double),
        ("ramp_duration", C.c_double),
    ]


class OrcForcingBlock(C.Structure):
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


class OrcMesh(C.Structure):
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
        ("forcing", C.POINTER(OrcForcingBlock)),
        ("n_levee_pairs", C.c_int32),
        ("levee_nodes", C.POINTER(C.c_int32)),
        ("levee_data", C.POINTER(C.c_double)),
    ]


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


class OracleProblem:
    def __init__(self, lib, cfg, mesh, n_threads=1):
        self.lib = lib
        c = OrcConfig()
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
        for i, v in enumerate(cfg.fn_params[:16]):
            c.fn_params[i] = v
        c.spherical = int(cfg.spherical)
        c.sp_lat0_deg = cfg.sp_lat0_deg
        c.sp_R = cfg.sp_R
        c.n_threads = n_threads
        c.bottom_friction = int(getattr(cfg, "bottom_friction", 0))
        c.friction_cf = float(getattr(cfg, "friction_cf", 0.0))
        c.ramp_duration = float(getattr(cfg, "ramp_duration", 0.0))
        self._keep = [np.ascontiguousarray(mesh.node_xyz, np.float64), np.ascontiguousarray(mesh.elem_nodes, np.int32),
                      None if mesh.elem_ids is None else np.ascontiguousarray(mesh.elem_ids, np.uint32),
                      np.ascontiguousarray(mesh.seg_type, np.int32), np.ascontiguousarray(mesh.seg_offsets, np.int64),
                      np.ascontiguousarray(mesh.seg_nodes, np.int32)]
        m = OrcMesh()
        m.n_nodes = self._keep[0].shape[0]
        m.node_xyz = _ptr(self._keep[0], C.c_double)
        m.n_elems = self._keep[1].shape[0]
        m.elem_nodes = _ptr(self._keep[1], C.c_int32)
        m.elem_ids = _ptr(self._keep[2], C.c_uint32)
        m.n_segments = self._keep[3].shape[0]
        m.seg_type = _ptr(self._keep[3], C.c_int32)
        m.seg_offsets = _ptr(self._keep[4], C.c_int64)
        m.seg_nodes = _ptr(self._keep[5], C.c_int32)
        mann = getattr(mesh, "node_manning_n", None)
        if mann is not None:
            mann = np.ascontiguousarray(mann, np.float64)
            self._keep.append(mann)
            m.node_manning_n = _ptr(mann, C.c_double)
        arr, nf, fkeep = forcing_blocks(mesh, OrcForcingBlock)
        self._keep.append(fkeep)
        m.n_forcing = nf
        m.forcing = arr
        nl, lp, ld = levee_arrays(mesh)
        if nl:
            self._keep += [lp, ld]
            m.n_levee_pairs = nl
            m.levee_nodes = _ptr(lp, C.c_int32)
            m.levee_data = _ptr(ld, C.c_double)
        h = C.c_void_p()
        rc = lib.orc_create(C.byref(c), C.byref(m), C.byref(h))
        if rc != 0:
            raise RuntimeError(lib.orc_last_error().decode())
        self.h = h
        self.ne = lib.orc_n_elements(h)
        self.nd = lib.orc_ndof(h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def get_state(self):
        q = np.empty((self.ne, 3, self.nd), np.float64)
        self.lib.orc_get_state(self.h, _ptr(q, C.c_double))
        return q

    def set_state(self, q):
        q = np.ascontiguousarray(q, np.float64)
        self.lib.orc_set_state(self.h, _ptr(q, C.c_double))

    def get_wet(self):
        w = np.empty(self.ne, np.uint8)
        self.lib.orc_get_wet(self.h, _ptr(w, C.c_uint8))
        return w

    def step(self, n=1):
        rc = self.lib.orc_step(self.h, n)
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())

    def stage(self):
        rc = self.lib.orc_stage(self.h)
        if rc != 0:
            raise RuntimeError(self.lib.orc_last_error().decode())

    def time(self):
        return self.lib.orc_time(self.h)

    def l2_error(self):
        out = C.c_double()
        self.lib.orc_l2_error(self.h, C.byref(out))
        return out.value

    def mass(self):
        out = C.c_double()
        self.lib.orc_mass(self.h, C.byref(out))
        return out.value

    def topology(self):
        nb = np.empty((self.ne, 3), np.int32)
        bt = np.empty((self.ne, 3), np.uint8)
        ni, nbd = C.c_int64(), C.c_int64()
        self.lib.orc_topology(self.h, None, None, C.byref(ni), None, C.byref(nbd), None)
        intf = np.empty((ni.value, 4), np.int32)
        bnd = np.empty((nbd.value, 3), np.int32)
        self.lib.orc_topology(self.h, _ptr(nb, C.c_int32), _ptr(bt, C.c_uint8), C.byref(ni), _ptr(intf, C.c_int32),
                              C.byref(nbd), _ptr(bnd, C.c_int32))
        return nb, bt, intf, bnd

    def limited_flags(self):
        f = np.empty(self.ne, np.uint8)
        self.lib.orc_limited_flags(self.h, _ptr(f, C.c_uint8))
        return f

    def trouble(self):
        I = np.empty(self.ne, np.float64)
        t = np.empty(self.ne, np.uint8)
        self.lib.orc_trouble(self.h, _ptr(I, C.c_double), _ptr(t, C.c_uint8))
        return I, t


class Oracle:
    def __init__(self, path):
        lib = C.CDLL(path)
        lib.orc_create.restype = C.c_int
        lib.orc_last_error.restype = C.c_char_p
        lib.orc_n_elements.restype = C.c_int64
        lib.orc_ndof.restype = C.c_int32
        lib.orc_time.restype = C.c_double
        lib.orc_destroy.argtypes = [C.c_void_p]
        for name in ["orc_get_state", "orc_set_state", "orc_get_wet", "orc_l2_error", "orc_mass", "orc_limited_flags",
                     "orc_trouble", "orc_topology"]:
            getattr(lib, name).restype = C.c_int
        lib.orc_step.argtypes = [C.c_void_p, C.c_int32]
        lib.orc_stage.argtypes = [C.c_void_p]
        lib.orc_time.argtypes = [C.c_void_p]
        lib.orc_n_elements.argtypes = [C.c_void_p]
        lib.orc_ndof.argtypes = [C.c_void_p]
        lib.orc_llf_flux.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_double,
                                     C.POINTER(C.c_double), C.POINTER(C.c_double)]
        D = C.POINTER(C.c_double)
        lib.orc_internal_flux.argtypes = [C.c_double, D, D, C.c_double, C.c_double, C.c_double, C.c_double, D, C.c_int,
                                          C.c_int, D, D]
        self.lib = lib

    def problem(self, cfg, mesh, n_threads=1):
        return OracleProblem(self.lib, cfg, mesh, n_threads)

    # unit-level entry points -----------------------------------------------------------------
    def llf_flux(self, g, q_in, q_ex, bath, sp, n):
        a = np.asarray(q_in, np.float64)
        b = np.asarray(q_ex, np.float64)
        nn = np.asarray(n, np.float64)
        F = np.zeros(3)
        self.lib.orc_llf_flux(g, _ptr(a, C.c_double), _ptr(b, C.c_double), bath, sp, _ptr(nn, C.c_double),
                              _ptr(F, C.c_double))
        return F

    def internal_flux(self, g, q_in, q_ex, bath_in, bath_ex, sp, n, wet_in, wet_ex):
        a = np.ascontiguousarray(q_in, np.float64)
        b = np.ascontiguousarray(q_ex, np.float64)
        nn = np.ascontiguousarray(n, np.float64)
        Fi, Fe = np.zeros(3), np.zeros(3)
        self.lib.orc_internal_flux(g, _ptr(a, C.c_double), _ptr(b, C.c_double), bath_in, bath_ex, sp, sp,
                                   _ptr(nn, C.c_double), int(wet_in), int(wet_ex), _ptr(Fi, C.c_double),
                                   _ptr(Fe, C.c_double))
        return Fi, Fe

    def fn_eval(self, fn_set, params, t, what, x, y):
        """function_sets.h as the oracle compiles it: what 0 true solution, 1 source ([n][3]), 2 bowl bathymetry."""
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        P = np.zeros(16)
        P[:len(params)] = params
        out = np.zeros((len(x), 3)) if what != 2 else np.zeros(len(x))
        self.lib.orc_fn_eval(int(fn_set), _ptr(P, C.c_double), C.c_double(t), int(what), len(x), _ptr(x, C.c_double),
                             _ptr(y, C.c_double), _ptr(out, C.c_double))
        return out

    def dubiner(self, p, pts):
        pts = np.asarray(pts, np.float64)
        z1 = np.ascontiguousarray(pts[:, 0])
        z2 = np.ascontiguousarray(pts[:, 1])
        nd = (p + 1) * (p + 2) // 2
        phi = np.zeros((nd, len(pts)))
        d1 = np.zeros((nd, len(pts)))
        d2 = np.zeros((nd, len(pts)))
        self.lib.orc_dubiner(p, len(pts), _ptr(z1, C.c_double), _ptr(z2, C.c_double), _ptr(phi, C.c_double),
                             _ptr(d1, C.c_double), _ptr(d2, C.c_double))
        return phi, d1, d2

    def triangle_rule(self, degree):
        cap = 256
        w, z1, z2 = np.zeros(cap), np.zeros(cap), np.zeros(cap)
        n = self.lib.orc_triangle_rule(degree, _ptr(w, C.c_double), _ptr(z1, C.c_double), _ptr(z2, C.c_double), cap)
        return w[:n], z1[:n], z2[:n]

    def gl_rule(self, degree):
        cap = 128
        w, z = np.zeros(cap), np.zeros(cap)
        n = self.lib.orc_gl_rule(degree, _ptr(w, C.c_double), _ptr(z, C.c_double), cap)
        return w[:n], z[:n]

    def element_integrals(self, p, verts, terms):
        xy = np.ascontiguousarray(np.asarray(verts, np.float64).reshape(-1))
        c = np.array([t[0] for t in terms], np.float64)
        ex = np.array([t[1] for t in terms], np.int32)
        ey = np.array([t[2] for t in terms], np.int32)
        nd = (p + 1) * (p + 2) // 2
        integ = C.c_double()
        ip, ix, iy = np.zeros(nd), np.zeros(nd), np.zeros(nd)
        self.lib.orc_element_integrals(p, _ptr(xy, C.c_double), len(c), _ptr(c, C.c_double), _ptr(ex, C.c_int),
                                       _ptr(ey, C.c_int), C.byref(integ), _ptr(ip, C.c_double), _ptr(ix, C.c_double),
                                       _ptr(iy, C.c_double))
        return integ.value, ip, ix, iy

    def wet_dry_single(self, verts, bath_vrtx, h_o, q_vrtx, wet_in):
        xy = np.ascontiguousarray(np.asarray(verts, np.float64).reshape(-1))
        b = np.asarray(bath_vrtx, np.float64)
        q = np.ascontiguousarray(np.asarray(q_vrtx, np.float64).reshape(-1))
        out = np.zeros(9)
        wet = C.c_int()
        self.lib.orc_wet_dry_single(_ptr(xy, C.c_double), _ptr(b, C.c_double), C.c_double(h_o), _ptr(q, C.c_double),
                                    int(wet_in), _ptr(out, C.c_double), C.byref(wet))
        return out.reshape(3, 3), bool(wet.value)

    def rk_table(self, ns, order):
        a, b, d = np.zeros(ns * ns), np.zeros(ns * ns), np.zeros(ns)
        rc = self.lib.orc_rk_table(ns, order, _ptr(a, C.c_double), _ptr(b, C.c_double), _ptr(d, C.c_double))
        if rc != 0:
            raise ValueError("unsupported RK pair")
        return a.reshape(ns, ns), b.reshape(ns, ns), d
