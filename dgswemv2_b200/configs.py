"""The synthetic workloads: meshes, problem configurations and function-set parameters.

1. manufactured p=1: [0,40000]^2 m, 20x20 quads -> 800 triangles, b = 2 m, g = 9.81,
   ze = 0.1 sin(2 pi x/L) cos(2 pi y/L) cos(w t), function BC on all sides, SSP-RK2, dt = 1 s, 1000 steps
2. manufactured p=2 at scale: 512x512 quads -> 524,288 triangles, interior nodes jittered by +-20% of the
   cell size (seed 2), Dunavant degree 4 / 3-point Gauss-Legendre, SSP-RK3, 200 steps of dt = 0.5 s
3. Thacker bowl with wetting/drying + slope limiter: +-4000 m, 256x256 quads -> 131,072 triangles,
   h0 = 10 m, a = 3000 m, amplitude 2 m, p=1, SSP-RK2, h_o = 0.01 m, two periods
4. learned troubled-cell indicator on bowl meshes with random Gaussian humps
5. ensemble of p=1 members with random smooth bathymetry and wet/dry
6. tidal channel: two-constituent tide on the open (x = 0) end, a steady + periodic river flow on the
   other, land sides, sloping bathymetry, Chezy or Manning bottom friction, forcing ramp
7. levee channel: the tidal channel cut across by an internal barrier that the tide overtops (optionally
   onto dry land, with wetting/drying and the slope limiter)
"""
import math

import numpy as np

from . import meshgen
from .types import (FLOW, FN_GAUSSIAN_HUMPS, FN_MANUFACTURED_SINE, FN_THACKER_BOWL, FRICTION_CHEZY, FRICTION_MANNING,
                    FRICTION_NONE, FUNCTION, LAND, TIDE, ForcingBlock, ProblemConfig)

L_MMS = 40000.0


def sine_params(L=L_MMS, A=0.1, H=2.0, g=9.81, w=0.0):
    p = [0.0] * 16
    p[0], p[1], p[2], p[3], p[4] = L, A, H, w, g
    return p


def manufactured(nq=20, p=1, rk=(2, 2), dt=1.0, jitter=0.0, seed=2, H=2.0, g=9.81, precision="fp64"):
    mesh = meshgen.quad_mesh(nq, nq, corners=((0, 0), (L_MMS, 0), (L_MMS, L_MMS), (0, L_MMS)),
                             bc=(FUNCTION,) * 4, jitter=jitter, seed=seed, bathymetry=meshgen.bath_flat(H),
                             name="manufactured_%d" % nq)
    cfg = ProblemConfig(p=p, rk_nstages=rk[0], rk_order=rk[1], dt=dt, g=g, function_source=True, ic_type=1,
                        function_set=FN_MANUFACTURED_SINE, fn_params=sine_params(H=H, g=g), precision=precision)
    return mesh, cfg


def config1(precision="fp64"):
    return manufactured(20, p=1, rk=(2, 2), dt=1.0, precision=precision)


def config2(nq=512, precision="fp64", dt=0.5):
    """dt is not part of the configuration; 0.5 s keeps the Courant number near 0.1 on the thinnest
    jittered triangles of the 512x512 mesh (dt = 1 s is unstable there, on the CPU oracle too)."""
    return manufactured(nq, p=2, rk=(3, 3), dt=dt, jitter=0.2, seed=2, precision=precision)


def thacker_params(h0=10.0, a=3000.0, eta0=2.0, g=9.81):
    p = [0.0] * 16
    p[0], p[1], p[2], p[3] = h0, a, eta0, g
    return p


def thacker_period(h0=10.0, a=3000.0, g=9.81):
    return 2 * math.pi / (math.sqrt(8 * g * h0) / a)


def config3(nq=256, dt=0.25, limiter=True, precision="fp64", extent=4000.0):
    mesh = meshgen.quad_mesh(nq, nq, corners=((-extent, -extent), (extent, -extent), (extent, extent), (-extent, extent)),
                             bc=(LAND,) * 4, bathymetry=meshgen.bath_thacker(10.0, 3000.0), name="bowl_%d" % nq)
    cfg = ProblemConfig(p=1, rk_nstages=2, rk_order=2, dt=dt, g=9.81, wetting_drying=True, h_o=0.01,
                        slope_limiting=limiter, sl_M=1.0e-8, sl_nu=1.5, ic_type=1, function_set=FN_THACKER_BOWL,
                        fn_params=thacker_params(), precision=precision)
    return mesh, cfg


def humps_params(humps, ze0=0.0):
    p = [0.0] * 16
    p[0] = ze0
    for i, (amp, xc, yc, w) in enumerate(humps[:3]):
        p[1 + 4 * i], p[2 + 4 * i], p[3 + 4 * i], p[4 + 4 * i] = amp, xc, yc, w
    return p


def random_humps(rng, extent=2500.0, n=None):
    n = n if n is not None else int(rng.integers(1, 4))
    out = []
    for _ in range(n):
        r = rng.uniform(0, extent * 0.7)
        th = rng.uniform(0, 2 * math.pi)
        out.append((rng.uniform(0.5, 3.0), r * math.cos(th), r * math.sin(th), rng.uniform(200.0, 1500.0)))
    return out


def bowl_humps(nq=256, seed=0, dt=0.25, precision="fp64", extent=4000.0, limiter=True):
    """Config-3 bowl bathymetry with random Gaussian humps on still water (config 4 training data)."""
    rng = np.random.default_rng(seed)
    mesh = meshgen.quad_mesh(nq, nq, corners=((-extent, -extent), (extent, -extent), (extent, extent), (-extent, extent)),
                             bc=(LAND,) * 4, bathymetry=meshgen.bath_thacker(10.0, 3000.0), name="bowl_humps_%d" % nq)
    cfg = ProblemConfig(p=1, rk_nstages=2, rk_order=2, dt=dt, g=9.81, wetting_drying=True, h_o=0.01,
                        slope_limiting=limiter, sl_M=1.0e-8, sl_nu=1.5, ic_type=1, function_set=FN_GAUSSIAN_HUMPS,
                        fn_params=humps_params(random_humps(rng)), precision=precision)
    return mesh, cfg


def ensemble_member(n, seed, extent=10000.0, dt=0.5, precision="fp32"):
    rng = np.random.default_rng(seed)
    bath = meshgen.bath_gaussians(seed, ((0, extent), (0, extent)))
    mesh = meshgen.quad_mesh(n, n, corners=((0, 0), (extent, 0), (extent, extent), (0, extent)), bc=(LAND,) * 4,
                             bathymetry=bath, name="member_%d" % seed)
    hump = [(rng.uniform(0.5, 2.0), rng.uniform(0.3, 0.7) * extent, rng.uniform(0.3, 0.7) * extent,
             rng.uniform(0.03, 0.1) * extent)]
    cfg = ProblemConfig(p=1, rk_nstages=2, rk_order=2, dt=dt, g=9.81, wetting_drying=True, h_o=0.01, ic_type=1,
                        function_set=FN_GAUSSIAN_HUMPS, fn_params=humps_params(hump), precision=precision)
    return mesh, cfg


def config5(n_members=256, seed=0, nmin=64, nmax=200, dt=0.5, precision="fp32"):
    """Ensemble of independent p=1 wet/dry runs: member k has n x n quads with n uniform in [nmin, nmax]
    (seeded), a bathymetry of 8 seeded Gaussians (depth 1-20 m) and a Gaussian hump on the surface.
    Returns (meshes, member_cfgs): every member shares the configuration except its function-set
    parameters (the hump)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nmin, nmax + 1, size=n_members)
    meshes, cfgs = [], []
    for k, n in enumerate(sizes):
        mesh, cfg = ensemble_member(int(n), seed * 100003 + k, dt=dt, precision=precision)
        meshes.append(mesh)
        cfgs.append(cfg)
    return meshes, cfgs


# tidal constituents used by the channel workload (frequencies in rad/s)
M2_FREQ = 1.405189e-4
K1_FREQ = 7.292117e-5


def tidal_channel(nx=24, ny=6, p=1, rk=(2, 2), dt=2.0, friction="chezy", cf=0.0025, ramp_days=0.01, flow=True,
                  precision="fp64", jitter=0.15, seed=3, length=10000.0, width=2000.0, depth=10.0):
    """Channel [0, length] x [0, width]: tide (M2 + K1, amplitude and phase varying along the open end) on
    x = 0, a river inflow (steady part plus a one-hour oscillation) on x = length (land there when
    flow=False), land along both sides; depth falls linearly from `depth` to 0.6 `depth`. friction:
    None, "chezy" (coefficient cf) or "manning" (n from 0.02 to 0.03 along the channel, lower bound cf).
    Starts at rest; the forcing ramps up over ramp_days."""
    def bath(x, y):
        return depth - 0.4 * depth * x / length

    mesh = meshgen.quad_mesh(nx, ny, corners=((0, 0), (length, 0), (length, width), (0, width)),
                             bc=(LAND, FLOW if flow else LAND, LAND, TIDE), jitter=jitter, seed=seed, bathymetry=bath,
                             name="tidal_channel_%dx%d" % (nx, ny))
    x, y = mesh.node_xyz[:, 0], mesh.node_xyz[:, 1]
    left = np.arange(ny + 1) * (nx + 1)
    right = nx + np.arange(ny + 1) * (nx + 1)
    yl = y[left] / width
    forcing = [ForcingBlock(TIDE, left, np.array([M2_FREQ, K1_FREQ]), np.array([1.0, 0.9]), np.array([30.0, 120.0]),
                            np.stack([0.4 + 0.1 * yl, 0.15 + 0.0 * yl]), np.stack([10.0 + 20.0 * yl, 50.0 + 0.0 * yl]))]
    if flow:
        yr = y[right] / width
        forcing.append(ForcingBlock(FLOW, right, np.array([0.0, 2 * math.pi / 3600.0]), np.array([1.0, 1.0]),
                                    np.array([0.0, 0.0]), np.stack([-0.3 + 0.0 * yr, 0.1 + 0.05 * yr]),
                                    np.stack([0.0 * yr, 90.0 + 0.0 * yr])))
    mesh.forcing = forcing
    kind = {None: FRICTION_NONE, "chezy": FRICTION_CHEZY, "manning": FRICTION_MANNING}[friction]
    if kind == FRICTION_MANNING:
        mesh.node_manning_n = 0.02 + 0.01 * x / length
    cfg = ProblemConfig(p=p, rk_nstages=rk[0], rk_order=rk[1], dt=dt, g=9.81, ic_type=0, ic_const=(0.0, 0.0, 0.0),
                        bottom_friction=kind, friction_cf=cf, ramp_duration=ramp_days, precision=precision)
    return mesh, cfg


def levee_channel(nx=24, ny=6, p=1, rk=(2, 2), dt=1.0, crest=0.1, c_sub=0.8, c_super=0.6, dry_right=False,
                  friction="chezy", cf=0.0025, ramp_days=0.005, precision="fp64", jitter=0.1, seed=4,
                  length=10000.0, width=2000.0, depth=10.0, limiter=False):
    """The tidal channel cut across its middle by a levee (an internal barrier of coincident but distinct
    nodes) with crest elevation `crest` and discharge coefficients c_sub / c_super: the tide (M2 + K1) on
    x = 0 overtops it into the right half. dry_right: the right half is land 0.05 m above datum (with
    wetting/drying, h_o = 0.01 m) that the overtopping floods; else it is 0.6 `depth` deep with a
    river flow on x = length. limiter: the Cockburn-Shu limiter (M = 1e-8, nu = 1.5)."""
    def bath(x, y):
        b = depth - 0.4 * depth * x / length
        return np.where(x > length / 2 + 1e-9, -0.05, b) if dry_right else b

    right_bc = LAND if dry_right else FLOW
    mesh = meshgen.barrier_channel(nx, ny, length, width, bc_left=TIDE, bc_right=right_bc, jitter=jitter, seed=seed,
                                   bathymetry=bath, name="levee_channel_%dx%d" % (nx, ny))
    x, y = mesh.node_xyz[:, 0], mesh.node_xyz[:, 1]
    left = mesh.seg_nodes[mesh.seg_offsets[2]:mesh.seg_offsets[3]]
    yl = y[left] / width
    forcing = [ForcingBlock(TIDE, left, np.array([M2_FREQ, K1_FREQ]), np.array([1.0, 0.9]), np.array([30.0, 120.0]),
                            np.stack([0.4 + 0.1 * yl, 0.15 + 0.0 * yl]), np.stack([10.0 + 20.0 * yl, 50.0 + 0.0 * yl]))]
    if not dry_right:
        right = mesh.seg_nodes[mesh.seg_offsets[4]:mesh.seg_offsets[5]]
        forcing.append(ForcingBlock(FLOW, right, np.array([0.0]), np.array([1.0]), np.array([0.0]),
                                    np.full((1, len(right)), -0.2), np.zeros((1, len(right)))))
    mesh.forcing = forcing
    npair = len(mesh.levee_pairs)
    yb = y[mesh.levee_pairs[:, 0]] / width
    mesh.levee_data = np.stack([crest + 0.05 * yb, np.full(npair, c_sub), np.full(npair, c_super)], 1)
    kind = {None: FRICTION_NONE, "chezy": FRICTION_CHEZY, "manning": FRICTION_MANNING}[friction]
    if kind == FRICTION_MANNING:
        mesh.node_manning_n = 0.02 + 0.01 * x / length
    cfg = ProblemConfig(p=p, rk_nstages=rk[0], rk_order=rk[1], dt=dt, g=9.81, ic_type=0, ic_const=(0.0, 0.0, 0.0),
                        bottom_friction=kind, friction_cf=cf, ramp_duration=ramp_days, precision=precision,
                        wetting_drying=dry_right, h_o=0.01, slope_limiting=limiter, sl_M=1.0e-8, sl_nu=1.5)
    return mesh, cfg
