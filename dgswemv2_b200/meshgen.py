"""Structured quadrilateral -> triangle mesh generator.

Follows the reference's mesh_generators/quad_mesh_generator.cpp: a bilinear map of the index grid
onto the quadrilateral (x1,y1)..(x4,y4) (:101-130), node numbering j*(m+1)+i, element patterns
simple/zigzag/checker (:464-541), and four boundary node chains bottom, right, top, left (:144-160).
Two additions the reference lacks: seeded jitter of interior nodes (uniform in +-frac of the local
cell size, boundary nodes fixed) and a choice of bathymetry functions evaluated at the nodes.
"""
import numpy as np

from .types import LAND, LEVEE, MeshArrays

SIMPLE, ZIGZAG, CHECKER = 0, 1, 2


def _triangles(m, n, pattern):
    j, i = np.meshgrid(np.arange(n), np.arange(m), indexing="ij")
    i = i.ravel()
    j = j.ravel()
    sw = i + (m + 1) * j
    se = sw + 1
    nw = i + m + 1 + (m + 1) * j
    ne = i + m + 2 + (m + 1) * j
    a = np.stack([sw, ne, nw], 1)  # element 2i + 2mj   (simple pattern)
    b = np.stack([sw, se, ne], 1)  # element 2i + 2mj + 1
    if pattern == SIMPLE:
        alt = np.zeros_like(i, bool)
    elif pattern == ZIGZAG:
        alt = (j % 2) == 1
    elif pattern == CHECKER:
        alt = ((i + j) % 2) == 1
    else:
        raise ValueError("unknown pattern")
    a2 = np.stack([sw, se, nw], 1)
    b2 = np.stack([se, ne, nw], 1)
    a = np.where(alt[:, None], a2, a)
    b = np.where(alt[:, None], b2, b)
    tri = np.empty((2 * m * n, 3), np.int32)
    idx = 2 * i + 2 * m * j
    tri[idx] = a
    tri[idx + 1] = b
    return tri


def bath_flat(depth):
    return lambda x, y: np.full_like(x, depth)


def bath_thacker(h0, a, xc=0.0, yc=0.0):
    return lambda x, y: h0 * (1.0 - ((x - xc) ** 2 + (y - yc) ** 2) / (a * a))


def bath_gaussians(seed, extent, n=8, dmin=1.0, dmax=20.0):
    """Sum of n seeded Gaussians scaled to depths in [dmin, dmax]."""
    rng = np.random.default_rng(seed)
    (x0, x1), (y0, y1) = extent
    cx = rng.uniform(x0, x1, n)
    cy = rng.uniform(y0, y1, n)
    s = rng.uniform(0.1, 0.3, n) * max(x1 - x0, y1 - y0)
    amp = rng.uniform(0.2, 1.0, n)

    def f(x, y):
        acc = np.zeros_like(x)
        for k in range(n):
            acc += amp[k] * np.exp(-((x - cx[k]) ** 2 + (y - cy[k]) ** 2) / (2 * s[k] ** 2))
        return dmin + (dmax - dmin) * acc / amp.sum()

    return f


def quad_mesh(m, n, corners=((0, 0), (1, 0), (1, 1), (0, 1)), bc=(LAND, LAND, LAND, LAND), pattern=SIMPLE,
              jitter=0.0, seed=0, bathymetry=None, name="quadrilateral"):
    """m x n quads -> 2mn triangles. corners = (x1,y1),(x2,y2),(x3,y3),(x4,y4) counter-clockwise.
    bc = boundary types of the chains bottom (1-2), right (2-3), top (4-3), left (1-4)."""
    (x1, y1), (x2, y2), (x3, y3), (x4, y4) = corners
    i = np.arange(m + 1)
    j = np.arange(n + 1)
    J, I = np.meshgrid(j, i, indexing="ij")
    xi = -1.0 + (2.0 / m) * I
    eta = -1.0 + (2.0 / n) * J
    N1 = (1.0 - xi) * (1.0 - eta) / 4.0
    N2 = (1.0 + xi) * (1.0 - eta) / 4.0
    N3 = (1.0 + xi) * (1.0 + eta) / 4.0
    N4 = (1.0 - xi) * (1.0 + eta) / 4.0
    x = x1 * N1 + x2 * N2 + x3 * N3 + x4 * N4
    y = y1 * N1 + y2 * N2 + y3 * N3 + y4 * N4
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        hx = np.hypot(x2 - x1, y2 - y1) / m
        hy = np.hypot(x4 - x1, y4 - y1) / n
        dx = rng.uniform(-jitter * hx, jitter * hx, x.shape)
        dy = rng.uniform(-jitter * hy, jitter * hy, y.shape)
        interior = (I > 0) & (I < m) & (J > 0) & (J < n)
        x = np.where(interior, x + dx, x)
        y = np.where(interior, y + dy, y)
    x = x.ravel()
    y = y.ravel()
    z = bathymetry(x, y) if bathymetry is not None else np.zeros_like(x)
    nodes = np.stack([x, y, z], 1).astype(np.float64)
    tri = _triangles(m, n, pattern)
    chains = [np.arange(m + 1), m + np.arange(n + 1) * (m + 1), np.arange(m + 1) + (m + 1) * n, np.arange(n + 1) * (m + 1)]
    seg_type = np.array(bc, np.int32)
    seg_offsets = np.concatenate([[0], np.cumsum([len(c) for c in chains])]).astype(np.int64)
    seg_nodes = np.concatenate(chains).astype(np.int32)
    return MeshArrays(nodes, tri, seg_type, seg_offsets, seg_nodes, None, name)


def barrier_channel(nx, ny, length, width, xb=None, bc_left=LAND, bc_right=LAND, jitter=0.0, seed=0,
                    bathymetry=None, name="barrier_channel"):
    """Channel [0, length] x [0, width] cut at x = xb by an internal barrier: two quad meshes (nx // 2 and
    nx - nx // 2 columns) whose facing node columns coincide but stay distinct nodes, joined by a LEVEE
    chain (front = the left part's column, back = the right part's, both bottom to top). Chains: left
    part bottom, top, left (bc_left); right part bottom, right (bc_right), top; then the barrier."""
    xb = length / 2 if xb is None else xb
    nl, nr = nx // 2, nx - nx // 2
    A = quad_mesh(nl, ny, corners=((0, 0), (xb, 0), (xb, width), (0, width)), bc=(LAND, LAND, LAND, bc_left),
                  jitter=jitter, seed=seed, bathymetry=bathymetry)
    B = quad_mesh(nr, ny, corners=((xb, 0), (length, 0), (length, width), (xb, width)), bc=(LAND, bc_right, LAND, LAND),
                  jitter=jitter, seed=seed + 1, bathymetry=bathymetry)
    off = A.n_nodes
    chains, types = [], []
    for k in (0, 2, 3):  # bottom, top, left of the left part
        chains.append(A.seg_nodes[A.seg_offsets[k]:A.seg_offsets[k + 1]])
        types.append(int(A.seg_type[k]))
    for k in (0, 1, 2):  # bottom, right, top of the right part
        chains.append(B.seg_nodes[B.seg_offsets[k]:B.seg_offsets[k + 1]] + off)
        types.append(int(B.seg_type[k]))
    front = A.seg_nodes[A.seg_offsets[1]:A.seg_offsets[2]]
    back = B.seg_nodes[B.seg_offsets[3]:B.seg_offsets[4]] + off
    chains.append(np.concatenate([front, back]))
    types.append(LEVEE)
    nodes = np.concatenate([A.node_xyz, B.node_xyz])
    tri = np.concatenate([A.elem_nodes, B.elem_nodes + off]).astype(np.int32)
    seg_offsets = np.concatenate([[0], np.cumsum([len(c) for c in chains])]).astype(np.int64)
    mesh = MeshArrays(nodes, tri, np.array(types, np.int32), seg_offsets, np.concatenate(chains).astype(np.int32),
                      None, name)
    mesh.levee_pairs = np.stack([front, back], 1).astype(np.int32)
    return mesh


def write_adcirc(mesh, path):
    """Write the mesh as ADCIRC fort.14. Tide chains become open boundaries; the other chains become
    land-boundary segments with IBTYPE 0 (land), 2 (flow), 77 (function), 88 (outflow)."""
    from .types import TIDE

    ib = {0: 0, 2: 2, 3: 77, 4: 88, LEVEE: 4}
    chains = [(int(mesh.seg_type[s]), mesh.seg_nodes[mesh.seg_offsets[s]:mesh.seg_offsets[s + 1]])
              for s in range(len(mesh.seg_type))]
    open_ch = [c for t, c in chains if t == TIDE]
    land_ch = [(t, c) for t, c in chains if t != TIDE]
    with open(path, "w") as f:
        f.write(mesh.name + "\n")
        f.write("%d    %d\n" % (mesh.n_elems, mesh.n_nodes))
        for k, (x, y, z) in enumerate(mesh.node_xyz):
            f.write("%d %.17g %.17g %.17g\n" % (k, x, y, z))
        ids = mesh.elem_ids if mesh.elem_ids is not None else np.arange(mesh.n_elems)
        for k, (a, b, c) in enumerate(mesh.elem_nodes):
            f.write("%d 3 %d %d %d\n" % (ids[k], a, b, c))
        f.write("%d = Number of open boundaries\n" % len(open_ch))
        f.write("%d = Total number of open boundary nodes\n" % sum(len(c) for c in open_ch))
        for s, chain in enumerate(open_ch):
            f.write("%d = Number of nodes for open boundary %d\n" % (len(chain), s + 1))
            for nd in chain:
                f.write("%d\n" % nd)
        f.write("%d = Number of land boundaries\n" % len(land_ch))
        f.write("%d = Total number of land boundary nodes\n" %
                sum(len(c) // 2 if t == LEVEE else len(c) for t, c in land_ch))
        for s, (t, chain) in enumerate(land_ch):
            if t == LEVEE:  # NBVV IBCONN BARINTH BARINCFSB BARINCFSP (the RKDG step takes these from .bcis)
                n = len(chain) // 2
                f.write("%d %d = Number of nodes for land boundary %d\n" % (n, ib[t], s + 1))
                for a, b in zip(chain[:n], chain[n:]):
                    f.write("%d %d 0.0 1.0 1.0\n" % (a, b))
                continue
            f.write("%d %d = Number of nodes for land boundary %d\n" % (len(chain), ib[t], s + 1))
            for nd in chain:
                f.write("%d\n" % nd)
        f.write("0 = Number of generic boundaries\n0 = Total number of generic boundary nodes\n")


def write_bcis(mesh, path):
    """Write the mesh's tide / flow forcing blocks as a `.bcis` file in the layout SWE::Inputs::read_bcis
    reads (swe_inputs.cpp:211-290): "type nnodes", the constituent count, then per constituent
    "frequency forcing_fact equilib_arg" and one "node amplitude phase" line per node."""
    with open(path, "w") as f:
        if getattr(mesh, "levee_pairs", None) is not None and len(mesh.levee_pairs):
            f.write("%d %d = levee pairs\n" % (LEVEE, len(mesh.levee_pairs)))
            for (a, b), (H, cs, cp) in zip(mesh.levee_pairs, mesh.levee_data):
                f.write("%d %d %.17g %.17g %.17g\n" % (a, b, H, cs, cp))
        for b in mesh.forcing:
            nodes = np.asarray(b.nodes)
            f.write("%d %d = %s boundary\n" % (int(b.type), len(nodes), "tide" if int(b.type) == 1 else "flow"))
            f.write("%d = number of constituents\n" % len(b.frequency))
            for c in range(len(b.frequency)):
                f.write("%.17g %.17g %.17g\n" % (b.frequency[c], b.forcing_fact[c], b.equilib_arg[c]))
                for j, nd in enumerate(nodes):
                    f.write("%d %.17g %.17g\n" % (nd, b.amplitude[c][j], b.phase[c][j]))


def write_manning(mesh, path):
    """Write the mesh's Manning n as "node n" lines (the file swe_pre_init_data.hpp:165-182 reads)."""
    with open(path, "w") as f:
        for k, n in enumerate(mesh.node_manning_n):
            f.write("%d %.17g\n" % (k, n))
