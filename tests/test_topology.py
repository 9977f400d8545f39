"""Integer topology of the library's host setup against the oracle's restatement of MeshMetaData and
interface/boundary creation: neighbours, face types, interface (in, ex, faces) order and boundary
order must match bit for bit."""
import numpy as np
import pytest

from dgswemv2_b200 import mesh_topology, meshgen
from dgswemv2_b200.types import FUNCTION, LAND, OUTFLOW, ProblemConfig


def _oracle_topology(oracle, mesh):
    cfg = ProblemConfig(p=1)
    P = oracle.problem(cfg, mesh)
    return P.topology()


@pytest.mark.parametrize("pattern", [meshgen.SIMPLE, meshgen.ZIGZAG, meshgen.CHECKER])
@pytest.mark.parametrize("jitter", [0.0, 0.2])
def test_topology_matches_oracle(oracle, pattern, jitter):
    mesh = meshgen.quad_mesh(7, 5, corners=((0, 0), (3, 0), (3, 2), (0, 2)), bc=(LAND, FUNCTION, OUTFLOW, LAND),
                             pattern=pattern, jitter=jitter, seed=3)
    a = mesh_topology(mesh)
    b = _oracle_topology(oracle, mesh)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_topology_with_permuted_element_ids(oracle):
    """Element IDs that are not the input order: the reference iterates elements by ID, and the
    smaller ID is the interface's "in" side."""
    mesh = meshgen.quad_mesh(6, 6, bc=(LAND, LAND, FUNCTION, FUNCTION), jitter=0.1, seed=1)
    rng = np.random.default_rng(7)
    mesh.elem_ids = rng.permutation(mesh.n_elems * 3)[: mesh.n_elems].astype(np.uint32)
    a = mesh_topology(mesh)
    b = _oracle_topology(oracle, mesh)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_topology_counts_structured():
    m, n = 20, 20
    mesh = meshgen.quad_mesh(m, n, bc=(FUNCTION,) * 4)
    nbr, bt, intf, bnd = mesh_topology(mesh)
    # 800 elements, 1160 interior edges, 80 boundary edges (the 20x20 manufactured-solution mesh)
    assert mesh.n_elems == 800
    assert intf.shape[0] == 1160
    assert bnd.shape[0] == 80
    assert np.all(intf[:, 0] < intf[:, 1])
    keys = intf[:, 0].astype(np.int64) * mesh.n_elems + intf[:, 1]
    assert np.all(np.diff(keys) > 0)


def test_boundary_lookup_error():
    """A boundary edge on no chain is an error (AdcircFormat::get_ibtype throws)."""
    from dgswemv2_b200._lib import DgswError

    mesh = meshgen.quad_mesh(3, 3)
    mesh.seg_type = mesh.seg_type[:3]
    mesh.seg_offsets = mesh.seg_offsets[:4]
    mesh.seg_nodes = mesh.seg_nodes[: mesh.seg_offsets[-1]]
    with pytest.raises(DgswError) as ei:
        mesh_topology(mesh)
    assert ei.value.status == 2


def test_tide_and_flow_boundaries_follow_land_in_creation_order(oracle):
    """Tide and flow faces are boundaries of their own types, created between land and function faces
    (ProblemBoundaryTypes order Land, Tide, Flow, Function)."""
    from dgswemv2_b200 import configs
    from dgswemv2_b200.types import FLOW, TIDE

    mesh, _ = configs.tidal_channel(nx=9, ny=4)
    a = mesh_topology(mesh)
    b = _oracle_topology(oracle, mesh)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    types = a[3][:, 2]
    assert set(types) == {LAND, TIDE, FLOW}
    assert np.all(np.diff(types) >= 0)  # grouped in type order
    assert int((types == TIDE).sum()) == 4 and int((types == FLOW).sum()) == 4


def test_tide_face_without_data_is_an_error(oracle):
    """A tide face whose nodes are in no tide block: create_boundaries' "unable to find tide data"."""
    from dgswemv2_b200 import configs

    mesh, cfg = configs.tidal_channel(nx=6, ny=3, flow=False)
    mesh.forcing[0].nodes = mesh.forcing[0].nodes[:2]
    mesh.forcing[0].amplitude = mesh.forcing[0].amplitude[:, :2]
    mesh.forcing[0].phase = mesh.forcing[0].phase[:, :2]
    with pytest.raises(RuntimeError, match="unable to find tide data"):
        oracle.problem(cfg, mesh)


def test_levee_interfaces_pair_the_two_sides_of_a_barrier(oracle):
    """Faces along an internal barrier become levee interfaces to the element across it (the node pair
    mirrored through the barrier's front/back strings), created after all internal interfaces."""
    from dgswemv2_b200 import configs
    from dgswemv2_b200.types import LEVEE

    mesh, _ = configs.levee_channel(nx=10, ny=4)
    a = mesh_topology(mesh)
    b = _oracle_topology(oracle, mesh)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    nbr, bt, intf, bnd = a
    lev = bt == LEVEE
    assert int(lev.sum()) == 2 * 4
    # the levee interfaces are the last ones, and each pairs one element of each half
    xc = mesh.node_xyz[mesh.elem_nodes, 0].mean(1)
    n_lev = 4
    for i_in, i_ex, f_in, f_ex in intf[-n_lev:]:
        assert bt[i_in, f_in] == LEVEE and bt[i_ex, f_ex] == LEVEE
        assert (xc[i_in] < 5000) != (xc[i_ex] < 5000)
    assert not np.any(bt[intf[:-n_lev, 0], intf[:-n_lev, 2]] == LEVEE)


def test_closed_chain_edge_is_found_at_any_occurrence(oracle):
    """A closed land chain lists its first node again at the end; the edge joining the last two nodes
    is found there (has_edge looks at every occurrence of a node)."""
    mesh = meshgen.quad_mesh(4, 3, bc=(LAND, LAND, LAND, LAND))
    m, n = 4, 3
    ring = list(range(m + 1)) + [m + j * (m + 1) for j in range(1, n + 1)] + \
        [m + n * (m + 1) - i for i in range(1, m + 1)] + [(n - j) * (m + 1) for j in range(1, n + 1)]
    assert ring[0] == ring[-1]
    mesh.seg_type = np.array([LAND], np.int32)
    mesh.seg_offsets = np.array([0, len(ring)], np.int64)
    mesh.seg_nodes = np.array(ring, np.int32)
    a = mesh_topology(mesh)
    b = _oracle_topology(oracle, mesh)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert len(a[3]) == 2 * (m + n)
