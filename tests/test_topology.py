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
