"""Plain-data containers shared by the Python host side: the problem configuration (the `.15` input
surface of SWE::Inputs, source/problem/SWE/problem_input/swe_inputs.hpp:126-155, plus the stepper
input) and the mesh arrays (nodes, element node triples, ADCIRC-style boundary segments)."""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

# boundary types (source/problem/SWE/swe_definitions.hpp:61-69)
LAND, TIDE, FLOW, FUNCTION, OUTFLOW = 0, 1, 2, 3, 4
INTERNAL = 128

# function sets (dgswemv2_b200/csrc/function_sets.h)
FN_NONE, FN_REFERENCE_MANUFACTURED, FN_MANUFACTURED_SINE, FN_THACKER_BOWL, FN_GAUSSIAN_HUMPS = range(5)


@dataclass
class ProblemConfig:
    p: int = 1
    rk_nstages: int = 2
    rk_order: int = 2
    dt: float = 1.0
    g: float = 9.81
    wetting_drying: bool = False
    h_o: float = 0.1
    slope_limiting: bool = False
    sl_M: float = 1.0e-8
    sl_nu: float = 1.5
    function_source: bool = False
    ic_type: int = 0  # 0 default/constant, 1 function
    ic_const: tuple = (0.0, 0.0, 0.0)
    function_set: int = FN_NONE
    fn_params: List[float] = field(default_factory=lambda: [0.0] * 16)
    spherical: bool = False
    sp_lat0_deg: float = 0.0
    sp_R: float = 6378200.0
    precision: str = "fp64"  # "fp64" or "fp32" (FP32 bulk, FP64 wet/dry tests and mass reduction)


@dataclass
class MeshArrays:
    node_xyz: np.ndarray  # (n_nodes, 3) x, y, bathymetry depth
    elem_nodes: np.ndarray  # (n_elems, 3) 0-based node indices
    seg_type: np.ndarray  # (n_segments,) boundary type of each node chain
    seg_offsets: np.ndarray  # (n_segments + 1,)
    seg_nodes: np.ndarray  # concatenated node chains
    elem_ids: Optional[np.ndarray] = None  # reference element IDs (default 0..n-1)
    name: str = "mesh"

    @property
    def n_elems(self):
        return int(self.elem_nodes.shape[0])

    @property
    def n_nodes(self):
        return int(self.node_xyz.shape[0])
