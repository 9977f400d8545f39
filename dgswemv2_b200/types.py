"""Plain-data containers shared by the Python host side: the problem configuration (the `.15` input
surface of SWE::Inputs, source/problem/SWE/problem_input/swe_inputs.hpp:126-155, plus the stepper
input) and the mesh arrays (nodes, element node triples, ADCIRC-style boundary segments)."""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

# boundary types (source/problem/SWE/swe_definitions.hpp:61-69)
LAND, TIDE, FLOW, FUNCTION, OUTFLOW = 0, 1, 2, 3, 4
INTERNAL = 128
LEVEE = 129  # an internal barrier chain: n front nodes, then the n back nodes across the barrier

# bottom friction types (source/problem/SWE/swe_definitions.hpp:92)
FRICTION_NONE, FRICTION_CHEZY, FRICTION_MANNING = 0, 1, 2

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
    bottom_friction: int = FRICTION_NONE  # problem.bottom_friction.type
    friction_cf: float = 0.0  # bottom_friction.coefficient
    ramp_duration: float = 0.0  # timestepping.ramp_duration (days) of the tide/flow forcing


@dataclass
class ForcingBlock:
    """One tide or flow block of a `.bcis` file (SWE::Inputs::read_bcis, swe_inputs.cpp:211-290)."""
    type: int  # TIDE or FLOW
    nodes: np.ndarray  # (n_nodes,) 0-based node indices
    frequency: np.ndarray  # (n_constituents,) rad/s
    forcing_fact: np.ndarray  # (n_constituents,)
    equilib_arg: np.ndarray  # (n_constituents,) degrees
    amplitude: np.ndarray  # (n_constituents, n_nodes)
    phase: np.ndarray  # (n_constituents, n_nodes) degrees


@dataclass
class MeshArrays:
    node_xyz: np.ndarray  # (n_nodes, 3) x, y, bathymetry depth
    elem_nodes: np.ndarray  # (n_elems, 3) 0-based node indices
    seg_type: np.ndarray  # (n_segments,) boundary type of each node chain
    seg_offsets: np.ndarray  # (n_segments + 1,)
    seg_nodes: np.ndarray  # concatenated node chains
    elem_ids: Optional[np.ndarray] = None  # reference element IDs (default 0..n-1)
    name: str = "mesh"
    node_manning_n: Optional[np.ndarray] = None  # (n_nodes,) Manning's n (FRICTION_MANNING)
    forcing: List[ForcingBlock] = field(default_factory=list)  # tide / flow data
    levee_pairs: Optional[np.ndarray] = None  # (n, 2) front, back node of each .bcis levee line
    levee_data: Optional[np.ndarray] = None  # (n, 3) H_barrier, C_subcritical, C_supercritical

    @property
    def n_elems(self):
        return int(self.elem_nodes.shape[0])

    @property
    def n_nodes(self):
        return int(self.node_xyz.shape[0])
