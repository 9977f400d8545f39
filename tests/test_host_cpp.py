"""The C++ host side (include/dgsw_rkdg_problem.hpp): `.15` YAML + ADCIRC parsing mirrors the reference's
InputParameters / SWE::Inputs / AdcircFormat, and the dgswemv2-b200-serial driver runs an input file
end to end on the GPU.

CPU tests compile tests/cpp/parse_check.cpp against the header and compare what it read with the values
written and with the Python mesh arrays (bit-exact hashes, host-only topology included)."""
import os
import re
import subprocess

import numpy as np
import pytest

from dgswemv2_b200 import Problem, configs, mesh_topology, meshgen
from dgswemv2_b200.types import FUNCTION, LAND, OUTFLOW

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dgswemv2_b200")
CLI = os.path.join(PKG, "dgswemv2-b200-serial")


@pytest.fixture(scope="module")
def parse_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "parse_check")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-Wall", "-Werror", "-o", exe,
                           os.path.join(ROOT, "tests", "cpp", "parse_check.cpp"), "-L" + PKG, "-ldgsw_rkdg",
                           "-Wl,-rpath," + PKG])
    return exe


def run_check(exe, path):
    r = subprocess.run([exe, path], capture_output=True, text=True)
    out = {}
    for line in r.stdout.splitlines():
        k, _, v = line.partition(" ")
        out[k] = v
    return r.returncode, out, r.stderr


def fnv(arr):
    h = 1469598103934665603
    for b in np.ascontiguousarray(arr).tobytes():
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return str(h)


def write_input(d, mesh, body, mesh_name="mesh.14"):
    meshgen.write_adcirc(mesh, os.path.join(d, mesh_name))
    path = os.path.join(d, "input.15")
    with open(path, "w") as f:
        f.write(body.replace("@MESH@", mesh_name))
    return path


CONFIG1_15 = """###############################################################################
#  config 1: manufactured solution, p=1, SSP-RK2, dt = 1 s, 1000 steps
###############################################################################

mesh:
  format: Adcirc
  file_name: @MESH@
  coordinate_system: cartesian

timestepping:
  start_time: 01-01-2000 00:00:00      # dd-mm-yyyy hh:mm:ss
  end_time: 01-01-2000 00:16:40
  dt: 1.0
  order: 2
  nstages: 2

polynomial_order: 1

problem:
  name: rkdg_swe
  gravity: 9.81
  density_water: 1000
  density_air: 1.225
  initial_conditions:
    type: Function
  function_source: Enable

b200:
  function_set: manufactured_sine
  function_parameters: [40000, 0.1, 2.0, 0.0, 9.81]
  precision: fp64
"""


def test_parse_config1_input_and_mesh(parse_check, tmp_path):
    mesh, cfg = configs.config1()
    rc, out, err = run_check(parse_check, write_input(str(tmp_path), mesh, CONFIG1_15))
    assert rc == 0, (out, err)
    assert out["p"] == "1" and out["mesh_format"] == "Adcirc" and out["mesh_file"] == "mesh.14"
    assert out["bcis_file"] == "mesh.bcis" and out["coordinate_system"] == "cartesian"
    assert float(out["run_time"]) == 1000.0 and float(out["dt"]) == 1.0
    assert out["order"] == "2" and out["nstages"] == "2" and out["name"] == "rkdg_swe"
    assert float(out["g"]) == 9.81 and float(out["rho_air"]) == 1.225
    assert out["ic_type"] == "1" and out["function_source"] == "1"
    assert out["wetting_drying"] == "0" and out["slope_limiting"] == "0"
    assert float(out["h_o"]) == 0.1 and float(out["sl_M"]) == 1e-8 and float(out["sl_nu"]) == 1.5  # defaults
    assert out["function_set"] == "2" and out["precision"] == "0" and out["n_params"] == "5"
    # the mesh round trip is bit-exact (names are 0..n-1, so ascending-name order is the input order)
    assert out["mesh_name"] == mesh.name
    assert int(out["n_nodes"]) == mesh.n_nodes and int(out["n_elems"]) == mesh.n_elems
    assert out["node_xyz_hash"] == fnv(mesh.node_xyz.astype(np.float64))
    assert out["elem_nodes_hash"] == fnv(mesh.elem_nodes.astype(np.int32))
    assert out["elem_ids_hash"] == fnv(np.arange(mesh.n_elems, dtype=np.uint32))
    assert out["seg_type_hash"] == fnv(mesh.seg_type.astype(np.int32))
    assert out["seg_nodes_hash"] == fnv(mesh.seg_nodes.astype(np.int32))
    nbr, bt, intf, bnd = mesh_topology(mesh)
    assert int(out["n_interfaces"]) == len(intf) and int(out["n_boundaries"]) == len(bnd)
    assert out["neighbors_hash"] == fnv(nbr) and out["btype_hash"] == fnv(bt)
    assert out["interfaces_hash"] == fnv(intf) and out["boundaries_hash"] == fnv(bnd)


BOWL_15 = """mesh:
  format: Adcirc
  file_name: '@MESH@'
  coordinate_system: cartesian
timestepping:
  start_time: 15-11-1987 12:00              #dd-mm-yyyy hh:mm
  end_time: 15-11-1987 13:00                #dd-mm-yyyy hh:mm
  dt: 0.25
  order: 2
  nstages: 2
polynomial_order: 1
problem:
  name: rkdg_swe
  initial_conditions:
    type: Constant
    initial_surface_height: 0.5
    initial_momentum_x: -1.5e-2
    initial_momentum_y: 0
  wetting_drying:
    h_o: 0.01
  slope_limiting:
    type: Cockburn-Shu
    M: 1.0e-6
    nu: 1.25
output:
  path: out
  modal:
    frequency: 10
"""


def test_parse_bowl_style_input(parse_check, tmp_path):
    """Constant IC, wetting/drying and Cockburn-Shu nodes, quoted scalars, end-of-line comments, times without
    seconds (strptime stops at the missing field, as in the reference's own bowl example), and a mesh whose
    elements are listed with shuffled names (the reader orders them by name) and with outflow segments."""
    mesh = meshgen.quad_mesh(6, 5, bc=(LAND, OUTFLOW, FUNCTION, LAND), jitter=0.1, seed=4,
                             bathymetry=meshgen.bath_flat(3.0))
    rng = np.random.default_rng(0)
    mesh.elem_ids = rng.permutation(mesh.n_elems).astype(np.uint32) * 3 + 7
    rc, out, err = run_check(parse_check, write_input(str(tmp_path), mesh, BOWL_15))
    assert rc == 0, (out, err)
    assert float(out["run_time"]) == 3600.0 and float(out["dt"]) == 0.25
    assert float(out["g"]) == 9.81  # default
    assert out["ic_type"] == "0" and [float(v) for v in out["ic_const"].split()] == [0.5, -1.5e-2, 0.0]
    assert out["wetting_drying"] == "1" and float(out["h_o"]) == 0.01
    assert out["slope_limiting"] == "1" and float(out["sl_M"]) == 1.0e-6 and float(out["sl_nu"]) == 1.25
    assert out["writing_modal"] == "1 40" and out["function_set"] == "0"
    order = np.argsort(mesh.elem_ids, kind="stable")
    assert out["elem_nodes_hash"] == fnv(mesh.elem_nodes[order].astype(np.int32))
    assert out["elem_ids_hash"] == fnv(np.sort(mesh.elem_ids).astype(np.uint32))
    nbr, bt, intf, bnd = mesh_topology(mesh)  # the library orders by element ID itself
    assert out["neighbors_hash"] == fnv(nbr) and out["interfaces_hash"] == fnv(intf)
    assert out["boundaries_hash"] == fnv(bnd)


@pytest.mark.parametrize("edit, status, text", [
    (lambda s: s.replace("polynomial_order: 1\n", ""), "-1", "P YAML node not specified"),
    (lambda s: s.replace("  dt: 1.0\n", ""), "-1", "Timestepping YAML node is malformatted"),
    (lambda s: s.replace("format: Adcirc", "format: Gmsh"), "-1", "Unsupported mesh format: Gmsh"),
    (lambda s: s.replace("cartesian", "conic"), "-1", "Unsupported coordinate system: conic"),
    (lambda s: s.replace("  function_source: Enable\n", "  bottom_friction:\n    type: Chezy\n    coefficient: -0.1\n"),
     "-1", "Chezy friction coefficient must be postive"),
    (lambda s: s.replace("  function_source: Enable\n", "  meteo_forcing:\n    type: Enable\n"), "5", "meteo forcing"),
    (lambda s: s.replace("function_set: manufactured_sine", "function_set: tsunami"), "-1", "unknown b200.function_set"),
    (lambda s: s.replace("name: rkdg_swe", "name: ehdg_swe"), "5", "is not rkdg_swe"),
])
def test_input_errors(parse_check, tmp_path, edit, status, text):
    mesh, _ = configs.config1()
    rc, out, _ = run_check(parse_check, write_input(str(tmp_path), mesh, edit(CONFIG1_15)))
    assert rc == 3 and out["error"].split(" ", 1)[0] == status and text in out["error"], out


def test_mesh_errors(parse_check, tmp_path):
    mesh, _ = configs.config1()
    path = write_input(str(tmp_path), mesh, CONFIG1_15)
    mpath = os.path.join(str(tmp_path), "mesh.14")
    src = open(mpath).read()
    # an undefined IBTYPE is rejected like AdcircFormat does
    open(mpath, "w").write(src.replace("77 = Number of nodes for land boundary 1", "5 = Number of nodes for land boundary 1"))
    rc, out, _ = run_check(parse_check, path)
    assert rc == 3 and "undefined boundary type in ADCIRC mesh: 5" in out["error"]
    # an internal barrier segment needs five columns per line (NBVV IBCONN BARINTH BARINCFSB BARINCFSP)
    open(mpath, "w").write(src.replace("77 = Number of nodes for land boundary 1", "4 = Number of nodes for land boundary 1"))
    rc, out, _ = run_check(parse_check, path)
    assert rc == 3 and "error" in out
    # an island segment (IBTYPE 1) is read but never matched: its edges then have no boundary type
    open(mpath, "w").write(src.replace("77 = Number of nodes for land boundary 1", "1 = Number of nodes for land boundary 1"))
    rc, out, _ = run_check(parse_check, path)
    assert rc == 3 and "boundary not found" in out["error"]
    os.remove(mpath)
    rc, out, _ = run_check(parse_check, path)
    assert rc == 3 and "was not found" in out["error"]


@pytest.mark.gpu
def test_serial_driver_runs_config1(tmp_path, oracle):
    """dgswemv2-b200-serial on the config-1 input: 1000 SSP-RK2 steps, L2 error equal to the FP64 oracle's
    within 1e-12 relative."""
    mesh, cfg = configs.config1()
    path = write_input(str(tmp_path), mesh, CONFIG1_15)
    r = subprocess.run([CLI, path], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"L2 error: ([0-9.eE+-]+)", r.stdout)
    assert m and "Time Elapsed (in us)" in r.stdout, r.stdout
    l2_cli = float(m.group(1))
    O = oracle.problem(cfg, mesh, n_threads=8)
    O.step(1000)
    l2_ref = O.l2_error()
    assert abs(l2_cli - l2_ref) <= 1e-12 * l2_ref, (l2_cli, l2_ref)
    P = Problem(cfg, mesh)
    P.step_serial(1000)
    assert abs(P.compute_residual_L2() - l2_cli) <= 1e-13 * l2_ref


TIDE_15 = """mesh:
  format: Adcirc
  file_name: @MESH@
  coordinate_system: cartesian

timestepping:
  start_time: 01-01-2000 00:00:00
  end_time: 01-01-2000 00:05:00
  dt: 1.0
  order: 3
  nstages: 3
  ramp_duration: 0.01

polynomial_order: 2

problem:
  name: rkdg_swe
  gravity: 9.81
  bottom_friction:
    type: Manning
    coefficient: 0.0005
    input_file: manning.dat
  initial_conditions:
    type: Constant
    initial_surface_height: 0.0
    initial_momentum_x: 0.0
    initial_momentum_y: 0.0

output:
  path: out/
  modal:
    frequency: 300
"""


def read_modal_last(path, ne, nd):
    """The last block of a write_modal_data file: its time and the modes [ne][nd] (elements in file order)."""
    lines = [l for l in open(path).read().split("\n") if l]
    block = ne * nd + 1
    assert len(lines) % block == 0, (len(lines), block)
    last = lines[-block:]
    vals = np.array([float(l.split()[1]) for l in last[1:]]).reshape(ne, nd)
    ids = np.array([int(l.split()[0]) for l in last[1:]]).reshape(ne, nd)
    return float(last[0]), vals, ids


def write_tide_input(d, mesh):
    path = write_input(d, mesh, TIDE_15, mesh_name="channel.14")
    meshgen.write_bcis(mesh, os.path.join(d, "channel.bcis"))
    meshgen.write_manning(mesh, os.path.join(d, "manning.dat"))
    return path


def test_parse_tide_flow_and_manning_input(parse_check, tmp_path):
    """Open boundaries read as tide, IBTYPE 2 as flow; the .bcis blocks, the Manning n file, bottom
    friction and the ramp duration come through bit for bit."""
    mesh, cfg = configs.tidal_channel(p=2, rk=(3, 3), dt=1.0, friction="manning", cf=0.0005)
    rc, out, err = run_check(parse_check, write_tide_input(str(tmp_path), mesh))
    assert rc == 0, (out, err)
    assert out["bottom_friction"] == "2 0.00050000000000000001" and out["manning_file"] == "manning.dat"
    assert float(out["ramp_duration"]) == 0.01
    assert out["n_forcing"] == "2"
    for k, b in enumerate(mesh.forcing):
        fields = out["forcing_%d" % k].split()
        assert fields[:3] == [str(b.type), str(len(b.nodes)), str(len(b.frequency))]
        assert fields[3] == fnv(np.asarray(b.nodes, np.int32))
        h = fnv(np.asarray(b.equilib_arg, np.float64))
        h2 = int(h)
        for arr in (np.asarray(b.forcing_fact, np.float64), np.asarray(b.frequency, np.float64)):
            for byte in arr.tobytes():
                h2 = ((h2 ^ byte) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
        assert fields[4] == str(h2)
        assert fields[5] == fnv(np.asarray(b.amplitude, np.float64)) and fields[6] == fnv(np.asarray(b.phase, np.float64))
    assert out["manning_hash"] == fnv(np.asarray(mesh.node_manning_n, np.float64))
    nbr, bt, intf, bnd = mesh_topology(mesh)
    assert out["boundaries_hash"] == fnv(bnd)


def test_bcis_reader_skips_levees_and_unknown_nodes(parse_check, tmp_path):
    """A levee block is read past, a node ID the mesh lacks is dropped, and a node listed twice for one
    constituent is an error (the reference would shift that node's constituents)."""
    mesh, cfg = configs.tidal_channel(friction="manning", cf=0.0005)
    path = write_tide_input(str(tmp_path), mesh)
    bpath = os.path.join(str(tmp_path), "channel.bcis")
    b = mesh.forcing[0]
    n_tide = len(b.nodes)
    lines = open(bpath).read().split("\n")
    flow_block = "\n".join(lines[2 + len(b.frequency) * (1 + n_tide):])
    tide = ["1 %d = tide boundary" % (n_tide + 1), "%d" % len(b.frequency)]
    for c in range(len(b.frequency)):
        tide.append("%.17g %.17g %.17g" % (b.frequency[c], b.forcing_fact[c], b.equilib_arg[c]))
        tide += ["%d %.17g %.17g" % (nd, b.amplitude[c][j], b.phase[c][j]) for j, nd in enumerate(b.nodes)]
        tide.append("99999 1.0 2.0")
    levee = "129 2 = levee\n5 6 1.0 0.5 0.5\n7 8 1.0 0.5 0.5\n"
    open(bpath, "w").write(levee + "\n".join(tide) + "\n" + flow_block)
    rc, out, err = run_check(parse_check, path)
    assert rc == 0, (out, err)
    assert out["n_forcing"] == "2"
    fields = out["forcing_0"].split()
    assert fields[:3] == ["1", str(n_tide), str(len(b.frequency))]
    assert fields[5] == fnv(np.asarray(b.amplitude, np.float64))
    dup = tide[:3] + tide[3:4] + tide[3:]
    open(bpath, "w").write("\n".join(dup) + "\n")
    rc, out, _ = run_check(parse_check, path)
    assert rc == 3 and "twice" in out["error"]


@pytest.mark.gpu
def test_serial_driver_runs_tidal_channel(tmp_path):
    """dgswemv2-b200-serial on a tidal channel input (tide + flow from the .bcis file, Manning n from its
    file, ramp): the modal output after 300 steps equals the Python API's state bit for bit."""
    mesh, cfg = configs.tidal_channel(p=2, rk=(3, 3), dt=1.0, friction="manning", cf=0.0005)
    d = str(tmp_path)
    path = write_tide_input(d, mesh)
    os.makedirs(os.path.join(d, "out"), exist_ok=True)
    r = subprocess.run([CLI, path], capture_output=True, text=True, timeout=300, cwd=d)
    assert r.returncode == 0, r.stdout + r.stderr
    P = Problem(cfg, mesh)
    P.step_serial(300)
    q = P.get_state()
    t, ze, ids = read_modal_last(os.path.join(d, "out", mesh.name + "_modal_ze.txt"), mesh.n_elems, P.nd)
    assert t == 300.0 and np.array_equal(ids[:, 0], np.arange(mesh.n_elems))
    # six significant digits (std::scientific), as the reference prints them
    assert np.allclose(ze, q[:, 0, :], rtol=2e-6, atol=1e-6 * np.abs(q[:, 0, :]).max())


LEVEE_15 = TIDE_15.replace("  bottom_friction:\n    type: Manning\n    coefficient: 0.0005\n    input_file: manning.dat\n",
                           "  bottom_friction:\n    type: Chezy\n    coefficient: 0.0025\n").replace(
    "polynomial_order: 2", "polynomial_order: 1").replace("order: 3\n  nstages: 3", "order: 2\n  nstages: 2").replace(
    "ramp_duration: 0.01", "ramp_duration: 0.005")


def test_parse_internal_barrier_and_levee_data(parse_check, tmp_path):
    """IBTYPE 4 segments become levee chains (front then back nodes) and the .bcis levee lines come
    through as (front, back) pairs with their crest height and coefficients, bit for bit; the host
    topology of the parsed mesh equals the Python mesh's."""
    mesh, cfg = configs.levee_channel()
    d = str(tmp_path)
    path = write_input(d, mesh, LEVEE_15, mesh_name="channel.14")
    meshgen.write_bcis(mesh, os.path.join(d, "channel.bcis"))
    rc, out, err = run_check(parse_check, path)
    assert rc == 0, (out, err)
    assert out["n_levee_pairs"] == str(len(mesh.levee_pairs))
    h_nodes, h_data = out["levee_hash"].split()
    assert h_nodes == fnv(np.asarray(mesh.levee_pairs, np.int32)) and h_data == fnv(np.asarray(mesh.levee_data, np.float64))
    nbr, bt, intf, bnd = mesh_topology(mesh)
    assert out["neighbors_hash"] == fnv(nbr) and out["interfaces_hash"] == fnv(intf)
    assert out["boundaries_hash"] == fnv(bnd) and out["btype_hash"] == fnv(bt)
    assert int((bt == 129).sum()) == 2 * (len(mesh.levee_pairs) - 1)


@pytest.mark.gpu
def test_serial_driver_runs_levee_channel(tmp_path):
    """dgswemv2-b200-serial on the levee channel (IBTYPE 4 barrier + .bcis levee and tide/flow data):
    the modal output after 300 steps equals the Python API's state."""
    mesh, cfg = configs.levee_channel()
    d = str(tmp_path)
    path = write_input(d, mesh, LEVEE_15, mesh_name="channel.14")
    meshgen.write_bcis(mesh, os.path.join(d, "channel.bcis"))
    os.makedirs(os.path.join(d, "out"), exist_ok=True)
    r = subprocess.run([CLI, path], capture_output=True, text=True, timeout=300, cwd=d)
    assert r.returncode == 0, r.stdout + r.stderr
    P = Problem(cfg, mesh)
    P.step_serial(300)
    q = P.get_state()
    t, ze, _ = read_modal_last(os.path.join(d, "out", mesh.name + "_modal_ze.txt"), mesh.n_elems, P.nd)
    assert t == 300.0
    assert np.allclose(ze, q[:, 0, :], rtol=2e-6, atol=1e-6 * np.abs(q[:, 0, :]).max())


VTK_15 = LEVEE_15.replace("  modal:\n    frequency: 300\n", "  vtk:\n    frequency: 300\n  vtu:\n    frequency: 300\n  modal:\n    frequency: 300\n").replace(
    "    initial_momentum_y: 0.0\n", "    initial_momentum_y: 0.0\n  wetting_drying:\n    h_o: 0.01\n")


def test_parse_vtk_vtu_output_nodes(parse_check, tmp_path):
    mesh, cfg = configs.levee_channel(dry_right=True)
    d = str(tmp_path)
    path = write_input(d, mesh, VTK_15.replace("  vtu:\n    frequency: 300\n", "  vtu:\n    frequency: 150.5\n"),
                       mesh_name="channel.14")
    rc, out, err = run_check(parse_check, path)
    assert rc == 0, (out, err)
    assert out["writing_vtk"] == "1 300" and out["writing_vtu"] == "1 151" and out["writing_modal"] == "1 300"
    rc, out, _ = run_check(parse_check, write_input(d, mesh, VTK_15.replace("  vtk:\n    frequency: 300\n", "  vtk:\n")))
    assert rc == 3 and "VTK YAML node is malformatted" in out["error"]


def _vtk_sections(path):
    lines = open(path).read().split("\n")
    out, i = {}, 0
    while i < len(lines):
        l = lines[i]
        if l.startswith("SCALARS "):
            name = l.split()[1]
            j = i + 2
            vals = []
            while j < len(lines) and lines[j] and not lines[j][0].isalpha():
                vals.append(float(lines[j]))
                j += 1
            out[name] = np.array(vals)
            i = j
        else:
            i += 1
    return out, lines


@pytest.mark.gpu
def test_serial_driver_writes_vtk_vtu_and_modal(tmp_path, oracle):
    """VTK / VTU / modal output of dgswemv2-b200-serial on the levee channel flooding dry land: files at
    steps 0 and 300 named like the reference's; the VTK cell and point values equal the state evaluated
    with the oracle's Dubiner basis at the centroids and vertices (to the printed float digits); IDs,
    wet flags and the VTU arrays agree."""
    mesh, cfg = configs.levee_channel(dry_right=True)
    d = str(tmp_path)
    path = write_input(d, mesh, VTK_15, mesh_name="channel.14")
    meshgen.write_bcis(mesh, os.path.join(d, "channel.bcis"))
    os.makedirs(os.path.join(d, "out"), exist_ok=True)
    r = subprocess.run([CLI, path], capture_output=True, text=True, timeout=300, cwd=d)
    assert r.returncode == 0, r.stdout + r.stderr
    for step in (0, 300):
        for ext in ("vtk", "vtu"):
            assert os.path.exists(os.path.join(d, "out", "%s_data_%d.%s" % (mesh.name, step, ext)))
    for v in ("ze", "qx", "qy", "bath"):
        assert os.path.exists(os.path.join(d, "out", "%s_modal_%s.txt" % (mesh.name, v)))
    P = Problem(cfg, mesh)
    P.step_serial(300)
    q = P.get_state()
    nd = P.nd
    phi_c = oracle.dubiner(cfg.p, np.array([[-1.0 + 2.0 / 3.0, -1.0 + 2.0 / 3.0]]))[0][:, 0]
    phi_v = oracle.dubiner(cfg.p, np.array([[-1.0, -1.0], [1.0, -1.0], [-1.0, 1.0]]))[0]
    sec, lines = _vtk_sections(os.path.join(d, "out", "%s_data_300.vtk" % mesh.name))
    ne = mesh.n_elems
    for k, v in enumerate(("ze", "qx", "qy")):
        cell = q[:, k, :] @ phi_c[:nd]
        scale = max(np.abs(cell).max(), 1e-30)
        assert np.allclose(sec[v + "_cell"], cell, rtol=1e-5, atol=1e-6 * scale), v
        pts = (q[:, k, :] @ phi_v[:nd, :]).reshape(-1)
        assert np.allclose(sec[v + "_point"], pts, rtol=1e-5, atol=1e-6 * max(np.abs(pts).max(), 1e-30)), v
    assert np.array_equal(sec["ID"], np.arange(ne))
    assert np.array_equal(sec["wet_dry"].astype(np.uint8), P.get_wet())
    assert 0 < P.get_wet().sum() < ne
    assert "POINTS %d double" % (3 * ne) in lines and "CELL_TYPES %d" % ne in lines
    vtu = open(os.path.join(d, "out", "%s_data_300.vtu" % mesh.name)).read()
    assert '<Piece NumberOfPoints="%d" NumberOfCells="%d">' % (3 * ne, ne) in vtu
    ze_cell = np.array(vtu.split('Name="ze_cell" format="ascii">')[1].split("</DataArray>")[0].split(), float)
    assert np.allclose(ze_cell, sec["ze_cell"])
    pt, cell, wet, wd = P.postprocess()
    assert np.allclose(cell[:, 0], sec["ze_cell"], rtol=1e-5, atol=1e-6)
    assert np.array_equal(wet, P.get_wet())


def test_spherical_mesh_is_projected(parse_check, tmp_path):
    """coordinate_system: spherical projects (longitude, latitude) onto the cylinder through
    (longitude_o, latitude_o) as SWE::preprocess_mesh_data does, with the reference's PI."""
    mesh, _ = configs.config1()
    lon = -95.0 + mesh.node_xyz[:, 0] / 40000.0
    lat = 28.0 + mesh.node_xyz[:, 1] / 40000.0
    mesh.node_xyz = np.stack([lon, lat, mesh.node_xyz[:, 2]], 1)
    body = CONFIG1_15.replace("cartesian", "spherical").replace(
        "  gravity: 9.81\n", "  gravity: 9.81\n  spherical_projection:\n    longitude_o: -94.5\n    latitude_o: 28.5\n    R: 6378200.0\n")
    rc, out, err = run_check(parse_check, write_input(str(tmp_path), mesh, body))
    assert rc == 0, (out, err)
    PI = 3.14159265359
    R_o = 6378200.0 * np.cos(28.5 * PI / 180.0)
    xyz = mesh.node_xyz.copy()
    xyz[:, 0] = R_o * (lon - (-94.5)) * PI / 180.0
    xyz[:, 1] = 6378200.0 * lat * PI / 180.0
    assert out["projected_xyz_hash"] == fnv(xyz)
    assert out["spherical"] == "1"
