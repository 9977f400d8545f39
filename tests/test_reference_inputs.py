"""The reference's own input files, copied byte for byte into tests/golden/reference_inputs/ by
tests/golden/make_golden.py:

- sample_fort.14, the mesh of the reference's mesh-metadata round trip (test/test_mesh_metadata.cpp:26-45);
- the weir case (test/files_for_testing/weir/{dgswemv2_input.15, weir.14, weir.bcis}): an ADCIRC mesh
  with an IBTYPE 4 levee across it, a two-constituent flow boundary from the .bcis file, land elsewhere,
  p = 1, SSP-RK2, dt = 3 s for two hours, and the Cockburn-Shu limiter. The reference runs it in
  scripts/correctness/test_rkdg_parallel_weirs.sh:30-60.

Each file is read by the C++ host readers (include/dgsw_rkdg_problem.hpp, through tests/cpp/parse_check.cpp,
which writes the arrays it read), and exactly those arrays go to the library and to the oracle.
Tolerances: integer topology bit for bit; the weir run (limiter on) within 1e-9 of each variable's scale
with limiter decisions within 0.5 %, as the other limited runs.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from dgswemv2_b200 import Problem, mesh_topology
from dgswemv2_b200.types import TIDE, ForcingBlock, MeshArrays, ProblemConfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "dgswemv2_b200")
CLI = os.path.join(PKG, "dgswemv2-b200-serial")
INPUTS = os.path.join(ROOT, "tests", "golden", "reference_inputs")
DTYPES = {"f64": np.float64, "i32": np.int32, "u32": np.uint32, "i64": np.int64}


@pytest.fixture(scope="module")
def parse_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "parse_check")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-Wall", "-Werror", "-o", exe,
                           os.path.join(ROOT, "tests", "cpp", "parse_check.cpp"), "-L" + PKG, "-ldgsw_rkdg",
                           "-Wl,-rpath," + PKG])
    return exe


def read_input(exe, path, dump):
    """Parse a .15 file and its mesh with the C++ readers; returns (printed values, MeshArrays, ProblemConfig)."""
    os.makedirs(dump, exist_ok=True)
    r = subprocess.run([exe, path, dump], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = dict(line.partition(" ")[::2] for line in r.stdout.splitlines())
    arrays = {}
    for line in open(os.path.join(dump, "arrays.txt")):
        name, typ, n = line.split()
        a = np.fromfile(os.path.join(dump, name + ".bin"), dtype=DTYPES[typ])
        assert a.size == int(n)
        arrays[name] = a
    forcing = []
    b = 0
    while "forcing%d_type" % b in arrays:
        g = lambda k: arrays["forcing%d_%s" % (b, k)]  # noqa: E731
        nn, nc = g("nodes").size, g("frequency").size
        forcing.append(ForcingBlock(int(g("type")[0]), g("nodes"), g("frequency"), g("forcing_fact"), g("equilib_arg"),
                                    g("amplitude").reshape(nc, nn), g("phase").reshape(nc, nn)))
        b += 1
    lev = arrays["levee_nodes"]
    mesh = MeshArrays(node_xyz=arrays["node_xyz"].reshape(-1, 3), elem_nodes=arrays["elem_nodes"].reshape(-1, 3),
                      seg_type=arrays["seg_type"], seg_offsets=arrays["seg_offsets"], seg_nodes=arrays["seg_nodes"],
                      elem_ids=arrays["elem_ids"], name=out["mesh_name"],
                      node_manning_n=arrays["node_manning_n"] if arrays["node_manning_n"].size else None,
                      forcing=forcing, levee_pairs=lev.reshape(-1, 2) if lev.size else None,
                      levee_data=arrays["levee_data"].reshape(-1, 3) if lev.size else None)
    ic = tuple(float(x) for x in out["ic_const"].split())
    bf, cf = out["bottom_friction"].split()
    cfg = ProblemConfig(p=int(out["p"]), rk_nstages=int(out["nstages"]), rk_order=int(out["order"]), dt=float(out["dt"]),
                        g=float(out["g"]), wetting_drying=out["wetting_drying"] == "1", h_o=float(out["h_o"]),
                        slope_limiting=out["slope_limiting"] == "1", sl_M=float(out["sl_M"]), sl_nu=float(out["sl_nu"]),
                        function_source=out["function_source"] == "1", ic_type=int(out["ic_type"]), ic_const=ic,
                        bottom_friction=int(bf), friction_cf=float(cf), ramp_duration=float(out["ramp_duration"]))
    return out, mesh, cfg


def plain_fort14(path):
    """The node and element tables of a fort.14 read with nothing but split(): (name, nodes {id: xyz},
    elements {id: node ids})."""
    lines = open(path).read().split("\n")
    ne, nn = (int(x) for x in lines[1].split()[:2])
    nodes = {int(l.split()[0]): [float(x) for x in l.split()[1:4]] for l in lines[2:2 + nn]}
    elems = {int(l.split()[0]): [int(x) for x in l.split()[2:5]] for l in lines[2 + nn:2 + nn + ne]}
    return lines[0].split()[0], nodes, elems


def minimal_15(mesh_file):
    return ("mesh:\n  format: Adcirc\n  file_name: %s\n  coordinate_system: cartesian\n\n"
            "timestepping:\n  start_time: 01-01-2000 00:00:00\n  end_time: 01-01-2000 00:00:10\n  dt: 1.0\n"
            "  order: 2\n  nstages: 2\n\npolynomial_order: 1\n\nproblem:\n  name: rkdg_swe\n" % mesh_file)


def test_sample_fort14_metadata_and_topology(parse_check, oracle, tmp_path):
    """The mesh-metadata fixture: the C++ reader gives the file's name, nodes and elements (against a
    plain split() of the file), and the integer topology (neighbours, face types, interface pairing and
    order, boundary order) of the library equals the oracle's bit for bit. The file has one open
    boundary (5 nodes) and one land boundary (55 nodes); the open boundary gets a one-constituent tide
    block, which create_boundaries needs and the metadata does not depend on."""
    shutil.copy(os.path.join(INPUTS, "sample_fort.14"), tmp_path / "sample_fort.14")
    (tmp_path / "input.15").write_text(minimal_15("sample_fort.14"))
    out, mesh, _ = read_input(parse_check, str(tmp_path / "input.15"), str(tmp_path / "dump"))
    name, nodes, elems = plain_fort14(os.path.join(INPUTS, "sample_fort.14"))
    assert out["mesh_name"] == name == "ADCIRC" and mesh.name == name
    assert mesh.n_nodes == len(nodes) == 130 and mesh.n_elems == len(elems) == 200
    ids = sorted(nodes)
    for k, nid in enumerate(ids):
        assert list(mesh.node_xyz[k]) == nodes[nid]
    assert list(mesh.elem_ids) == sorted(elems)
    for k, eid in enumerate(sorted(elems)):
        assert [ids[i] for i in mesh.elem_nodes[k]] == elems[eid]
    open_nodes = mesh.seg_nodes[mesh.seg_offsets[0]:mesh.seg_offsets[1]]
    assert mesh.seg_type[0] == TIDE and len(open_nodes) == 5
    n = len(open_nodes)
    mesh.forcing = [ForcingBlock(TIDE, open_nodes, np.array([1.405189e-4]), np.array([1.0]), np.array([0.0]),
                                 np.full((1, n), 0.1), np.zeros((1, n)))]
    a = mesh_topology(mesh)
    b = oracle.problem(ProblemConfig(p=1), mesh).topology()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    nbr, bt, intf, bnd = a
    # every face is an interface side or a boundary: 3 x 200 faces = 2 interfaces sides + boundaries
    assert 2 * len(intf) + len(bnd) == 3 * mesh.n_elems
    assert int((nbr >= 0).sum()) == 2 * len(intf)
    assert out["n_interfaces"] == str(len(intf)) and out["n_boundaries"] == str(len(bnd))


def test_weir_inputs_and_topology(parse_check, oracle, tmp_path):
    """The weir case as the reference ships it: its .15 keys, the levee chain and the .bcis flow and
    levee lines come through the C++ readers, and the library's integer topology equals the oracle's."""
    out, mesh, cfg = read_input(parse_check, os.path.join(INPUTS, "weir", "dgswemv2_input.15"), str(tmp_path / "dump"))
    assert (cfg.p, cfg.rk_nstages, cfg.rk_order, cfg.dt) == (1, 2, 2, 3.0)
    assert cfg.slope_limiting and (cfg.sl_M, cfg.sl_nu) == (1.0e-8, 1.5) and not cfg.wetting_drying
    assert float(out["run_time"]) == 7200.0
    assert mesh.n_elems == 900 and mesh.n_nodes == 513
    assert len(mesh.forcing) == 1 and len(mesh.forcing[0].nodes) == 19 and len(mesh.forcing[0].frequency) == 2
    assert len(mesh.levee_pairs) == 19
    a = mesh_topology(mesh)
    b = oracle.problem(cfg, mesh).topology()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    nbr, bt, intf, bnd = a
    assert int((bt == 129).sum()) == 2 * 18  # 18 levee faces on each side of the barrier


@pytest.mark.gpu
def test_weir_case_runs_like_the_oracle(parse_check, oracle, tmp_path):
    """The whole weir case (2,400 steps of SSP-RK2 with the limiter, levee overtopping driven by the
    flow boundary) on the GPU in FP64 against the oracle; then dgswemv2-b200-serial on the same .15
    file (with a modal output block appended) writes the Python API's final state."""
    d = str(tmp_path)
    for f in ("dgswemv2_input.15", "weir.14", "weir.bcis"):
        shutil.copy(os.path.join(INPUTS, "weir", f), os.path.join(d, f))
    out, mesh, cfg = read_input(parse_check, os.path.join(d, "dgswemv2_input.15"), os.path.join(d, "dump"))
    nsteps = int(round(float(out["run_time"]) / cfg.dt))
    assert nsteps == 2400
    P = Problem(cfg, mesh)
    O = oracle.problem(cfg, mesh, n_threads=8)
    P.step_serial(nsteps)
    O.step(nsteps)
    qg, qo = P.get_state(), O.get_state()
    for v in range(3):
        scale = max(np.abs(qo[:, v]).max(), 1e-300)
        assert np.abs(qg[:, v] - qo[:, v]).max() <= 1e-9 * scale, v
    assert np.abs(qo[:, 1]).max() > 0.0  # the flow boundary has moved water
    assert np.mean(P.get_limited() != O.limited_flags()) <= 0.005
    # the serial driver on the same input
    with open(os.path.join(d, "dgswemv2_input.15"), "a") as f:
        f.write("\n\noutput:\n  path: out/\n  modal:\n    frequency: 7200\n")
    os.makedirs(os.path.join(d, "out"), exist_ok=True)
    r = subprocess.run([CLI, os.path.join(d, "dgswemv2_input.15")], capture_output=True, text=True, timeout=300, cwd=d)
    assert r.returncode == 0, r.stdout + r.stderr
    assert re.search(r"Time Elapsed \(in us\)", r.stdout)
    lines = [l for l in open(os.path.join(d, "out", mesh.name + "_modal_ze.txt")).read().split("\n") if l]
    block = lines[-(mesh.n_elems * P.nd + 1):]
    assert float(block[0]) == 7200.0
    ze = np.array([float(l.split()[1]) for l in block[1:]]).reshape(mesh.n_elems, P.nd)
    assert np.allclose(ze, qg[:, 0, :], rtol=2e-6, atol=1e-6 * np.abs(qg[:, 0, :]).max())
