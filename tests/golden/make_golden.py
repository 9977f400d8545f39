"""Extract the known-answer vectors of the reference's unit tests into JSON fixtures.

Run where a checkout of the reference is available, giving its path; the fixtures are committed so
the tests never read the reference at run time.

    python tests/golden/make_golden.py /path/to/dgswemv2

Sources (paths inside the reference project):
  test/test_llf_flux.cpp:66-171            three LLF configurations and their expected fluxes
  test/test_basis_dubiner_2d.cpp:4-1612    phi and grad phi of 66 Dubiner modes at 15 points
  test/test_element_triangle.hpp:17-63     IntegrationPhi / IntegrationDPhi on an equilateral triangle
  test/test_element_triangle.cpp:1-48      the triangle and the integrand (x+1)^2 + (y-1)^2
  test/test_wetting_drying.cpp:15-380      five single-element wetting/drying cases
The numbers are read from the files; nothing here re-types them.

Input files the reference's tests and correctness scripts run, copied byte for byte into
tests/golden/reference_inputs/:
  test/files_for_testing/sample_fort.14              the mesh of test/test_mesh_metadata.cpp:26-45
  test/files_for_testing/weir/{dgswemv2_input.15, weir.14, weir.bcis}
                                                     the RKDG levee / flow / limiter case of
                                                     scripts/correctness/test_rkdg_parallel_weirs.sh
"""
import json
import math
import os
import re
import sys

REF = None  # the reference checkout, from the command line
OUT = os.path.dirname(os.path.abspath(__file__))

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def cexpr(expr, env=None):
    """Evaluate a small C++ arithmetic expression from the test sources."""
    e = expr.strip()
    e = e.replace("std::sqrt", "math.sqrt").replace("(double)", "float")
    e = e.replace("SWE::PostProcessing::h_o", "h_o")
    e = re.sub(r"wd_state\.bath_at_vrtx\[(\w+)\]", r"bath[\1]", e)
    e = re.sub(r"(\d)\.(?=\s*[/*+\-),])", r"\1.0", e)
    return eval(e, {"math": math, "float": float}, env or {})


def brace_block(text, start):
    """Return the text between the '{' at/after start and its matching '}'."""
    i = text.index("{", start)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i + 1 : j]
    raise ValueError("unbalanced braces")


def llf():
    src = read("test/test_llf_flux.cpp")
    cases = []
    for m in re.finditer(r"\{\s*// Configuration (\d+)", src):
        blk = brace_block(src, m.start())
        vals = {}
        for name in ["ze_in", "ze_ex", "qx_in", "qx_ex", "qy_in", "qy_ex", "bath", "sp"]:
            vals[name] = float(re.search(r"double\s+%s\s*=\s*(%s)\s*;" % (name, NUM), blk).group(1))
        nrm = re.search(r"normal\{([^}]*)\}", blk).group(1)
        nx, ny = [cexpr(x) for x in nrm.split(",")]
        call = blk[blk.index("test_configuration(") :]
        nums = re.findall(NUM, call.split("normal,")[1])
        cases.append(
            {
                "config": int(m.group(1)),
                "q_in": [vals["ze_in"], vals["qx_in"], vals["qy_in"]],
                "q_ex": [vals["ze_ex"], vals["qx_ex"], vals["qy_ex"]],
                "bath": vals["bath"],
                "sp": vals["sp"],
                "normal": [nx, ny],
                "F_expected": [float(x) for x in nums[:3]],
            }
        )
    g = float(re.search(r"almost_equal\(SWE::Global::g,\s*(%s)\)" % NUM, src).group(1))
    return {"source": "test/test_llf_flux.cpp", "gravity": g, "tolerance_factor": 100, "cases": cases}


def table(src, name):
    i = src.index(name)
    blk = brace_block(src, i)
    rows = []
    for r in re.finditer(r"\{([^{}]*)\}", blk):
        rows.append([float(x) for x in re.findall(NUM, r.group(1))])
    if not rows:
        rows = [float(x) for x in re.findall(NUM, blk)]
    return rows


def dubiner():
    src = read("test/test_basis_dubiner_2d.cpp")
    vals = table(src, "true_vals =")
    dvals = table(src, "true_Dvals =")
    pts = {}
    for m in re.finditer(r"points\[(\d+)\]\[(\d)\]\s*=\s*(%s);" % NUM, src):
        pts.setdefault(int(m.group(1)), [0.0, 0.0])[int(m.group(2))] = float(m.group(3))
    points = [pts[i] for i in sorted(pts)]
    p = int(re.search(r"GetPhi\((\d+),\s*points\)", src).group(1))
    return {
        "source": "test/test_basis_dubiner_2d.cpp",
        "p": p,
        "points": points,
        "phi": vals,
        "dphi": dvals,  # per dof: [d/dz1 pt0, d/dz2 pt0, d/dz1 pt1, ...]
        "phi_tolerance_factor": 100,
        "dphi_tolerance_factor": 1000,
    }


def element():
    hdr = read("test/test_element_triangle.hpp")
    src = read("test/test_element_triangle.cpp")
    out = {"source": "test/test_element_triangle.hpp", "tolerance_factor": 1.0e4}
    for key in ["IntegrationPhi_true", "IntegrationDPhiDX_true", "IntegrationDPhiDY_true"]:
        out[key] = table(hdr, key + " =")
    verts = []
    for m in re.finditer(r"vrtxs\[(\d)\]\s*=\s*\{([^}]*)\};", src):
        verts.append([cexpr(x) for x in m.group(2).split(",")][:2])
    out["vertices"] = verts[:3]
    out["p"] = int(re.search(r"MasterType master\((\d+)\)", src).group(1))
    # integrand f = (x + 1)^2 + (y - 1)^2 as polynomial terms c * x^i * y^j
    assert "std::pow(x(0, gp) + 1., 2) + std::pow(y(0, gp) - 1., 2)" in src
    out["f_terms"] = [[1.0, 2, 0], [2.0, 1, 0], [1.0, 0, 0], [1.0, 0, 2], [-2.0, 0, 1], [1.0, 0, 0]]
    return out


def wet_dry():
    src = read("test/test_wetting_drying.cpp")
    h_o = float(re.search(r"SWE::PostProcessing::h_o\s*=\s*(%s);" % NUM, src).group(1))
    bath = [float(m.group(2)) for m in re.finditer(r"wd_state\.bath_at_vrtx\[(\d)\]\s*=\s*(%s);" % NUM, src)]
    bath_min = float(re.search(r"wd_state\.bath_min\s*=\s*(%s);" % NUM, src).group(1))
    verts = [[cexpr(x) for x in m.group(2).split(",")][:2] for m in re.finditer(r"vrtxs\[(\d)\]\s*=\s*\{([^}]*)\};", src)]
    # split into the five cases at the comment headers
    heads = list(re.finditer(r"//\s*(Completely dry element|Completely wet element|Dry element on average|"
                             r"Some nodes dry element of flood-type|Some nodes dry element of dam-break-type)", src))
    env = {"h_o": h_o, "bath": bath}
    cases = []
    wet = True  # default of SWE::WetDry::wet
    for k, h in enumerate(heads):
        blk = src[h.end() : heads[k + 1].start() if k + 1 < len(heads) else len(src)]
        if re.search(r"wd_state\.wet\s*=\s*false", blk):
            wet = False
        q = [[0.0] * 3 for _ in range(3)]
        for m in re.finditer(r"wd_state\.q_at_vrtx\(SWE::Variables::(ze|qx|qy),\s*(\d)\)\s*=\s*([^;]+);", blk):
            q["ze qx qy".split().index(m.group(1))][int(m.group(2))] = cexpr(m.group(3), env)
        expect_wet = None
        mw = re.search(r"if \((!?)wd_state\.wet\) \{", blk)
        if mw:
            expect_wet = mw.group(1) == "!"
        checks = []
        for m in re.finditer(
            r"almost_equal\(\s*wd_state\.q_at_vrtx\(SWE::Variables::(ze|qx|qy),\s*(\w+)\),\s*([^;]*?)(?:,\s*(%s))?\)\)"
            % NUM,
            blk,
        ):
            checks.append({"var": m.group(1), "vrtx": m.group(2), "expr": m.group(3).strip(), "tol": m.group(4)})
        # expand to numbers; h_avg is the mean of the element's vertex depths as the test computes it
        hv = [q[0][i] + bath[i] for i in range(3)]
        expected = {}
        for c in checks:
            idx = range(3) if c["vrtx"] == "vrtx" else [int(c["vrtx"])]
            for i in idx:
                val = cexpr(c["expr"], dict(env, vrtx=i, h_avg=sum(hv) / 3.0))
                expected["%s%d" % (c["var"], i)] = [val, float(c["tol"]) if c["tol"] else 100.0]
        cases.append({"name": h.group(1), "wet_in": wet, "q_vrtx_in": q, "expect_wet": expect_wet, "expected": expected})
        if expect_wet is not None:
            wet = expect_wet
    return {"source": "test/test_wetting_drying.cpp", "h_o": h_o, "bath_vrtx": bath, "bath_min": bath_min,
            "vertices": verts[:3], "cases": cases}


INPUT_FILES = [
    ("test/files_for_testing/sample_fort.14", "sample_fort.14"),
    ("test/files_for_testing/weir/dgswemv2_input.15", "weir/dgswemv2_input.15"),
    ("test/files_for_testing/weir/weir.14", "weir/weir.14"),
    ("test/files_for_testing/weir/weir.bcis", "weir/weir.bcis"),
]


def copy_inputs():
    for src, dst in INPUT_FILES:
        out = os.path.join(OUT, "reference_inputs", dst)
        os.makedirs(os.path.dirname(out), exist_ok=True)
        with open(os.path.join(REF, src), "rb") as f, open(out, "wb") as g:
            g.write(f.read())
        print("copied", dst)


def main():
    global REF
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/dgswemv2")
    REF = sys.argv[1]
    fixtures = {"llf_flux.json": llf(), "dubiner_2d.json": dubiner(), "element_triangle.json": element(),
                "wetting_drying.json": wet_dry()}
    for name, data in fixtures.items():
        with open(os.path.join(OUT, name), "w") as f:
            json.dump(data, f, indent=1)
        print("wrote", name)
    copy_inputs()


if __name__ == "__main__":
    main()
