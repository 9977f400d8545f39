"""The C-ABI library loads without a GPU and exports every entry point include/dgsw_rkdg.h declares."""
import os
import re

from dgswemv2_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    with open(os.path.join(ROOT, "include", "dgsw_rkdg.h")) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w]+\s*\*?\s+(dgsw_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    # the Python binding gives every declared symbol a signature
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_abi_version_and_status_strings():
    lib = _lib.load()
    assert lib.dgsw_abi_version() == 3
    assert lib.dgsw_status_string(0) == b"ok"
    assert lib.dgsw_status_string(4) == b"NaN in solution"


def test_create_without_device_fails_cleanly():
    """On a host with no CUDA device, create returns DGSW_ERR_NO_DEVICE instead of crashing."""
    import ctypes as C

    import torch

    if torch.cuda.is_available():
        return
    from dgswemv2_b200 import Problem, configs

    mesh, cfg = configs.manufactured(4)
    try:
        Problem(cfg, mesh)
        raise AssertionError("expected DgswError")
    except _lib.DgswError as e:
        assert e.status == 6
    assert C is not None


def _c_layout(header, structs, tmp_path, include_dir):
    """sizeof and field offsets of C structs, as gcc lays them out."""
    import subprocess

    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "%s"' % header, "int main(void) {"]
    for name, fields in structs.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (name, name))
        for f in fields:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (name, f, name, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-x", "c++" if header.endswith("hpp") else "c", "-I", include_dir, "-o", str(exe), str(src)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    return {k: int(v) for k, v in (l.split() for l in out if l.strip())}


def test_ctypes_structs_match_the_c_header(tmp_path):
    """The Python mirrors of dgsw_config / dgsw_mesh / dgsw_forcing_block have the C header's layout."""
    import ctypes as C

    pairs = {"dgsw_config": _lib.Config, "dgsw_mesh": _lib.Mesh, "dgsw_forcing_block": _lib.ForcingBlock}
    structs = {n: [f[0] for f in cls._fields_] for n, cls in pairs.items()}
    got = _c_layout("dgsw_rkdg.h", structs, tmp_path, os.path.join(ROOT, "include"))
    for n, cls in pairs.items():
        assert got[n] == C.sizeof(cls), n
        for f in structs[n]:
            assert got["%s.%s" % (n, f)] == getattr(cls, f).offset, (n, f)


def test_oracle_ctypes_structs_match_the_oracle_header(tmp_path):
    import ctypes as C

    from tests.oracle_ctypes import OrcConfig, OrcForcingBlock, OrcMesh

    pairs = {"orc_config": OrcConfig, "orc_mesh": OrcMesh, "orc_forcing_block": OrcForcingBlock}
    structs = {n: [f[0] for f in cls._fields_] for n, cls in pairs.items()}
    got = _c_layout("oracle.hpp", structs, tmp_path, os.path.join(ROOT, "oracle"))
    for n, cls in pairs.items():
        assert got[n] == C.sizeof(cls), n
        for f in structs[n]:
            assert got["%s.%s" % (n, f)] == getattr(cls, f).offset, (n, f)
