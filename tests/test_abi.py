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
    assert lib.dgsw_abi_version() == 1
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
