"""C-ABI checks that need no GPU: the library builds for sm_100a, loads,
exports every entry point declared in include/cosa_gpu.h, and agrees with the
Python mirror of cosa_params on its size."""
import ctypes as C
import os
import re

from cosa_b200 import build, gpu
from cosa_b200.params import CosaParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "cosa_gpu.h")).read()
    return sorted(set(re.findall(r"\b(cosa_(?:gpu|serve)_\w+)\s*\(", src)))


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    lib = C.CDLL(path)
    for name in _declared():
        assert hasattr(lib, name), name


def test_python_symbol_list_matches_header():
    assert sorted(gpu.SYMBOLS) == _declared()


def test_params_struct_size():
    lib = gpu.load()
    assert lib.cosa_gpu_params_size() == C.sizeof(CosaParams)


def test_init_without_gpu_fails_cleanly():
    """On a host with no GPU cosa_gpu_init returns an error code, never a
    silent CPU path."""
    import torch
    if torch.cuda.is_available():
        return
    from cosa_b200 import cases
    case = cases.bump_channel(8, 4, 2)
    try:
        gpu.Context([case.tables], case.params)
    except gpu.CosaError as e:
        assert e.code & 0x20
    else:
        raise AssertionError("init succeeded without a GPU")
