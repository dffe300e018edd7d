"""C-ABI checks that need no GPU: the library builds for sm_100a, loads,
exports every entry point declared in include/*.h, and agrees with the
Python mirrors of cosa_params and cosa_run_opts on their sizes."""
import ctypes as C
import os
import re

from cosa_b200 import build, gpu
from cosa_b200.params import CosaParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(headers=None):
    inc = os.path.join(ROOT, "include")
    names = set()
    for h in headers or sorted(f for f in os.listdir(inc) if f.endswith(".h")):
        src = open(os.path.join(inc, h)).read()
        names |= set(re.findall(r"\b(cosa_(?:gpu|serve|io)_\w+)\s*\(", src))
    return sorted(names)


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    lib = C.CDLL(path)
    for name in _declared():
        assert hasattr(lib, name), name


def test_python_symbol_list_matches_header():
    from cosa_b200 import casefiles
    assert sorted(gpu.SYMBOLS) == _declared(["cosa_gpu.h"])
    assert sorted(casefiles.SYMBOLS) == _declared(["cosa_io.h"])


def test_run_opts_struct_layout():
    """cosa_run_opts: the Python mirror's size is the C struct's (16 int32,
    9 doubles, two 16-byte strings, 8 + 512 int32)."""
    from cosa_b200.casefiles import RunOpts
    assert C.sizeof(RunOpts) == 4 * 16 + 8 * 9 + 32 + 4 * (8 + 8 * 64)


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
