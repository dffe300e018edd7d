"""cosa_b200 -- B200-native (sm_100a) explicit residual-and-update path of COSA.

Layout of the package:
  csrc/      CUDA kernels and the C-ABI library source (include/cosa_gpu.h)
  lib/       the built libcosa_gpu.so (in-tree build, see build.py)
  params.py  cosa_params (module globals of the hot path) as a ctypes struct
  tables.py  block / BC / cut tables in COSA's input.dat encoding
  cases.py   synthetic grids and states of the benchmark configurations
  gpu.py     ctypes binding of the C-ABI and a single-level solver driver
"""
__all__ = ["params", "tables", "cases", "gpu", "build"]
