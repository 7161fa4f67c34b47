"""B200-native in-place 213 transpose (drop-in for kaihsin/213transpose).

The package directory name starts with a digit, so import it with
``importlib.import_module("213transpose_b200")``.  The compute path is the
CUDA library built by ``213transpose_b200/build.py`` (sm_100a); importing the
API without it raises, there is no CPU fallback.
"""
from ._lib import T213Error, lib, header_functions, SO_PATH  # noqa: F401
from .api import (inplace, transpose, c2r_transpose, r2c_transpose, skinny_c2r_transpose,  # noqa: F401
                  skinny_r2c_transpose, rotate, shuffle_fn, col_shuffle_fn, scatter_permute, permute,
                  transpose_with_plan, transpose_host, describe, plan_launches, pass_timing,
                  release_cache, Batch, Server, device_status, tuner)

__all__ = ["inplace", "transpose", "c2r_transpose", "r2c_transpose", "skinny_c2r_transpose",
           "skinny_r2c_transpose", "rotate", "shuffle_fn", "col_shuffle_fn", "scatter_permute", "permute",
           "transpose_with_plan", "transpose_host", "describe", "plan_launches", "pass_timing",
           "release_cache", "Batch", "Server", "device_status", "tuner", "T213Error", "lib"]
