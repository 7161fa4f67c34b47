"""ORACLE — TEST INFRASTRUCTURE ONLY.

ctypes front end of the CPU checker for the in-place 213 transpose:

* ``liboracle213.so`` (``t213_oracle.c``): this project's C restatement of the
  reference algorithm — the out-of-place gather ``seq_tt``
  (src/tensor_util.cpp:79-92), every index functor of include/equations.h and
  include/skinny.h, and host executors of every C2R/R2C pass and driver
  (src/transpose.cu:18-124, src/skinny.cu:313-363).
* ``_ref/libref_seqtt.so`` and ``_ref/gen_ans``: the reference's own CPU answer
  generator compiled from its sources (see Makefile), used to pin the
  restatement and as the timed CPU baseline.
* ``_ref/libref_inplace.so``: the reference's own GPU library compiled for
  sm_100a, used by GPU tests only on shapes where it is correct and in bounds.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only to check or time; the product never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle213.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SEQTT = os.path.join(REF_DIR, "libref_seqtt.so")
REF_GENANS = os.path.join(REF_DIR, "gen_ans")
REF_GPU = os.path.join(REF_DIR, "libref_inplace.so")

# functor kinds, mirrored from include/t213.h (tests check they agree)
FN_C2R_PREROTATOR = 1
FN_C2R_POSTROTATOR = 2
FN_R2C_PREROTATOR = 3
FN_R2C_POSTROTATOR = 4
FN_C2R_SHUFFLE = 10
FN_C2R_LONG_SHUFFLE = 11
FN_R2C_SHUFFLE = 12
FN_C2R_FUSED_PREOP = 20
FN_C2R_FUSED_POSTOP = 21
FN_R2C_FUSED_PREOP = 22
FN_R2C_FUSED_POSTOP = 23
FN_C2R_POSTPERMUTER = 30
FN_R2C_PREPERMUTER = 31

REF_POSTOP_BUG = 1
REF_REG8_BUG = 2

_lib = None
_ref = None


def build(reference: str | None = None) -> None:
    """Compiles liboracle213.so and, when the reference's source tree is given
    (argument, or the environment's T213_REFERENCE) and present, the
    reference's CPU and GPU builds under _ref/."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    ref = reference or os.environ.get("T213_REFERENCE")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = ctypes.CDLL(LIB_PATH)
        i64, vp, ip = ctypes.c_int64, ctypes.c_void_p, ctypes.c_int
        L.t213o_seq_tt.argtypes = [vp, vp, ip, ctypes.POINTER(i64), ctypes.POINTER(i64), i64]
        L.t213o_gather213.argtypes = [vp, vp, i64, i64, i64, i64]
        L.t213o_gather213.restype = None
        L.t213o_ramp.argtypes = [vp, i64, i64]
        L.t213o_ramp.restype = None
        L.t213o_ext_gcd.argtypes = [i64, i64, ctypes.POINTER(i64)]
        L.t213o_ext_gcd.restype = i64
        L.t213o_index.argtypes = [ip, ctypes.POINTER(i64), i64, i64]
        L.t213o_index.restype = i64
        for name in ("t213o_rotate", "t213o_row_shuffle", "t213o_col_shuffle", "t213o_scatter_permute"):
            getattr(L, name).argtypes = [ip, ctypes.POINTER(i64), vp, i64, i64, i64, i64]
        for name in ("t213o_c2r", "t213o_r2c", "t213o_transpose"):
            getattr(L, name).argtypes = [vp, i64, i64, i64, i64, ip]
        for name in ("t213o_skinny_c2r", "t213o_skinny_r2c"):
            getattr(L, name).argtypes = [vp, i64, i64, i64, i64]
        L.t213o_permuter_cycles.argtypes = [ip, ctypes.POINTER(i64), i64, ctypes.POINTER(i64),
                                            ctypes.POINTER(i64)]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> ctypes.c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


def _prm(params) -> ctypes.Array:
    vals = list(params) + [0] * (4 - len(params))
    return (ctypes.c_int64 * 4)(*vals)


# ---------------------------------------------------------------- answers ---

def seq_tt(data: np.ndarray, dims, perm=(1, 0, 2)) -> np.ndarray:
    """The reference's rank-N gather restated (src/tensor_util.cpp:79-92);
    returns a new array holding the answer bytes."""
    out = np.empty_like(data)
    rank = len(dims)
    d = (ctypes.c_int64 * rank)(*dims)
    p = (ctypes.c_int64 * rank)(*perm)
    rc = lib().t213o_seq_tt(_p(out), _p(data), rank, d, p, data.itemsize)
    assert rc == 0
    return out


def gather213(data: np.ndarray, d1: int, d2: int, d3: int) -> np.ndarray:
    """The 213 answer, blocked and OpenMP-parallel (this project's code)."""
    out = np.empty_like(data)
    lib().t213o_gather213(_p(out), _p(data), d1, d2, d3, data.itemsize)
    return out


def ramp(n: int, elem_bytes: int) -> np.ndarray:
    """data[i] = i, the reference's known-answer input."""
    out = np.empty(n * elem_bytes, dtype=np.uint8)
    lib().t213o_ramp(_p(out), n, elem_bytes)
    return out


def dtype_for(elem_bytes: int):
    return {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}.get(elem_bytes)


def random_bits(n_elems: int, elem_bytes: int, seed: int) -> np.ndarray:
    """Seeded random bit patterns viewed as raw bytes (NaN-safe comparisons)."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, size=n_elems * elem_bytes, dtype=np.uint8)


def uniform_f32(n_elems: int, seed: int) -> np.ndarray:
    """uniform[-1,1) fp32 from numpy's default_rng(seed), as raw bytes."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n_elems).astype(np.float32).view(np.uint8)


def uniform_f64(n_elems: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n_elems).astype(np.float64).view(np.uint8)


# --------------------------------------------------------------- functors ---

def ext_gcd(a: int, b: int):
    mmi = ctypes.c_int64(0)
    g = lib().t213o_ext_gcd(a, b, ctypes.byref(mmi))
    return int(g), int(mmi.value)


def index(kind: int, params, i: int = 0, j: int = 0) -> int:
    return int(lib().t213o_index(kind, _prm(params), i, j))


def permuter_cycles(kind: int, params, m: int):
    nc, ml = ctypes.c_int64(0), ctypes.c_int64(0)
    rc = lib().t213o_permuter_cycles(kind, _prm(params), m, ctypes.byref(nc), ctypes.byref(ml))
    assert rc == 0
    return int(nc.value), int(ml.value)


# ----------------------------------------------------------------- passes ---
# All executors work in place on a byte buffer holding d3 slices of m x n
# elements of elem_bytes each.

def _run(name, kind, params, buf, d3, m, n, eb):
    rc = getattr(lib(), name)(kind, _prm(params), _p(buf), d3, m, n, eb)
    if rc != 0:
        raise ValueError(f"{name} failed ({rc}): index out of range or bad functor")


def rotate(kind, params, buf, d3, m, n, eb):
    _run("t213o_rotate", kind, params, buf, d3, m, n, eb)


def row_shuffle(kind, params, buf, d3, m, n, eb):
    _run("t213o_row_shuffle", kind, params, buf, d3, m, n, eb)


def col_shuffle(kind, params, buf, d3, m, n, eb):
    _run("t213o_col_shuffle", kind, params, buf, d3, m, n, eb)


def scatter_permute(kind, params, buf, d3, m, n, eb):
    _run("t213o_scatter_permute", kind, params, buf, d3, m, n, eb)


def c2r(buf, d1, d2, d3, eb, flags=0):
    assert lib().t213o_c2r(_p(buf), d1, d2, d3, eb, flags) == 0


def r2c(buf, d1, d2, d3, eb, flags=0):
    assert lib().t213o_r2c(_p(buf), d1, d2, d3, eb, flags) == 0


def skinny_c2r(buf, d1, d2, d3, eb):
    assert lib().t213o_skinny_c2r(_p(buf), d1, d2, d3, eb) == 0


def skinny_r2c(buf, d1, d2, d3, eb):
    assert lib().t213o_skinny_r2c(_p(buf), d1, d2, d3, eb) == 0


def transpose(buf, d1, d2, d3, eb, flags=0):
    """The reference's dispatcher restated (src/transpose.cu:99-124)."""
    assert lib().t213o_transpose(_p(buf), d1, d2, d3, eb, flags) == 0


# ------------------------------------------------------- reference builds ---

def ref_available() -> bool:
    return os.path.exists(REF_SEQTT)


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_SEQTT)
        L.ref_seq_tt.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int]
        L.ref_init_data.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int]
        _ref = L
    return _ref


def ref_seq_tt(data: np.ndarray, d1: int, d2: int, d3: int, elem_bytes: int) -> np.ndarray:
    """The reference's own TensorUtil::seq_tt (4- or 8-byte elements)."""
    out = np.empty_like(data)
    rc = ref_lib().ref_seq_tt(_p(out), _p(data), d1, d2, d3, elem_bytes)
    if rc != 0:
        raise ValueError("reference seq_tt supports 4- and 8-byte elements only")
    return out


def ref_seq_tt_into(out: np.ndarray, data: np.ndarray, d1, d2, d3, elem_bytes) -> None:
    rc = ref_lib().ref_seq_tt(_p(out), _p(data), d1, d2, d3, elem_bytes)
    if rc != 0:
        raise ValueError("reference seq_tt supports 4- and 8-byte elements only")
