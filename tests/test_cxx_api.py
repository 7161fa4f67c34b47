"""The reference-compatible C++ interface, compiled and called the way a
reference caller does it.

tests/cxx/detail_api.cu includes this project's transpose.h and the
compatibility headers (rotate.h, shuffle.h, col_shuffle.h, permute.h,
skinny.h, equations.h), constructs the reference's functors with the
reference's constructor signatures, calls inplace::transpose / c2r / r2c,
the skinny transposes and detail::rotate / shuffle_fn / col_shuffle_fn /
scatter_permute on managed memory, and links lib/libinplacett.a.  CPU: the
program compiles and links.  GPU: every call's bytes equal the oracle's
restatement of the same reference function (include/equations.h,
include/skinny.h, src/transpose.cu, src/skinny.cu)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "detail_api.cu")
STATIC = os.path.join(ROOT, "lib", "libinplacett.a")

TYPES = {"int": 4, "longlong": 8, "float": 4, "double": 8, "int4": 16, "float4": 16, "longlong2": 16,
         "double2": 16}


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    pytest.skip("nvcc not found")


@pytest.fixture(scope="module")
def detail_api(tmp_path_factory):
    if not os.path.exists(STATIC):
        pytest.fail("lib/libinplacett.a is missing: run 213transpose_b200/build.py")
    exe = str(tmp_path_factory.mktemp("cxx") / "detail_api")
    cmd = [_nvcc(), "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe, "-L" + os.path.join(ROOT, "lib"), "-linplacett"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_reference_caller_compiles_and_links(detail_api):
    assert os.access(detail_api, os.X_OK)


def _c2r_k(oracle, m, n):
    c, t = oracle.ext_gcd(m, n)
    return c, (oracle.ext_gcd(m // c, n // c)[1] if c > 1 else t)


def _r2c_q(oracle, m, n):
    c, t = oracle.ext_gcd(n, m)
    return c, (oracle.ext_gcd(n // c, m // c)[1] if c > 1 else t)


def _cases(oracle):
    m, n = 96, 144  # rows (d2), columns (d1): c = 48, a = 2, b = 3
    c, k = _c2r_k(oracle, m, n)
    _, q = _r2c_q(oracle, m, n)
    a, b = m // c, n // c
    O = oracle
    detail = [
        ("rotate", "c2r_prerotator", [b], O.FN_C2R_PREROTATOR, [b]),
        ("rotate", "c2r_postrotator", [m], O.FN_C2R_POSTROTATOR, [m]),
        ("rotate", "r2c_prerotator", [m], O.FN_R2C_PREROTATOR, [m]),
        ("rotate", "r2c_postrotator", [b, m], O.FN_R2C_POSTROTATOR, [b, m]),
        ("shuffle", "c2r_shuffle", [m, n, c, k], O.FN_C2R_SHUFFLE, [m, n, c, k]),
        ("shuffle", "c2r_long_shuffle", [m, n, c, k], O.FN_C2R_LONG_SHUFFLE, [m, n, c, k]),
        ("shuffle", "r2c_shuffle", [m, n, c, q], O.FN_R2C_SHUFFLE, [m, n, c, q]),
        ("col_shuffle", "c2r_fused_preop", [m, b], O.FN_C2R_FUSED_PREOP, [m, b]),
        ("col_shuffle", "c2r_fused_postop", [m, n, c], O.FN_C2R_FUSED_POSTOP, [m, n, c]),
        ("col_shuffle", "r2c_fused_preop", [a, c, m, q], O.FN_R2C_FUSED_PREOP, [a, c, m, q]),
        ("col_shuffle", "r2c_fused_postop", [m, b], O.FN_R2C_FUSED_POSTOP, [m, b]),
        ("scatter_permute", "c2r_scatter_postpermuter", [m, n, c], O.FN_R2C_PREPERMUTER, [m, n, c]),
        ("scatter_permute", "r2c_scatter_prepermuter", [m, n, c], O.FN_C2R_POSTPERMUTER, [m, n, c]),
    ]
    out = []
    for i, (call, fname, args, kind, prm) in enumerate(detail):
        typ = ["float", "double", "int4", "int", "longlong2"][i % 5]
        out.append((f"{call}-{fname}-{typ}", call, typ, (n, m, 2), [fname] + args, (kind, prm)))
    whole = [
        ("transpose", "float", (512, 384, 2)), ("transpose", "double", (37, 1000, 2)),
        ("transpose", "int4", (300, 200, 1)), ("transpose", "longlong", (7, 5000, 3)),
        ("transpose", "float4", (64, 48, 2)), ("transpose", "double2", (33, 40, 2)),
        ("c2r", "float", (512, 384, 2)), ("c2r", "int", (1000, 37, 1)),
        ("r2c", "double", (600, 200, 2)), ("r2c", "int4", (97, 31, 2)),
        ("skinny_c2r", "int", (1000, 20, 2)), ("skinny_c2r", "double", (999, 32, 1)),
        ("skinny_r2c", "float4", (1000, 16, 1)), ("skinny_r2c", "float", (4096, 3, 3)),
    ]
    for call, typ, shape in whole:
        out.append((f"{call}-{typ}-{'x'.join(map(str, shape))}", call, typ, shape, [], None))
    return out


def _expected(oracle, call, shape, eb, x, fn):
    d1, d2, d3 = shape
    y = x.copy()
    if call == "transpose":
        oracle.transpose(y, d1, d2, d3, eb)
        assert np.array_equal(y, oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8))
    elif call == "c2r":
        oracle.c2r(y, d1, d2, d3, eb)
    elif call == "r2c":
        oracle.r2c(y, d1, d2, d3, eb)
    elif call == "skinny_c2r":
        oracle.skinny_c2r(y, d1, d2, d3, eb)
    elif call == "skinny_r2c":
        oracle.skinny_r2c(y, d1, d2, d3, eb)
    else:
        kind, prm = fn
        {"rotate": oracle.rotate, "shuffle": oracle.row_shuffle, "col_shuffle": oracle.col_shuffle,
         "scatter_permute": oracle.scatter_permute}[call](kind, prm, y, d3, d2, d1, eb)
    return y


@pytest.mark.gpu
def test_reference_calls_match_the_oracle(detail_api, oracle, cuda, tmp_path):
    for i, (name, call, typ, shape, extra, fn) in enumerate(_cases(oracle)):
        d1, d2, d3 = shape
        eb = TYPES[typ]
        x = oracle.random_bits(d1 * d2 * d3, eb, 300 + i)
        fin, fout = tmp_path / f"{i}.in", tmp_path / f"{i}.out"
        x.tofile(fin)
        r = subprocess.run([detail_api, call, typ, str(d1), str(d2), str(d3), str(fin), str(fout)]
                           + [str(v) for v in extra], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, (name, r.stderr)
        got = np.fromfile(fout, dtype=np.uint8)
        want = _expected(oracle, call, shape, eb, x, fn)
        assert np.array_equal(got, want), name
