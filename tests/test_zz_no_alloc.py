"""t213_row_shuffle_noalloc (include/t213_noalloc.h): the row shuffle staged
through the library's fixed 32 MiB device scratch gives exactly the result of
t213_row_shuffle and of the oracle's row shuffle, call after call, and
allocates no device memory once the first call on the device has loaded the
scratch.

Collected last on purpose (the name sorts after every other test file): the
scratch is shared state of the library, and this file must pass both alone and
after everything else has run in the same process."""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCRATCH = 32 << 20


def _c2r_shuffle_params(oracle, m, n):
    c, t = oracle.ext_gcd(m, n)
    k = oracle.ext_gcd(m // c, n // c)[1] if c > 1 else t
    return (m, n, c, k)


def _r2c_shuffle_params(oracle, m, n):
    c, _ = oracle.ext_gcd(n, m)
    return (m, n, c, 0)


def _both(t213, torch, kind, prm, d3, d2, d1, eb, seed, oracle=None):
    """Runs t213_row_shuffle and the no-alloc variant on the same seeded
    bytes; with the oracle given, also checks the no-alloc result against
    the oracle's row shuffle."""
    L = t213.lib()
    nbytes = d1 * d2 * d3 * eb
    g = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    a.random_(0, 256, generator=g)
    b = a.clone()
    host = a.cpu().numpy() if oracle is not None else None
    arr = (ctypes.c_int64 * 4)(*prm)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.t213_row_shuffle(kind, arr, 4, ctypes.c_void_p(a.data_ptr()), d3, d2, d1, eb, st) == 0, \
        L.t213_last_error().decode()
    assert L.t213_row_shuffle_noalloc(kind, arr, 4, ctypes.c_void_p(b.data_ptr()), d3, d2, d1, eb, st) == 0, \
        L.t213_last_error().decode()
    torch.cuda.synchronize()
    if oracle is not None:
        oracle.row_shuffle(kind, prm, host, d3, d2, d1, eb)
        assert np.array_equal(b.cpu().numpy(), host), "no-alloc row shuffle differs from the oracle"
    return a, b


def test_matches_row_shuffle_on_two_calls_in_a_row(t213, oracle, cuda):
    import torch
    # first call: short rows, many rows per scratch group, fp32 words of 16 B
    m, n = 257, 6000
    a, b = _both(t213, torch, 10, _c2r_shuffle_params(oracle, m, n), 3, m, n, 4, seed=1, oracle=oracle)
    assert torch.equal(a, b)
    # second call right after: 24 MB rows (one row per group), 16-byte elements,
    # the R2C shuffler
    m, n = 6, 1_500_000
    a, b = _both(t213, torch, 12, _r2c_shuffle_params(oracle, m, n), 2, m, n, 16, seed=2, oracle=oracle)
    assert torch.equal(a, b)


@pytest.mark.parametrize("eb", [1, 2, 8])
def test_matches_row_shuffle_narrow_elements(t213, oracle, cuda, eb):
    import torch
    m, n = 96, 70_001  # odd row length: element-wide accesses
    a, b = _both(t213, torch, 10, _c2r_shuffle_params(oracle, m, n), 2, m, n, eb, seed=3 + eb, oracle=oracle)
    assert torch.equal(a, b)


# A fresh process: the device's free memory across the first (empty) call,
# which may load the module holding the scratch, the first real call, which
# may load its kernel's code, and the calls after them.
_FIRST_CALL = r"""
import ctypes, importlib, json, sys
import torch
sys.path.insert(0, sys.argv[1])
torch.cuda.init()
m, n = 512, 4096
x = torch.zeros(2 * m * n * 4, dtype=torch.uint8, device="cuda")
x.random_(0, 256)
torch.cuda.synchronize()
L = importlib.import_module("213transpose_b200").lib()
arr = (ctypes.c_int64 * 4)(*[int(v) for v in sys.argv[2:6]])
call = lambda d3: L.t213_row_shuffle_noalloc(10, arr, 4, ctypes.c_void_p(x.data_ptr()), d3, m, n, 4, None)
free0, _ = torch.cuda.mem_get_info()
rcs = [call(0)]
torch.cuda.synchronize()
free1, _ = torch.cuda.mem_get_info()
rcs.append(call(2))
torch.cuda.synchronize()
free2, _ = torch.cuda.mem_get_info()
rcs += [call(2) for _ in range(3)]
torch.cuda.synchronize()
free3, _ = torch.cuda.mem_get_info()
print(json.dumps({"rcs": rcs, "first": free0 - free1, "code": free1 - free2, "later": free2 - free3}))
"""


def test_first_call_reserves_the_scratch_later_calls_nothing(t213, oracle, cuda):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    prm = [str(v) for v in _c2r_shuffle_params(oracle, 512, 4096)]
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL, root] + prm, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["rcs"] == [0, 0, 0, 0, 0]
    # the empty warm-up call and the first real one take at most the scratch
    # plus the module's code; every call after them takes nothing
    assert out["first"] >= 0 and out["code"] >= 0, out
    assert out["first"] + out["code"] <= SCRATCH + (16 << 20), out
    assert out["later"] == 0, out


def test_allocates_no_device_memory(t213, oracle, cuda):
    import torch
    m, n = 512, 4096
    _both(t213, torch, 10, _c2r_shuffle_params(oracle, m, n), 2, m, n, 4, seed=9)  # set-up done
    L = t213.lib()
    x = torch.zeros(2 * m * n * 4, dtype=torch.uint8, device="cuda")
    arr = (ctypes.c_int64 * 4)(*_c2r_shuffle_params(oracle, m, n))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert L.t213_row_shuffle_noalloc(10, arr, 4, ctypes.c_void_p(x.data_ptr()), 2, m, n, 4, None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_rejects_rows_longer_than_the_scratch(t213, oracle, cuda):
    import torch
    L = t213.lib()
    m, n, eb = 2, SCRATCH // 4 + 4, 4  # one row is 16 bytes longer than the scratch
    x = torch.arange(m * n, dtype=torch.int32, device="cuda")
    before = x.clone()
    arr = (ctypes.c_int64 * 4)(*_c2r_shuffle_params(oracle, m, n))
    rc = L.t213_row_shuffle_noalloc(10, arr, 4, ctypes.c_void_p(x.data_ptr()), 1, m, n, eb, None)
    assert rc == 2  # T213_ERR_UNSUPPORTED
    assert b"32 MiB" in L.t213_last_error()
    torch.cuda.synchronize()
    assert torch.equal(x, before)
