"""Parity with the reference's own GPU output.

The reference's library (src/*.cu compiled unmodified for sm_100a by
oracle/Makefile into oracle/_ref/libref_inplace.so) runs in a child process
(tests/ref_gpu_child.py) on the same seeded inputs as this project's
``t213_transpose``.  Three kinds of cases:

* Shapes on which the reference is correct: its bytes equal ours and the
  gather oracle's.  These are the large fp32/int32 configuration
  (8192, 6144, 4), int32 (3, 2^22, 8) and a skinny fp32 (32, 2^22, 1).
* A seeded sweep of C2R, R2C and skinny shapes of all four of the
  reference's element types: the reference's bytes equal the oracle's
  restatement of its pass sequence with its two bugs switched on, and where
  that restatement gives the right answer, they equal ours.
* The documented divergences of the reference: its bytes equal the oracle run
  with the reference's bugs switched on, and differ from the gather answer.
  (1) c2r::col_op passes d2/c where fused_postop needs c (src/transpose.cu:22):
  fp32 (512, 384, 16), the first configuration, and (2^20, 48, 1).  (2) The
  8-byte register row shuffles launch without a slice offset
  (src/shuffle.cu:40-49): fp64 (6500, 6151, 2), and the R2C form int64
  (300, 6500, 2), both on the R = 18 variant (rows of 6144 to 6917
  elements).
* A shape the reference cannot run on sm_100a: rows of 6918 to 29695 8-byte
  elements take register_row_shuffle<T, F, 57> with 512 threads
  (src/shuffle.cu:44-48), which needs more registers than an SM has for that
  block, so the launch is refused (cudaErrorLaunchOutOfResources) and the
  reference's error check ends its process.  This is fp64 (7919, 6151, 2),
  the coprime large configuration.  The refusal is host-side; nothing runs.

Shapes are chosen so that the reference stays in bounds and its barriers stay
uniform: every dimension that a column kernel strides over in 32-wide groups
is a multiple of 32 except on the kernels that give each slice its own CTA,
and no shape reaches the 32-bit wrap of c2r::shuffle (include/equations.h:49),
which needs n / gcd(m, n) above 46341.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import from_device, to_device
import ref_gpu_child as child

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BUGS = 1 | 2  # oracle flags: REF_POSTOP_BUG | REF_REG8_BUG


def _sweep():
    rng = np.random.default_rng(2024)
    types = list(child.CODES)
    cases = []
    for i in range(24):  # C2R and R2C shapes, both dimensions multiples of 32
        d1 = 32 * int(rng.integers(2, 65))
        d2 = 32 * int(rng.integers(2, 65))
        cases.append((f"sweep{i}", d1, d2, int(rng.integers(1, 4)), types[i % 4], "bits", 100 + i))
    for i in range(12):  # skinny: one side at most 32, the other a multiple of 32
        s = int(rng.integers(2, 33))
        l = 32 * int(rng.integers(2, 3000))
        d1, d2 = (s, l) if i % 2 else (l, s)
        cases.append((f"skinny{i}", d1, d2, int(rng.integers(1, 4)), types[(i + 1) % 4], "bits", 200 + i))
    return cases


CORRECT = [
    ("fp32_8192x6144x4", 8192, 6144, 4, "float32", "uniform", 0),
    ("int32_8192x6144x4", 8192, 6144, 4, "int32", "bits", 0),
    ("int32_3x2p22x8", 3, 1 << 22, 8, "int32", "bits", 3),
    ("fp32_32x2p22x1", 32, 1 << 22, 1, "float32", "bits", 3),
]
SWEEP = _sweep()

# name, shape, type, generator, seed, which bug, misplaced elements if known
DIVERGENT = [
    ("fp32_512x384x16", 512, 384, 16, "float32", "uniform", 0, "postop", 3_121_152),
    ("fp32_2p20x48x1", 1 << 20, 48, 1, "float32", "bits", 5, "postop", None),
    ("fp64_6500x6151x2", 6500, 6151, 2, "float64", "uniform", 0, "reg8", None),
    ("int64_300x6500x2", 300, 6500, 2, "int64", "bits", 6, "reg8", None),
]

# shapes whose reference launch is refused on sm_100a (each in a child of its own)
REFUSED = [("fp64_7919x6151x2", 7919, 6151, 2, "float64", "uniform", 0)]

SAVE_LIMIT = 64 << 20  # results up to this size come back as bytes


def _eb(typ):
    return child.CODES[typ][1]


@pytest.fixture(scope="module")
def ref_results(tmp_path_factory, cuda):
    if not os.path.exists(child.REF_GPU):
        pytest.fail("oracle/_ref/libref_inplace.so is missing: build the checker (oracle/Makefile ref-gpu)")
    tmp = tmp_path_factory.mktemp("ref_gpu")
    jobs = []
    for name, d1, d2, d3, typ, gen, seed, *rest in CORRECT + SWEEP + DIVERGENT:
        job = {"name": name, "d1": d1, "d2": d2, "d3": d3, "type": typ, "gen": gen, "seed": seed}
        if d1 * d2 * d3 * _eb(typ) <= SAVE_LIMIT:
            job["save"] = str(tmp / f"{name}.bin")
        jobs.append(job)
    jf, rf = tmp / "jobs.json", tmp / "results.json"
    jf.write_text(json.dumps(jobs))
    r = subprocess.run([sys.executable, os.path.join(HERE, "ref_gpu_child.py"), str(jf), str(rf)],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(rf.read_text())
    for job in jobs:
        if "save" in job and job["name"] in res:
            res[job["name"]]["bytes"] = np.fromfile(job["save"], dtype=np.uint8)
    return res


def _ours(cuda, t213, x, d1, d2, d3, eb):
    dev = to_device(cuda, x)
    t213.transpose(dev, d1, d2, d3, elem_bytes=eb)
    return from_device(dev)


@pytest.mark.parametrize("case", CORRECT, ids=[c[0] for c in CORRECT])
def test_reference_gpu_equals_ours(ref_results, cuda, oracle, t213, case):
    name, d1, d2, d3, typ, gen, seed = case
    eb = _eb(typ)
    r = ref_results[name]
    assert r["rc"] == 0, r
    x = child.make_input(gen, d1 * d2 * d3, eb, seed)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    got = _ours(cuda, t213, x, d1, d2, d3, eb)
    assert np.array_equal(got, want), "ours differs from the gather oracle"
    if "bytes" in r:
        assert np.array_equal(r["bytes"], got), "the reference's GPU output differs from ours"
    assert r["digest"] == child.digest(got), "the reference's GPU output differs from ours"


@pytest.mark.parametrize("case", SWEEP, ids=[c[0] for c in SWEEP])
def test_reference_gpu_sweep(ref_results, cuda, oracle, t213, case):
    name, d1, d2, d3, typ, gen, seed = case
    eb = _eb(typ)
    r = ref_results[name]
    assert r["rc"] == 0, r
    x = child.make_input(gen, d1 * d2 * d3, eb, seed)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    emulated = x.copy()
    oracle.transpose(emulated, d1, d2, d3, eb, flags=BUGS)
    assert r["digest"] == child.digest(emulated), "reference output is not its restated pass sequence"
    got = _ours(cuda, t213, x, d1, d2, d3, eb)
    assert np.array_equal(got, want), "ours differs from the gather oracle"
    if np.array_equal(emulated, want):
        assert r["digest"] == child.digest(got), "the reference's GPU output differs from ours"


@pytest.mark.parametrize("case", REFUSED, ids=[c[0] for c in REFUSED])
def test_reference_gpu_launch_refused_on_sm100(cuda, oracle, t213, tmp_path, case):
    name, d1, d2, d3, typ, gen, seed = case
    eb = _eb(typ)
    jf, rf = tmp_path / "jobs.json", tmp_path / "results.json"
    jf.write_text(json.dumps([{"name": name, "d1": d1, "d2": d2, "d3": d3, "type": typ, "gen": gen, "seed": seed}]))
    r = subprocess.run([sys.executable, os.path.join(HERE, "ref_gpu_child.py"), str(jf), str(rf)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode != 0
    assert "register 58 shuffle" in r.stderr and "too many resources requested for launch" in r.stderr, r.stderr
    # ours transposes it exactly
    x = child.make_input(gen, d1 * d2 * d3, eb, seed)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    assert np.array_equal(_ours(cuda, t213, x, d1, d2, d3, eb), want)


@pytest.mark.parametrize("case", DIVERGENT, ids=[c[0] for c in DIVERGENT])
def test_reference_gpu_divergence_is_the_documented_bug(ref_results, cuda, oracle, t213, case):
    name, d1, d2, d3, typ, gen, seed, bug, misplaced = case
    eb = _eb(typ)
    r = ref_results[name]
    assert r["rc"] == 0, r
    x = child.make_input(gen, d1 * d2 * d3, eb, seed)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    emulated = x.copy()
    oracle.transpose(emulated, d1, d2, d3, eb, flags=BUGS)
    # the bug is the whole story: the reference's bytes are the emulated ones ...
    assert r["digest"] == child.digest(emulated), f"reference output is not the emulated {bug} bug"
    # ... they are wrong ...
    wrong = int(np.count_nonzero((emulated.view(np.dtype((np.void, eb))) != want.view(np.dtype((np.void, eb))))))
    assert wrong > 0
    if misplaced is not None:
        assert wrong == misplaced
    # ... and ours is right
    got = _ours(cuda, t213, x, d1, d2, d3, eb)
    assert np.array_equal(got, want)
