"""Parity of the CUDA path with the oracle: every plan family, every entry
point, every element size, on seeded inputs at sizes the oracle finishes in
seconds.  Bit-exact (data movement only)."""
import random

import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu

EBS = (4, 8, 16, 1, 2)

SHAPES = [
    (7, 5, 3), (33, 40, 2), (64, 48, 4), (3, 97, 2), (100, 37, 1), (97, 3, 2), (35, 35, 1),
    (120, 300, 1), (1, 7, 2), (7, 1, 2), (64, 64, 2), (600, 45, 1), (40, 600, 1), (2, 2, 1),
    (31, 33, 3), (256, 192, 1), (512, 384, 2), (700, 450, 1), (450, 700, 1), (1000, 999, 1),
    (999, 1000, 1), (128, 4096, 1), (4096, 96, 1), (384, 512, 1), (2048, 1536, 1), (1, 1, 5),
    (0, 5, 2), (5, 0, 2), (5, 5, 0),
]


def random_shapes(n, seed, lo=1, hi=700):
    rng = random.Random(seed)
    return [(rng.randint(lo, hi), rng.randint(lo, hi), rng.randint(1, 3)) for _ in range(n)]


def check_transpose(cuda, oracle, fn, d1, d2, d3, eb, seed=0):
    x = oracle.random_bits(d1 * d2 * d3, eb, seed)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    dev = to_device(cuda, x)
    fn(dev, d1, d2, d3, elem_bytes=eb)
    cuda.cuda.synchronize()
    got = from_device(dev)
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, f"{(d1, d2, d3, eb)}: {bad.size} bytes differ, first at byte {bad[0]}"


@pytest.mark.parametrize("eb", EBS)
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_transpose_auto(cuda, oracle, t213, shape, eb):
    check_transpose(cuda, oracle, t213.transpose, *shape, eb)


@pytest.mark.parametrize("eb", (4, 8, 16))
@pytest.mark.parametrize("shape", random_shapes(24, 7), ids=lambda s: "x".join(map(str, s)))
def test_transpose_random(cuda, oracle, t213, shape, eb):
    check_transpose(cuda, oracle, t213.transpose, *shape, eb, seed=shape[0])


PLAN_SHAPES = [(64, 48, 2), (512, 384, 2), (100, 37, 1), (37, 100, 2), (600, 45, 1), (45, 600, 2),
               (1000, 999, 1), (128, 96, 3), (96, 128, 3), (4096, 30, 1), (30, 4096, 1), (300, 300, 2),
               (3000, 2000, 2), (2000, 3000, 1), (2048, 1536, 2), (6144, 32, 2), (32, 6144, 2)]


@pytest.mark.parametrize("eb", (4, 8, 16, 1))
@pytest.mark.parametrize("plan", ["c2r", "r2c", "blocks", "bands", "bands_t", "skinny", "slice"])
@pytest.mark.parametrize("shape", PLAN_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_every_plan(cuda, oracle, t213, shape, plan, eb):
    d1, d2, d3 = shape
    try:
        t213.describe(d1, d2, d3, eb, plan)
    except t213.T213Error as e:
        assert e.status == 2, e  # the family does not apply to this shape
        pytest.skip(f"{plan} does not apply")
    check_transpose(cuda, oracle,
                    lambda dev, a, b, c, elem_bytes: t213.transpose_with_plan(dev, a, b, c, plan, elem_bytes=elem_bytes),
                    d1, d2, d3, eb)


@pytest.mark.parametrize("eb", (4, 8, 16))
@pytest.mark.parametrize("shape", [(64, 48, 2), (512, 384, 2), (100, 37, 3), (1000, 999, 1), (450, 700, 1),
                                   (96, 4096, 1), (4096, 96, 1), (33, 33, 2)], ids=lambda s: "x".join(map(str, s)))
def test_c2r_r2c_entry_points(cuda, oracle, t213, shape, eb):
    """c2r::transpose(d1,d2) maps d2 x d1 to d1 x d2; r2c::transpose(d2,d1)
    does the same (the reference's dispatcher, src/transpose.cu:117-123)."""
    d1, d2, d3 = shape
    check_transpose(cuda, oracle, t213.c2r_transpose, d1, d2, d3, eb)
    check_transpose(cuda, oracle, lambda dev, a, b, c, elem_bytes: t213.r2c_transpose(dev, b, a, c, elem_bytes=elem_bytes),
                    d1, d2, d3, eb)


@pytest.mark.parametrize("eb", (4, 8, 16))
@pytest.mark.parametrize("shape", [(100, 7, 3), (4096, 32, 1), (97, 3, 2), (5000, 30, 1), (64, 2, 4)],
                         ids=lambda s: "x".join(map(str, s)))
def test_skinny_entry_points(cuda, oracle, t213, shape, eb):
    d1, d2, d3 = shape  # d2 <= 32 < d1
    check_transpose(cuda, oracle, t213.skinny_c2r_transpose, d1, d2, d3, eb)
    # r2c skinny with the reference's swapped arguments: the transposed shape
    check_transpose(cuda, oracle,
                    lambda dev, a, b, c, elem_bytes: t213.skinny_r2c_transpose(dev, b, a, c, elem_bytes=elem_bytes),
                    d2, d1, d3, eb)


def test_ramp_known_answer(cuda, oracle, t213):
    """The reference's known-answer input data[i] = i (src/tensor_util.cpp:42-47)."""
    d1, d2, d3 = 512, 384, 16
    x = oracle.ramp(d1 * d2 * d3, 4)
    want = oracle.seq_tt(x.view(np.int32), (d1, d2, d3)).view(np.uint8)
    dev = to_device(cuda, x)
    t213.transpose(dev, d1, d2, d3, elem_bytes=4)
    assert np.array_equal(from_device(dev), want)
