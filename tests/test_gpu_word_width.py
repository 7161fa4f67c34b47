"""4-byte elements on a pitch that is a multiple of 8 bytes but not of 16 (row
lengths of 2 mod 4): the gather kernels move them in 8-byte words.  Every
plan that runs the row and column gathers, both orientations, coprime and
non-coprime shapes, tall (cluster) and short (single-CTA) strips, and a base
pointer 8 bytes off a 16-byte boundary.  Bit-exact against the oracle."""
import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu

SHAPES = [(7918, 6150, 1), (6150, 7918, 1), (1002, 334, 3), (334, 1002, 2), (30, 1002, 4), (1002, 30, 4),
          (2, 9002, 3), (9002, 6, 2), (4098, 4094, 1), (98, 34, 5)]


@pytest.mark.parametrize("offset", (0, 8))
@pytest.mark.parametrize("plan", ("c2r", "r2c", "skinny", "auto"))
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_eight_byte_words(cuda, oracle, t213, shape, plan, offset):
    d1, d2, d3 = shape
    eb = 4
    if plan == "skinny" and min(d1, d2) > 32:
        pytest.skip("skinny plans need a side of at most 32")
    x = oracle.random_bits(d1 * d2 * d3, eb, d1 * 3 + d2)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    guard = np.full(offset + 32, 0x3C, np.uint8)
    dev = to_device(cuda, np.concatenate([guard, x.view(np.uint8), guard[:32]]))
    view = dev[guard.size:guard.size + x.nbytes]
    t213.transpose_with_plan(view, d1, d2, d3, plan, elem_bytes=eb)
    cuda.cuda.synchronize()
    got = from_device(view)
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, f"{shape} {plan}: {bad.size} bytes differ, first at byte {bad[0]}"
    assert (from_device(dev[:guard.size]) == 0x3C).all()
    assert (from_device(dev[guard.size + x.nbytes:]) == 0x3C).all()


def test_describe_shows_eight_byte_words(t213):
    assert "aw=8" in t213.describe(1002, 334, 3, 4, "c2r")
