"""4-byte elements on a pitch that is a multiple of 8 bytes but not of 16 (row
lengths of 2 mod 4): by default the row and column gathers take their peeled
16-byte kernels there; pinned to the word-width variants (col=5, row=3) they
move the elements in 8-byte words.  Every plan that runs the row and column
gathers, both orientations, coprime and non-coprime shapes, tall (cluster)
and short (single-CTA) strips, and a base pointer 8 bytes off a 16-byte
boundary.  Bit-exact against the oracle."""
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


PLAN = {"c2r": 1, "r2c": 2}
WORD_WIDTH = 5 | 3 << 4  # variant col=5 (word-width column strips), row=3 (word-width rows)


def _pinned(t213, tmp_path, d1, d2, d3, plan):
    path = tmp_path / "pinned.txt"
    path.write_text(f"shape {d1} {d2} {d3} 4 {PLAN[plan]} 0 {WORD_WIDTH}\n")
    t213.tuner.clear()
    t213.tuner.load(path)


def test_describe_shows_eight_byte_words(t213, tmp_path):
    _pinned(t213, tmp_path, 1002, 334, 3, "c2r")
    try:
        d = t213.describe(1002, 334, 3, 4)
        assert "aw=8" in d and "peeled" not in d, d
    finally:
        t213.tuner.clear()


@pytest.mark.parametrize("offset", (0, 8))
@pytest.mark.parametrize("plan", ("c2r", "r2c"))
@pytest.mark.parametrize("shape", SHAPES[:6] + [SHAPES[8]], ids=lambda s: "x".join(map(str, s)))
def test_eight_byte_words_pinned(cuda, oracle, t213, tmp_path, shape, plan, offset):
    d1, d2, d3 = shape
    _pinned(t213, tmp_path, d1, d2, d3, plan)
    try:
        d = t213.describe(d1, d2, d3, 4)
        assert d.startswith(plan) and "aw=8" in d and "peeled" not in d, d
        x = oracle.random_bits(d1 * d2 * d3, 4, d1 * 5 + d2)
        want = oracle.gather213(x.view(np.dtype((np.void, 4))), d1, d2, d3).view(np.uint8)
        guard = np.full(offset + 32, 0x3C, np.uint8)
        dev = to_device(cuda, np.concatenate([guard, x.view(np.uint8), guard[:32]]))
        view = dev[guard.size:guard.size + x.nbytes]
        t213.transpose(view, d1, d2, d3, elem_bytes=4)
        cuda.cuda.synchronize()
        got = from_device(view)
        bad = np.flatnonzero(got != want)
        assert bad.size == 0, f"{shape} {plan}: {bad.size} bytes differ, first at byte {bad[0]}"
        assert (from_device(dev[:guard.size]) == 0x3C).all()
        assert (from_device(dev[guard.size + x.nbytes:]) == 0x3C).all()
    finally:
        t213.tuner.clear()
