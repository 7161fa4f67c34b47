"""The column passes of C2R and R2C (rotations and fused column shuffles) on
rows whose pitch is not a 16-byte multiple: the peeled kernel (each slot of
a strip takes the 16-byte blocks that cover the strip's bytes of one row,
output rows are written as 16-byte vectors between the row's 16-byte
boundaries and single elements at its ends) and the word-width kernel it
replaces (pinned as variant col=5), over 4- and 8-byte elements, odd and
even row lengths, whole strips in one CTA and strips split over a cluster,
the narrower last strip, and base pointers off a 16-byte boundary.  Guard
bytes on both sides of the tensor must stay as they were: the peeled kernel
reads past a strip's ends but never writes there.  Bit-exact against the
oracle."""
import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu

PLAN = {"c2r": 1, "r2c": 2}

# (d1, d2, d3): column heights from 3 to 7919 (one CTA and clusters), row
# lengths odd and 2 mod 4, gcd 1 and above
SHAPES = [(2001, 3001, 1), (3001, 2001, 2), (7919, 601, 1), (601, 7919, 1), (4001, 1502, 1), (1502, 4001, 1),
          (1001, 333, 3), (333, 1001, 2), (97, 33, 5), (30, 1003, 4), (1003, 30, 4), (5, 3, 7), (6, 1021, 2)]
GUARD = 48


def _run(cuda, oracle, t213, d1, d2, d3, eb, plan, offset, seed):
    x = oracle.random_bits(d1 * d2 * d3, eb, seed)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    head = np.full(offset + GUARD, 0xA5, np.uint8)
    tail = np.full(GUARD, 0x5A, np.uint8)
    dev = to_device(cuda, np.concatenate([head, x.view(np.uint8), tail]))
    view = dev[head.size:head.size + x.nbytes]
    t213.transpose_with_plan(view, d1, d2, d3, plan, elem_bytes=eb)
    cuda.cuda.synchronize()
    got = from_device(view)
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, f"{(d1, d2, d3, eb, plan, offset)}: {bad.size} bytes differ, first at byte {bad[0]}"
    assert (from_device(dev[:head.size]) == 0xA5).all(), "bytes before the tensor were written"
    assert (from_device(dev[head.size + x.nbytes:]) == 0x5A).all(), "bytes after the tensor were written"


@pytest.mark.parametrize("offset", (0, 4, 8, 12))
@pytest.mark.parametrize("plan", ("c2r", "r2c"))
@pytest.mark.parametrize("eb", (4, 8))
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_peeled_col_pass(cuda, oracle, t213, shape, eb, plan, offset):
    if offset % eb:
        pytest.skip("the base keeps the element alignment")
    _run(cuda, oracle, t213, *shape, eb, plan, offset, seed=sum(shape) * eb + offset)


@pytest.mark.parametrize("plan", ("c2r", "r2c"))
@pytest.mark.parametrize("eb", (4, 8))
@pytest.mark.parametrize("shape", SHAPES[:6], ids=lambda s: "x".join(map(str, s)))
def test_word_width_col_pass(cuda, oracle, t213, tmp_path, shape, eb, plan):
    d1, d2, d3 = shape
    path = tmp_path / "pinned.txt"
    path.write_text(f"shape {d1} {d2} {d3} {eb} {PLAN[plan]} 0 {5}\n")
    t213.tuner.clear()
    t213.tuner.load(path)
    try:
        desc = t213.describe(d1, d2, d3, eb)  # the automatic choice takes the pinned entry
        col = desc[desc.index("col_gather"):].split("]")[0]
        assert desc.startswith(plan) and "[variant" in desc and "local" in col and "peeled" not in col, desc
        _run(cuda, oracle, t213, d1, d2, d3, eb, "auto", 8, seed=d1 * d2 + eb)
    finally:
        t213.tuner.clear()
