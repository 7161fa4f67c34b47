"""The row passes of C2R and R2C on rows whose pitch is not a 16-byte
multiple: the peeled kernel (16-byte loads of the blocks that cover a unit,
16-byte stores between the unit's 16-byte boundaries, single elements at the
ends) and the word-width kernel it replaces (pinned as variant row=3), over
element sizes 1, 2 and 4, odd and even row lengths, coprime and non-coprime
shapes (the stepped and the re-evaluated shuffles), and base pointers off a
16-byte boundary.  Guard bytes on both sides of the tensor must stay as they
were: the peeled kernel reads past a unit's ends but never writes there.
Bit-exact against the oracle."""
import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu

PLAN = {"c2r": 1, "r2c": 2}

# (d1, d2, d3): row lengths odd and even, gcd 1 and above, long and short rows
SHAPES = [(7919, 601, 1), (601, 7919, 1), (1001, 333, 3), (333, 1001, 2), (3951, 3210, 1), (97, 33, 5),
          (30, 1003, 4), (1003, 30, 4), (5, 3, 7), (2, 9001, 3), (9001, 2, 3), (6, 1021, 2)]
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
@pytest.mark.parametrize("eb", (1, 2, 4))
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_peeled_row_pass(cuda, oracle, t213, shape, eb, plan, offset):
    if offset % eb:
        pytest.skip("the base keeps the element alignment")
    _run(cuda, oracle, t213, *shape, eb, plan, offset, seed=sum(shape) + eb)


@pytest.mark.parametrize("plan", ("c2r", "r2c"))
@pytest.mark.parametrize("eb", (1, 2, 4))
@pytest.mark.parametrize("shape", SHAPES[:6], ids=lambda s: "x".join(map(str, s)))
def test_word_width_row_pass(cuda, oracle, t213, tmp_path, shape, eb, plan):
    d1, d2, d3 = shape
    path = tmp_path / "pinned.txt"
    path.write_text(f"shape {d1} {d2} {d3} {eb} {PLAN[plan]} 0 {3 << 4}\n")
    t213.tuner.clear()
    t213.tuner.load(path)
    try:
        desc = t213.describe(d1, d2, d3, eb)  # the automatic choice takes the pinned entry
        rows = [seg for seg in desc.split("] ") if "row_gather" in seg]
        assert desc.startswith(plan) and "[variant" in desc and rows and not any("peeled" in r for r in rows), desc
        _run(cuda, oracle, t213, d1, d2, d3, eb, "auto", 4, seed=d1 * d2 + eb)
    finally:
        t213.tuner.clear()


def _row_passes(desc):
    return [seg for seg in desc.split("] ") if "row_gather" in seg]


def test_describe_names_the_peeled_kernel(t213):
    assert any("peeled" in r for r in _row_passes(t213.describe(7919, 601, 1, 4, "c2r")))
    # 8-byte elements: the row pass keeps 8-byte words (the column pass is peeled)
    assert not any("peeled" in r for r in _row_passes(t213.describe(7919, 601, 1, 8, "c2r")))
    assert "peeled" not in t213.describe(7920, 600, 1, 4, "c2r")  # 16-byte pitch: plain 16-byte words
