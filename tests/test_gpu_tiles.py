"""Parity of both square-block tile-swap kernels of the BLOCKS plan (the TMA
ring and the register-prefetch kernel) with the oracle, over ring depths and
element sizes, plus the unaligned fallback.  Bit-exact."""
import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu

# (d1, d2, d3): gcd(d1, d2) is the block side t of the BLOCKS plan
TILE_SHAPES = [(512, 384, 2), (2048, 1536, 2), (128, 96, 3), (96, 128, 3), (6144, 32, 2), (64, 64, 3),
               (48, 80, 2), (4096, 4096, 1), (1024, 3072, 1), (160, 96, 5)]


def run_blocks(cuda, oracle, t213, d1, d2, d3, eb, offset=0):
    x = oracle.random_bits(d1 * d2 * d3, eb, d1 + d2)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    dev = to_device(cuda, np.concatenate([np.zeros(offset, np.uint8), x.view(np.uint8)]))
    view = dev[offset:]
    t213.transpose_with_plan(view, d1, d2, d3, "blocks", elem_bytes=eb)
    cuda.cuda.synchronize()
    got = from_device(view)
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, f"{(d1, d2, d3, eb)}: {bad.size} bytes differ, first at byte {bad[0]}"
    assert not from_device(dev[:offset]).any(), "bytes before the tensor were written"


@pytest.mark.parametrize("kernel", ["tma", "vec"])
@pytest.mark.parametrize("eb", (4, 8, 16))
@pytest.mark.parametrize("shape", TILE_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_tile_swap_kernels(cuda, oracle, t213, monkeypatch, shape, eb, kernel):
    monkeypatch.setenv("T213_TILE_SWAP", kernel)
    run_blocks(cuda, oracle, t213, *shape, eb)


@pytest.mark.parametrize("stages", (2, 3, 5, 8, 24))
@pytest.mark.parametrize("eb", (4, 8, 16))
def test_tma_ring_depths(cuda, oracle, t213, monkeypatch, stages, eb):
    monkeypatch.setenv("T213_TILE_SWAP", "tma")
    monkeypatch.setenv("T213_TILE_STAGES", str(stages))
    run_blocks(cuda, oracle, t213, 2048, 1536, 2, eb)
    run_blocks(cuda, oracle, t213, 160, 96, 5, eb)


@pytest.mark.parametrize("warps", (1, 4, 16))
@pytest.mark.parametrize("ts", (8, 16, 32, 64))
@pytest.mark.parametrize("eb", (4, 8, 16))
def test_tma_launch_shapes(cuda, oracle, t213, monkeypatch, warps, ts, eb):
    """Consumer-warp counts and tile sides (the launcher maps a side an
    element size cannot use to its default)."""
    monkeypatch.setenv("T213_TILE_SWAP", "tma")
    monkeypatch.setenv("T213_TILE_WARPS", str(warps))
    monkeypatch.setenv("T213_TILE_TS", str(ts))
    run_blocks(cuda, oracle, t213, 2048, 1536, 2, eb)
    run_blocks(cuda, oracle, t213, 192, 128, 3, eb)


@pytest.mark.parametrize("group", (1, 2, 4, 8))
@pytest.mark.parametrize("eb", (4, 8, 16))
def test_tma_pair_orders(cuda, oracle, t213, monkeypatch, group, eb):
    """Super-tile pair orders, including tile grids the group does not
    divide (the launcher falls back to a smaller group)."""
    monkeypatch.setenv("T213_TILE_SWAP", "tma")
    monkeypatch.setenv("T213_TILE_GROUP", str(group))
    run_blocks(cuda, oracle, t213, 2048, 1536, 2, eb)
    run_blocks(cuda, oracle, t213, 192 * 3, 192 * 2, 2, eb)
    run_blocks(cuda, oracle, t213, 64 * 7, 64 * 5, 1, eb)


@pytest.mark.parametrize("offset", (4, 8))
def test_unaligned_base_falls_back(cuda, oracle, t213, offset):
    """A base address that is not 16-byte aligned cannot feed TMA; the pass
    must take the element-wise kernel and stay exact."""
    run_blocks(cuda, oracle, t213, 512, 384, 2, 4, offset=offset)


def test_status_clear_after_tile_swaps(cuda, t213):
    assert t213.device_status() == 0
