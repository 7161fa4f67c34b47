"""The workload's configurations at their full sizes.

Every configuration, the large skinny tensors of 2.1 and 3.2 GB included, is
compared byte for byte with the oracle (the blocked, OpenMP-parallel 213
gather finishes in seconds at these sizes), and the large ones also through
the round trip (d1,d2) -> (d2,d1) restoring the input bit for bit.  Tensors
of more than 2^31 elements are checked through size-independent properties:
equality with torch's out-of-place permute on the device, and the round
trip."""
import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu


def _oracle_check(cuda, oracle, t213, x, d1, d2, d3, eb):
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    dev = to_device(cuda, x)
    t213.transpose(dev, d1, d2, d3, elem_bytes=eb)
    got = from_device(dev)
    assert np.array_equal(got, want), (d1, d2, d3, eb)
    return dev


def test_config1_fp32_512x384x16(cuda, oracle, t213):
    d1, d2, d3 = 512, 384, 16
    x = oracle.uniform_f32(d1 * d2 * d3, 0)  # uniform[-1,1), seed 0
    _oracle_check(cuda, oracle, t213, x, d1, d2, d3, 4)


def test_config2_fp32_8192x6144x4(cuda, oracle, t213):
    d1, d2, d3 = 8192, 6144, 4
    x = oracle.uniform_f32(d1 * d2 * d3, 0)
    dev = _oracle_check(cuda, oracle, t213, x, d1, d2, d3, 4)
    # and back: the transposed tensor is a (6144, 8192, 4) array
    t213.transpose(dev, d2, d1, d3, elem_bytes=4)
    assert np.array_equal(from_device(dev), x)


def test_config2_fp64_7919x6151x2(cuda, oracle, t213):
    d1, d2, d3 = 7919, 6151, 2
    x = oracle.uniform_f64(d1 * d2 * d3, 0)
    dev = _oracle_check(cuda, oracle, t213, x, d1, d2, d3, 8)
    t213.transpose(dev, d2, d1, d3, elem_bytes=8)
    assert np.array_equal(from_device(dev), x)


def _device_property_check(cuda, t213, d1, d2, d3, eb, seed):
    gen = cuda.Generator(device="cuda").manual_seed(seed)
    x = cuda.empty(d1 * d2 * d3 * eb, dtype=cuda.uint8, device="cuda")
    x.random_(0, 256, generator=gen)
    orig = x.clone()
    t213.transpose(x, d1, d2, d3, elem_bytes=eb)
    want = orig.view(d3, d2, d1, eb).permute(0, 2, 1, 3).contiguous().view(-1)
    assert cuda.equal(x, want), (d1, d2, d3, eb)
    del want
    t213.transpose(x, d2, d1, d3, elem_bytes=eb)
    assert cuda.equal(x, orig), ("round trip", d1, d2, d3, eb)
    assert t213.device_status() == 0


@pytest.mark.parametrize("shape", [(32, 1 << 24, 1, 4), (1 << 24, 48, 1, 4)], ids=["32x2^24", "2^24x48"])
def test_config3_large_skinny_fp32(cuda, oracle, t213, shape):
    d1, d2, d3, eb = shape
    x = oracle.random_bits(d1 * d2 * d3, eb, 3)
    dev = _oracle_check(cuda, oracle, t213, x, d1, d2, d3, eb)
    t213.transpose(dev, d2, d1, d3, elem_bytes=eb)
    assert np.array_equal(from_device(dev), x), "round trip"
    assert t213.device_status() == 0


def test_config3_int32_3x2p22x8(cuda, oracle, t213):
    d1, d2, d3 = 3, 1 << 22, 8
    x = oracle.random_bits(d1 * d2 * d3, 4, 3)
    _oracle_check(cuda, oracle, t213, x, d1, d2, d3, 4)


def test_config3_16byte_1024x1024(cuda, oracle, t213):
    d1, d2, d3 = 1024, 1024, 1
    x = oracle.random_bits(d1 * d2 * d3, 16, 3)
    _oracle_check(cuda, oracle, t213, x, d1, d2, d3, 16)


@pytest.mark.parametrize("plan", ["c2r", "r2c", "skinny", "bands", "bands_t", "blocks", "slice"])
def test_config3_skinny_every_applicable_plan(cuda, oracle, t213, plan):
    """Every decomposition that applies to a (mid-size) skinny shape agrees."""
    for d1, d2, d3, eb in [(32, 1 << 16, 2, 4), (1 << 16, 48, 1, 4), (3, 1 << 14, 4, 4)]:
        try:
            t213.describe(d1, d2, d3, eb, plan)
        except t213.T213Error:
            continue
        x = oracle.random_bits(d1 * d2 * d3, eb, 5)
        want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
        dev = to_device(cuda, x)
        t213.transpose_with_plan(dev, d1, d2, d3, plan, elem_bytes=eb)
        assert np.array_equal(from_device(dev), want), (plan, d1, d2, d3)


@pytest.mark.parametrize("shape", [(1 << 16, (1 << 15) + 1, 1, 4), (46341, 46345, 1, 4)],
                         ids=["65536x32769", "46341x46345"])
def test_more_than_2p31_elements(cuda, t213, shape):
    """Tensors of more than 2^31 elements (8.6 GB fp32): the 64-bit index
    paths of the functors, checked against torch's out-of-place permute on
    the device and by the round trip."""
    d1, d2, d3, eb = shape
    assert d1 * d2 * d3 > (1 << 31)
    _device_property_check(cuda, t213, d1, d2, d3, eb, seed=7)
