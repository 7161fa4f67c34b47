"""Failure detection on the device without a fault.

The batched form's persistent kernel orders a tensor's passes with per-pass
counters: a CTA that runs an item of pass k first waits, bounded, until pass
k-1 has completed all its items.  Here the batch is told (through the test
hook t213_batch_debug_stall) to cap that wait at a few milliseconds and to
make one pass wait for an item its predecessor does not have, a flag that
nothing sets.  The launch must come back on its own, report T213_ERR_TIMEOUT
once through t213_batch_status, and leave the device usable: a plain call
right after it is exact against the oracle.  The reference's equivalent
waits are unbounded grid-wide syncs (src/memory_ops.cu:18-33,
src/skinny.cu:31-60), which no test can make run out.
"""
import time

import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu

T213_ERR_TIMEOUT = 5
SHAPES = [(512, 384, 2, 4), (600, 200, 2, 8), (96, 70, 3, 16)]


def test_batch_dependency_wait_runs_out(cuda, oracle, t213):
    torch = cuda
    L = t213.lib()
    xs = [to_device(torch, oracle.random_bits(d1 * d2 * d3, eb, 40 + i)) for i, (d1, d2, d3, eb) in enumerate(SHAPES)]
    b = t213.Batch([(x, d1, d2, d3, eb) for x, (d1, d2, d3, eb) in zip(xs, SHAPES)])
    try:
        assert L.t213_batch_debug_stall(b._h, 5_000_000, -1) == 0, L.t213_last_error().decode()
        st = torch.cuda.Stream()
        t0 = time.perf_counter()
        b.execute(st)
        assert b.status(st) == T213_ERR_TIMEOUT
        elapsed = time.perf_counter() - t0
        # came back through the 5 ms limit, not the default 2 s one
        assert elapsed < 1.0, elapsed
        assert b"bounded wait" in L.t213_last_error()
        assert b.status(st) == 0  # reading cleared the word
    finally:
        b.close()
    # the context is intact: the next plain call is exact
    d1, d2, d3, eb = 700, 300, 3, 4
    x = oracle.random_bits(d1 * d2 * d3, eb, 7)
    want = oracle.gather213(x.view(np.uint32), d1, d2, d3).view(np.uint8)
    dev = to_device(torch, x)
    t213.transpose(dev, d1, d2, d3, elem_bytes=eb)
    assert np.array_equal(from_device(dev), want)
    assert t213.device_status() == 0


def test_batch_without_stall_keeps_the_default_limit(cuda, oracle, t213):
    """The same batch without the hook completes with status 0 and exact bytes."""
    torch = cuda
    hosts = [oracle.random_bits(d1 * d2 * d3, eb, 40 + i) for i, (d1, d2, d3, eb) in enumerate(SHAPES)]
    xs = [to_device(torch, h) for h in hosts]
    b = t213.Batch([(x, d1, d2, d3, eb) for x, (d1, d2, d3, eb) in zip(xs, SHAPES)])
    try:
        st = torch.cuda.Stream()
        b.execute(st)
        assert b.status(st) == 0
    finally:
        b.close()
    for h, x, (d1, d2, d3, eb) in zip(hosts, xs, SHAPES):
        want = oracle.gather213(h.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
        assert np.array_equal(from_device(x), want)


def test_debug_stall_rejects_a_pass_without_predecessor(cuda, oracle, t213):
    torch = cuda
    L = t213.lib()
    x = to_device(torch, oracle.random_bits(512 * 384, 4, 1))
    b = t213.Batch([(x, 512, 384, 1, 4)])
    try:
        assert L.t213_batch_debug_stall(b._h, 5_000_000, 0) == 1  # pass 0 waits on nothing
        assert L.t213_batch_debug_stall(b._h, 0, -1) == 1
    finally:
        b.close()
