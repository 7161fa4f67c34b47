"""The batched form: one persistent, graph-captured launch over many uneven
tensors gives, for every tensor, the same bytes as the oracle and as the
looped plain call."""
import importlib
import random

import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu


def _mixed_shapes(seed):
    rng = random.Random(seed)
    out = []
    plans = ["auto", "c2r", "r2c", "blocks", "bands", "bands_t", "skinny"]
    for i in range(48):
        d1, d2 = rng.randint(1, 700), rng.randint(1, 700)
        if i % 5 == 0:  # gcd-rich shapes for block plans
            g = rng.choice([32, 64, 96, 128])
            d1, d2 = g * rng.randint(1, 6), g * rng.randint(1, 6)
        if i % 7 == 0:  # skinny
            d2 = rng.randint(1, 32)
        d3 = rng.randint(1, 3)
        eb = rng.choice([4, 8, 16, 4, 1, 2])
        out.append((d1, d2, d3, eb, plans[i % len(plans)]))
    return out


def _applicable(t213, d1, d2, d3, eb, plan):
    try:
        t213.describe(d1, d2, d3, eb, plan)
        return plan
    except t213.T213Error:
        return "auto"


def test_batch_matches_oracle_and_loop(cuda, oracle, t213):
    shapes = [(d1, d2, d3, eb, _applicable(t213, d1, d2, d3, eb, p)) for d1, d2, d3, eb, p in _mixed_shapes(11)]
    hosts, wants, devs = [], [], []
    for i, (d1, d2, d3, eb, _) in enumerate(shapes):
        x = oracle.random_bits(d1 * d2 * d3, eb, 100 + i)
        hosts.append(x)
        wants.append(oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8))
        devs.append(to_device(cuda, x))
    B = t213.Batch([(dev, d1, d2, d3, eb, plan) for dev, (d1, d2, d3, eb, plan) in zip(devs, shapes)])
    assert "batch: 48 tensors" in B.describe()
    for rep in range(2):  # first call captures the graph, the second replays it
        for dev, x in zip(devs, hosts):
            dev.copy_(cuda.from_numpy(x))
        B.execute()
        assert B.status() == 0
        for i, (dev, want) in enumerate(zip(devs, wants)):
            assert np.array_equal(from_device(dev), want), (rep, shapes[i])
    for dev, x in zip(devs, hosts):
        dev.copy_(cuda.from_numpy(x))
    B.looped()
    cuda.cuda.synchronize()
    for i, (dev, want) in enumerate(zip(devs, wants)):
        assert np.array_equal(from_device(dev), want), ("looped", shapes[i])
    B.close()


def test_batch_full_config_round_trip(cuda, t213):
    """All 512 tensors of the batched configuration (seed 1): one batch, then a
    second batch with the axes swapped restores every tensor bit for bit."""
    w = importlib.import_module("213transpose_b200.workloads")
    shapes = w.batched_shapes(1, 512)
    gen = cuda.Generator(device="cuda").manual_seed(1)
    devs, origs = [], []
    for d1, d2, d3, eb, _ in shapes:
        x = cuda.empty(d1 * d2 * d3 * eb, dtype=cuda.uint8, device="cuda")
        x.random_(0, 256, generator=gen)
        devs.append(x)
        origs.append(x.clone())
    fwd = t213.Batch([(x, d1, d2, d3, eb) for x, (d1, d2, d3, eb, _) in zip(devs, shapes)])
    back = t213.Batch([(x, d2, d1, d3, eb) for x, (d1, d2, d3, eb, _) in zip(devs, shapes)])
    fwd.execute()
    assert fwd.status() == 0
    # spot-check a few tensors of the forward batch against torch's permute
    for i in range(0, 512, 97):
        d1, d2, d3, eb, _ = shapes[i]
        want = origs[i].view(d3, d2, d1, eb).permute(0, 2, 1, 3).contiguous().view(-1)
        assert cuda.equal(devs[i], want), shapes[i]
    # and a sample of 24 (the three largest among them) byte for byte against the oracle
    from oracle import oracle as O
    size = [d1 * d2 * d3 * eb for d1, d2, d3, eb, _ in shapes]
    largest = sorted(range(512), key=lambda i: -size[i])[:3]
    for i in sorted(set(largest) | set(range(5, 512, 23))):
        d1, d2, d3, eb, _ = shapes[i]
        x = origs[i].cpu().numpy()
        want = O.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
        assert np.array_equal(from_device(devs[i]), want), shapes[i]
    back.execute()
    assert back.status() == 0
    bad = [shapes[i] for i in range(512) if not cuda.equal(devs[i], origs[i])]
    assert not bad, bad[:5]


def test_batch_unaligned_column_items(cuda, oracle, t213):
    """Column items over pitches that are not 16-byte multiples (4- and
    8-byte elements, word-width accesses): tensors of odd and 2 mod 4 row
    lengths, column heights up to about 1200, placed in one buffer at bases
    off a 16-byte boundary with guard bytes between them.  Each tensor must
    match the oracle and no guard byte may change."""
    specs = [(701, 333, 1, 4, "c2r"), (333, 701, 2, 4, "r2c"), (1001, 1187, 1, 8, "c2r"), (1187, 1001, 1, 8, "r2c"),
             (998, 601, 2, 4, "c2r"), (601, 998, 1, 4, "r2c"), (97, 1201, 3, 8, "c2r"), (1201, 97, 3, 8, "r2c"),
             (35, 35, 4, 8, "c2r"), (5, 3, 7, 4, "r2c"), (4001, 9, 2, 4, "c2r"), (9, 4001, 2, 8, "r2c")]
    guard = 64
    offs, pos = [], guard
    for i, (d1, d2, d3, eb, _) in enumerate(specs):
        pos += (4 * (i % 3 + 1)) if eb == 4 else 8  # bases 4, 8 or 12 past a 16-byte boundary
        offs.append(pos)
        pos += d1 * d2 * d3 * eb + guard
        pos = (pos + 15) // 16 * 16
    host = np.full(pos, 0xC3, np.uint8)
    wants = []
    for i, ((d1, d2, d3, eb, _), o) in enumerate(zip(specs, offs)):
        x = oracle.random_bits(d1 * d2 * d3, eb, 500 + i)
        host[o:o + x.nbytes] = x.view(np.uint8)
        wants.append(oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8))
    dev = to_device(cuda, host)
    views = [dev[o:o + d1 * d2 * d3 * eb] for (d1, d2, d3, eb, _), o in zip(specs, offs)]
    B = t213.Batch([(v, d1, d2, d3, eb, plan) for v, (d1, d2, d3, eb, plan) in zip(views, specs)])
    B.execute()
    assert B.status() == 0
    got = from_device(dev)
    mask = np.ones(pos, bool)
    for (d1, d2, d3, eb, plan), o, want in zip(specs, offs, wants):
        n = d1 * d2 * d3 * eb
        assert np.array_equal(got[o:o + n], want), (d1, d2, d3, eb, plan, o)
        mask[o:o + n] = False
    assert (got[mask] == 0xC3).all(), "bytes outside the tensors were written"
    B.close()
