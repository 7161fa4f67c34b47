"""The autotuner: tune -> lookup -> save -> clear -> load -> lookup round trip,
tuned plans exact against the oracle, every kernel variant the tuner can pin
exact against the oracle, and a tuned batch exact against the oracle.

The tuner's cache is process-wide state that the automatic plan choice
reads, so every test here clears it when it ends."""
import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu

PLAN = {"c2r": 1, "r2c": 2, "skinny": 3, "blocks": 4, "bands": 5, "bands_t": 6, "slice": 8}


def _var(col=0, row=0, tile=0, seg=0):
    return col | row << 4 | tile << 8 | seg << 12


@pytest.fixture
def clean_tuner(t213):
    t213.tuner.clear()
    yield
    t213.tuner.clear()


def _exact(cuda, oracle, t213, d1, d2, d3, eb, seed):
    x = oracle.random_bits(d1 * d2 * d3, eb, seed)
    want = oracle.gather213(x.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
    dev = to_device(cuda, x)
    t213.transpose(dev, d1, d2, d3, elem_bytes=eb)
    assert np.array_equal(from_device(dev), want), (d1, d2, d3, eb, t213.describe(d1, d2, d3, eb))


def test_tune_save_clear_load_lookup(cuda, oracle, t213, clean_tuner, tmp_path):
    shapes = [(1000, 600, 2, 4), (512, 384, 3, 8), (96, 2048, 1, 16), (997, 601, 1, 4), (64, 100000, 1, 4)]
    chosen = {}
    for i, s in enumerate(shapes):
        chosen[s] = t213.tuner.tune(*s)
        assert t213.tuner.lookup(*s) == chosen[s]
        assert t213.describe(*s).startswith(chosen[s][0])
        _exact(cuda, oracle, t213, *s, seed=50 + i)  # the plain call now runs the tuned plan
    path = tmp_path / "tuner.txt"
    t213.tuner.save(path)
    t213.tuner.clear()
    assert all(t213.tuner.lookup(*s) is None for s in shapes)
    t213.tuner.load(path)
    for s in shapes:
        assert t213.tuner.lookup(*s) == chosen[s]
    # a shape of the same class, not tuned itself, takes the class's family
    d1, d2, d3, eb = shapes[0]
    other = (800, 600, d3, eb)  # same log2 sizes and log2 gcd as (1000, 600)
    looked = t213.tuner.lookup(*other)
    assert looked is not None and looked[0] == chosen[shapes[0]][0]
    _exact(cuda, oracle, t213, *other, seed=60)


# shape, family, block size (0: the planner's), pinned variant
VARIANTS = [
    ((7919, 601, 1, 8), "c2r", 0, _var(col=1)),
    ((7919, 601, 1, 8), "c2r", 0, _var(col=2)),
    ((7919, 601, 1, 8), "c2r", 0, _var(row=2)),
    ((7919, 601, 1, 8), "c2r", 0, _var(col=3)),
    ((7919, 6151, 1, 8), "c2r", 0, _var(col=3)),
    ((7919, 6151, 1, 8), "c2r", 0, _var(col=4)),
    ((3001, 2000, 2, 4), "r2c", 0, _var(col=4)),
    ((30, 100000, 1, 4), "skinny", 0, _var(col=3)),
    ((3001, 2000, 2, 4), "r2c", 0, _var(col=2, row=2)),
    ((3001, 2000, 2, 4), "r2c", 0, _var(col=1, row=1)),
    ((1024, 768, 2, 4), "blocks", 256, _var(tile=1)),
    ((1024, 768, 2, 4), "blocks", 256, _var(tile=2, seg=2)),
    ((1024, 768, 2, 8), "blocks", 256, _var(tile=1, seg=3)),
    ((4096, 96, 1, 8), "bands", 0, _var(seg=2)),
    ((4096, 96, 1, 8), "bands", 0, _var(seg=3)),
    ((96, 3000, 2, 16), "bands_t", 0, _var(seg=3)),
    ((30, 100000, 1, 4), "skinny", 0, _var(col=2, row=2)),
    ((30, 100000, 1, 4), "skinny", 0, _var(col=1)),
]


@pytest.mark.parametrize("case", VARIANTS, ids=[f"{c[1]}-{'x'.join(map(str, c[0]))}-v{c[3]:x}" for c in VARIANTS])
def test_pinned_variants_are_exact(cuda, oracle, t213, clean_tuner, tmp_path, case):
    (d1, d2, d3, eb), fam, t, var = case
    path = tmp_path / "pinned.txt"
    path.write_text(f"shape {d1} {d2} {d3} {eb} {PLAN[fam]} {t} {var}\n")
    t213.tuner.load(path)
    desc = t213.describe(d1, d2, d3, eb)
    assert desc.startswith(fam) and "[variant" in desc, desc
    _exact(cuda, oracle, t213, d1, d2, d3, eb, seed=var)


def test_tuned_batch_is_exact(cuda, oracle, t213, clean_tuner):
    shapes = [(300, 200, 2, 4), (1000, 37, 1, 8), (2048, 1536, 1, 4), (97, 33, 3, 16), (4096, 96, 1, 8)]
    hosts = [oracle.random_bits(d1 * d2 * d3, eb, 70 + i) for i, (d1, d2, d3, eb) in enumerate(shapes)]
    devs = [to_device(cuda, h) for h in hosts]
    b = t213.Batch([(x, d1, d2, d3, eb) for x, (d1, d2, d3, eb) in zip(devs, shapes)], tune=True)
    try:
        for s in shapes:
            assert t213.tuner.lookup(*s) is not None
        for dev, h in zip(devs, hosts):  # tuning ran on scratch memory: the data are untouched
            assert np.array_equal(from_device(dev), h)
        b.execute()
        assert b.status() == 0
    finally:
        b.close()
    for h, dev, (d1, d2, d3, eb) in zip(hosts, devs, shapes):
        want = oracle.gather213(h.view(np.dtype((np.void, eb))), d1, d2, d3).view(np.uint8)
        assert np.array_equal(from_device(dev), want), (d1, d2, d3, eb)
