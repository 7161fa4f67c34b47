"""The serving form: requests admitted by HBM budget and run concurrently give
exactly the result they give alone, which is the checksum of a correct 213
transpose computed from the fill (exact: data movement).  Sampled requests
are also copied back and compared byte for byte with the oracle's gather of
the same fill, restated here on the host; small requests admitted together
share grouped launches, and their bytes are the same with grouping off."""
import importlib
import math
import random

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def _smix(x):
    """splitmix64's finaliser (Vigna) on uint64 arrays, as the server's fill uses it."""
    x = x + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def fill_host(r) -> np.ndarray:
    """The bytes the server's device fill gives request r: word w of element e
    is smix(seed * 0xD1B54A32D192ED03 ^ (2e + w)); an element keeps the low
    elem_bytes bytes of word 0, or words 0 and 1 for 16-byte elements."""
    n = int(r["d1"]) * int(r["d2"]) * int(r["d3"])
    eb = int(r["elem_bytes"])
    key = np.uint64((int(r["seed"]) * 0xD1B54A32D192ED03) & M64)
    e2 = np.arange(n, dtype=np.uint64) * np.uint64(2)
    with np.errstate(over="ignore"):
        w0 = _smix(key ^ e2)
        if eb == 16:
            w1 = _smix(key ^ (e2 + np.uint64(1)))
            return np.stack([w0, w1], axis=1).reshape(-1).view(np.uint8)
    return w0.view(np.uint8).reshape(n, 8)[:, :eb].reshape(-1).copy()


def _expect_bytes(oracle, r):
    eb = int(r["elem_bytes"])
    x = fill_host(r)
    return oracle.gather213(x.view(np.dtype((np.void, eb))), int(r["d1"]), int(r["d2"]), int(r["d3"])).view(np.uint8)


def _requests(seed, n, lo, hi, span_s):
    rng = random.Random(seed)
    out = []
    for i in range(n):
        size = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        eb = rng.choice([4, 8, 4, 16])
        d3 = rng.choice([1, 2, 4, 8])
        elems = max(1, int(size / (eb * d3)))
        d1 = max(1, int(math.exp(rng.uniform(0, math.log(max(1, elems))))))
        d2 = max(1, elems // d1)
        out.append({"d1": d1, "d2": d2, "d3": d3, "elem_bytes": eb, "t": rng.uniform(0, span_s), "seed": 1000 + i})
    return out


def test_mix_equals_alone_equals_expected(t213, cuda):
    srv = t213.Server(hbm_budget_bytes=8 << 30, max_inflight=32, streams=4)
    reqs = _requests(7, 120, 1e3, 64e6, 0.02)
    stats, sums, lat = srv.run(reqs)
    assert stats["completed"] == len(reqs) and stats["rejected"] == 0
    assert stats["max_inflight"] > 1  # requests overlapped on the device
    for r, s in zip(reqs, sums):
        assert s == srv.expected_checksum(r), r
    for r, s in list(zip(reqs, sums))[::7]:
        assert srv.run_alone(r) == s, r
    assert all(v >= 0 for v in lat)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    srv.close()


def test_admission_under_budget_pressure(t213, cuda):
    budget = 512 << 20
    srv = t213.Server(hbm_budget_bytes=budget, max_inflight=16, streams=4)
    reqs = [{"d1": 4096, "d2": 3000 + i, "d3": 2, "elem_bytes": 4, "t": 0.0, "seed": i} for i in range(12)]  # ~100 MB
    reqs.append({"d1": 65536, "d2": 65536, "d3": 1, "elem_bytes": 4, "t": 0.0, "seed": 99})  # 17 GB > budget
    stats, sums, lat = srv.run(reqs)
    assert stats["rejected"] == 1 and stats["completed"] == 12
    assert stats["peak_resident_bytes"] <= budget
    assert lat[-1] < 0 and sums[-1] == 0
    for r, s in zip(reqs[:-1], sums[:-1]):
        assert s == srv.expected_checksum(r)
    srv.close()


def test_served_workload(t213, cuda, oracle):
    """The serving configuration: Poisson 2000 req/s, 1 KB-2 GB log-uniform,
    150 GB budget, 64 in flight on 8 streams, all 2000 requests.  Every fifth
    checksum is checked; 24 requests, the five largest under 512 MB among
    them, come back as bytes and equal the oracle's answer."""
    w = importlib.import_module("213transpose_b200.workloads")
    reqs = w.serving_requests(5, 2000)
    for i, r in enumerate(reqs):
        r["seed"] = 7 + i
    size = [r["d1"] * r["d2"] * r["d3"] * r["elem_bytes"] for r in reqs]
    under = sorted((i for i in range(len(reqs)) if size[i] <= (512 << 20)), key=lambda i: -size[i])
    sample = sorted(set(under[:5]) | set(random.Random(3).sample(range(len(reqs)), 19)))
    capture = {i: np.empty(size[i], dtype=np.uint8) for i in sample}
    srv = t213.Server(hbm_budget_bytes=150 * 10**9, max_inflight=64, streams=8)
    stats, sums, lat = srv.run(reqs, capture=capture)
    assert stats["completed"] == len(reqs)
    assert stats["group_launches"] > 0 and stats["grouped_requests"] >= 2 * stats["group_launches"]
    assert t213.device_status() == 0
    for r, s in list(zip(reqs, sums))[::5]:
        assert s == srv.expected_checksum(r), r
    srv.close()
    for i in sample:
        assert np.array_equal(capture[i], _expect_bytes(oracle, reqs[i])), (i, reqs[i])


def test_grouped_launches_equal_single_launches(t213, cuda, oracle, monkeypatch):
    """A burst of small requests: admitted together they share grouped
    launches; with grouping off every request runs alone on its stream.  The
    bytes are identical both ways and equal the oracle's."""
    rng = random.Random(21)
    reqs = []
    for i in range(48):
        eb = rng.choice([1, 2, 4, 8, 16])
        d3 = rng.choice([1, 2, 3])
        d1, d2 = rng.randint(1, 900), rng.randint(1, 900)
        reqs.append({"d1": d1, "d2": d2, "d3": d3, "elem_bytes": eb, "t": 0.0, "seed": 900 + i})
    size = [r["d1"] * r["d2"] * r["d3"] * r["elem_bytes"] for r in reqs]
    out = {}
    for groups in ("4", "0"):
        monkeypatch.setenv("T213_SERVE_GROUPS", groups)
        srv = t213.Server(hbm_budget_bytes=4 << 30, max_inflight=64, streams=4)
        srv.run(reqs)  # every plan built: the planners only look them up in the burst below
        capture = {i: np.empty(size[i], dtype=np.uint8) for i in range(len(reqs))}
        stats, sums, lat = srv.run(reqs, capture=capture)
        srv.close()
        assert stats["completed"] == len(reqs)
        if groups == "4":
            assert stats["group_launches"] >= 1 and stats["grouped_requests"] >= 2
        else:
            assert stats["group_launches"] == 0
        out[groups] = (sums, capture)
    assert out["4"][0] == out["0"][0]
    for i, r in enumerate(reqs):
        assert np.array_equal(out["4"][1][i], out["0"][1][i]), r
        assert np.array_equal(out["4"][1][i], _expect_bytes(oracle, r)), r


def test_fresh_cycle_tables_on_concurrent_streams(t213, cuda):
    """Shapes whose plans walk segment cycles, each seen for the first time,
    all arriving at once on 8 non-blocking streams: a pass must not start
    before its cycle table has landed on the device."""
    t213.release_cache()
    rng = random.Random(11)
    reqs = []
    while len(reqs) < 96:
        eb = rng.choice([4, 8, 16])
        d3 = rng.choice([1, 2, 4])
        d1 = int(math.exp(rng.uniform(math.log(16), math.log(20000))))
        d2 = max(16, int(rng.uniform(2e5, 4e6) / (d1 * d3 * eb)))
        if "segment_cycles" not in t213.describe(d1, d2, d3, eb):
            continue
        reqs.append({"d1": d1, "d2": d2, "d3": d3, "elem_bytes": eb, "t": 0.0, "seed": 500 + len(reqs)})
    t213.release_cache()
    srv = t213.Server(hbm_budget_bytes=32 << 30, max_inflight=64, streams=8)
    stats, sums, lat = srv.run(reqs)
    assert stats["completed"] == len(reqs)
    assert t213.device_status() == 0
    for r, s in zip(reqs, sums):
        assert s == srv.expected_checksum(r), r
    srv.close()
