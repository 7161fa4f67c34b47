"""The serving form: requests admitted by HBM budget and run concurrently give
exactly the result they give alone, which is the checksum of a correct 213
transpose computed from the fill (exact: data movement)."""
import importlib
import math
import random

import pytest

pytestmark = pytest.mark.gpu


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


def test_served_workload(t213, cuda):
    """The serving configuration: Poisson 2000 req/s, 1 KB-2 GB log-uniform,
    150 GB budget, 64 in flight on 8 streams, all 2000 requests."""
    w = importlib.import_module("213transpose_b200.workloads")
    reqs = w.serving_requests(5, 2000)
    for i, r in enumerate(reqs):
        r["seed"] = 7 + i
    srv = t213.Server(hbm_budget_bytes=150 * 10**9, max_inflight=64, streams=8)
    stats, sums, lat = srv.run(reqs)
    assert stats["completed"] == len(reqs)
    assert t213.device_status() == 0
    for r, s in list(zip(reqs, sums))[::5]:
        assert s == srv.expected_checksum(r), r
    srv.close()


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
