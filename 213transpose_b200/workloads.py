"""Synthetic workloads of the batched and served forms.

batched_shapes(seed=1, count=512): tensors with d1, d2 log-uniform in
  [16, 4096], d3 from {1, 2, 4, 8}, element type fp32 / fp64 / int32 / 16-byte
  with equal probability (numpy default_rng(seed), drawn in that order per
  tensor).

serving_requests(seed, n, rate=2000.0, lo=1e3, hi=2e9): a Poisson arrival
  stream (exponential gaps at `rate` per second) of requests whose total size
  is log-uniform in [lo, hi] bytes.  For each request the element type and d3
  are drawn as above, then d1 log-uniform within the bounds that keep d2 >= 1
  and d1, d2 >= 16 where the size allows, and d2 = size / (d1 * d3 * elem).
"""
from __future__ import annotations

import math

import numpy as np

ELEM = {"f32": 4, "f64": 8, "i32": 4, "b16": 16}
KINDS = ("f32", "f64", "i32", "b16")


def batched_shapes(seed: int = 1, count: int = 512):
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = math.log(16), math.log(4096)
    for _ in range(count):
        d1 = int(round(math.exp(rng.uniform(lo, hi))))
        d2 = int(round(math.exp(rng.uniform(lo, hi))))
        d3 = int(rng.choice([1, 2, 4, 8]))
        kind = KINDS[int(rng.integers(0, 4))]
        out.append((d1, d2, d3, ELEM[kind], kind))
    return out


def total_bytes(shapes) -> int:
    return sum(d1 * d2 * d3 * eb for d1, d2, d3, eb, _ in shapes)


def serving_requests(seed: int, n: int, rate: float = 2000.0, lo: float = 1e3, hi: float = 2e9):
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        size = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        kind = KINDS[int(rng.integers(0, 4))]
        eb = ELEM[kind]
        d3 = int(rng.choice([1, 2, 4, 8]))
        elems = max(1.0, size / (eb * d3))
        # d1 log-uniform in [16, elems/16] when that range exists
        lo1, hi1 = 16.0, max(16.0, elems / 16.0)
        if elems < 256:
            lo1, hi1 = 1.0, max(1.0, elems)
        d1 = int(round(math.exp(rng.uniform(math.log(lo1), math.log(hi1)))))
        d1 = max(1, min(d1, int(elems)))
        d2 = max(1, int(elems // d1))
        out.append({"t": t, "d1": d1, "d2": d2, "d3": d3, "elem_bytes": eb, "kind": kind})
    return out
