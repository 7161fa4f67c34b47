"""Command-line tool of the package.

  python -m 213transpose_b200.cli run D1 D2 D3 ELEM_BYTES [--plan P] [--t T] [--iters N] [--check]
      transposes a seeded random tensor in place N times on cuda:0 and prints
      the per-call time and effective bandwidth (2*bytes/time); --check
      compares the first call with the answer computed by a second, out-of-
      place torch permute on the GPU.
  python -m 213transpose_b200.cli describe D1 D2 D3 ELEM_BYTES [--plan P]
  python -m 213transpose_b200.cli tune D1 D2 D3 ELEM_BYTES [--save FILE]
"""
from __future__ import annotations

import argparse
import importlib
import json


def main(argv=None):
    ap = argparse.ArgumentParser(prog="213transpose_b200.cli")
    sub = ap.add_subparsers(dest="cmd", required=True)
    for name in ("run", "describe", "tune"):
        p = sub.add_parser(name)
        p.add_argument("d1", type=int)
        p.add_argument("d2", type=int)
        p.add_argument("d3", type=int)
        p.add_argument("elem_bytes", type=int)
        p.add_argument("--plan", default="auto")
        p.add_argument("--t", type=int, default=0)
        if name == "run":
            p.add_argument("--iters", type=int, default=3)
            p.add_argument("--check", action="store_true")
        if name == "tune":
            p.add_argument("--save", default=None)
    a = ap.parse_args(argv)
    t213 = importlib.import_module("213transpose_b200")
    if a.cmd == "describe":
        print(t213.describe(a.d1, a.d2, a.d3, a.elem_bytes, a.plan, a.t))
        return
    import torch
    n = a.d1 * a.d2 * a.d3 * a.elem_bytes
    x = torch.empty(n, dtype=torch.uint8, device="cuda:0")
    gen = torch.Generator(device="cuda:0").manual_seed(0)
    x.random_(0, 256, generator=gen)
    if a.cmd == "tune":
        import ctypes
        kind, tt = ctypes.c_int32(0), ctypes.c_int64(0)
        t213._lib.check(t213.lib().t213_tune_shape(ctypes.c_void_p(x.data_ptr()), a.d1, a.d2, a.d3, a.elem_bytes,
                                                   None, ctypes.byref(kind), ctypes.byref(tt)))
        print(json.dumps({"plan_kind": kind.value, "t": tt.value,
                          "desc": t213.describe(a.d1, a.d2, a.d3, a.elem_bytes)}))
        if a.save:
            t213._lib.check(t213.lib().t213_tuner_save(a.save.encode()))
        return
    want = None
    if a.check:
        eb = a.elem_bytes
        want = x.view(a.d3, a.d2, a.d1, eb).permute(0, 2, 1, 3).contiguous().view(-1)
    times = []
    for i in range(a.iters):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        t213.transpose_with_plan(x, a.d1, a.d2, a.d3, a.plan, a.t, elem_bytes=a.elem_bytes)
        e.record()
        e.synchronize()
        times.append(s.elapsed_time(e))
        if i == 0 and want is not None:
            ok = bool(torch.equal(x, want))
            print(json.dumps({"check": "bit-exact" if ok else "MISMATCH"}))
            if not ok:
                raise SystemExit(1)
    best = min(times)
    print(json.dumps({"shape": [a.d1, a.d2, a.d3, a.elem_bytes],
                      "plan": t213.describe(a.d1, a.d2, a.d3, a.elem_bytes, a.plan, a.t),
                      "ms_best": round(best, 4), "ms_all": [round(t, 4) for t in times],
                      "eff_GBps": round(2 * n / best / 1e6, 1)}))


if __name__ == "__main__":
    main()
