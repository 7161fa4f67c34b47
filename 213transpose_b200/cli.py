"""Command-line tool of the package.

  python -m 213transpose_b200.cli run D1 D2 D3 ELEM_BYTES [--plan P] [--t T] [--iters N] [--check]
      transposes a seeded random tensor in place N times on cuda:0 and prints
      the per-call time and effective bandwidth (2*bytes/time); --check
      compares the first call with the answer computed by a second, out-of-
      place torch permute on the GPU.
  python -m 213transpose_b200.cli describe D1 D2 D3 ELEM_BYTES [--plan P]
  python -m 213transpose_b200.cli tune D1 D2 D3 ELEM_BYTES [--save FILE]
  python -m 213transpose_b200.cli compare FILE_A FILE_B D1 D2 D3 TYPE_SIZE
      compares two raw output files of the drivers (test_213inplace, gen_ans:
      vol elements of TYPE_SIZE bytes, no header, as TensorUtil::write_file
      writes them, src/tensor_util.cpp:69-72) element by element; prints the
      mismatch count and the first mismatch as transposed-layout coordinates
      (i2, i1, i3); exit status 1 on any difference.
  python -m 213transpose_b200.cli dump FILE D1 D2 D3 TYPE_SIZE [--slice K] [--rows R]
      prints slice K of a driver's output (transposed layout: d1 rows of d2).
"""
from __future__ import annotations

import argparse
import importlib
import json


def _raw(path, d1, d2, d3, ts):
    import numpy as np
    vol = d1 * d2 * d3
    dt = {1: np.uint8, 2: np.uint16, 4: np.int32, 8: np.int64}.get(ts)
    a = np.fromfile(path, dtype=np.uint8)
    if a.size != vol * ts:
        raise SystemExit(f"{path}: {a.size} bytes, expected {vol} elements of {ts} bytes ({vol * ts} bytes)")
    return a.view(dt) if dt is not None else a.reshape(vol, ts)


def compare(a_path, b_path, d1, d2, d3, ts) -> dict:
    import numpy as np
    a, b = _raw(a_path, d1, d2, d3, ts), _raw(b_path, d1, d2, d3, ts)
    diff = (a != b) if a.ndim == 1 else (a != b).any(axis=1)
    bad = np.flatnonzero(diff)
    out = {"elements": int(d1 * d2 * d3), "mismatches": int(bad.size)}
    if bad.size:
        e = int(bad[0])  # transposed layout: i2 fastest, then i1, then i3
        out["first"] = {"index": e, "i2": e % d2, "i1": (e // d2) % d1, "i3": e // (d1 * d2)}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="213transpose_b200.cli")
    sub = ap.add_subparsers(dest="cmd", required=True)
    pc = sub.add_parser("compare")
    pc.add_argument("a")
    pc.add_argument("b")
    pd = sub.add_parser("dump")
    pd.add_argument("file")
    for p in (pc, pd):
        for name in ("d1", "d2", "d3", "type_size"):
            p.add_argument(name, type=int)
    pd.add_argument("--slice", type=int, default=0)
    pd.add_argument("--rows", type=int, default=8)
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
    if a.cmd == "compare":
        r = compare(a.a, a.b, a.d1, a.d2, a.d3, a.type_size)
        print(json.dumps(r))
        raise SystemExit(1 if r["mismatches"] else 0)
    if a.cmd == "dump":
        x = _raw(a.file, a.d1, a.d2, a.d3, a.type_size)
        per = a.d1 * a.d2
        sl = x[a.slice * per:(a.slice + 1) * per]
        for r in range(min(a.rows, a.d1)):
            print(" ".join(str(v) for v in sl[r * a.d2:(r + 1) * a.d2][:16]) + (" ..." if a.d2 > 16 else ""))
        return
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
