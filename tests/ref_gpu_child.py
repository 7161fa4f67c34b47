"""Runs the reference's own GPU transpose in a process of its own.

Test infrastructure: ``tests/test_gpu_ref_parity.py`` starts this script with
a JSON list of jobs.  For each job it makes the seeded input (``make_input``,
the same generator the test uses), copies it into managed memory (the
reference prefetches its argument as managed memory, src/transpose.cu:104),
calls ``inplace::transpose<T>`` of the reference's library compiled from its
sources (``oracle/_ref/libref_inplace.so``, through ``oracle/ref_gpu_shim.cu``)
and writes a digest of the result bytes, and for small jobs the bytes
themselves, to the result file.  A job with ``time_reps`` also times that
many further calls on the resident buffer (wall time per call, best and
median; each call ends in a device synchronisation).

The reference runs here and not inside pytest because it prints to stdout and
exits the process on a CUDA error (src/cudacheck.cu:4-9); in a child process
neither reaches the test runner, and no other library shares its CUDA runtime.

Usage: python ref_gpu_child.py jobs.json results.json
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_inplace.so")

# type codes of ref_inplace_transpose_typed (oracle/ref_gpu_shim.cu)
CODES = {"int32": (0, 4), "float32": (1, 4), "int64": (2, 8), "float64": (3, 8)}


def make_input(kind: str, n_elems: int, eb: int, seed: int) -> np.ndarray:
    """Seeded input as raw bytes: ``uniform`` draws uniform[-1,1) floats of the
    element size from numpy's default_rng(seed); ``bits`` draws random bytes."""
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        ft = {4: np.float32, 8: np.float64}[eb]
        return rng.uniform(-1.0, 1.0, n_elems).astype(ft).view(np.uint8)
    return rng.integers(0, 256, size=n_elems * eb, dtype=np.uint8)


def digest(buf: np.ndarray) -> str:
    return hashlib.blake2b(memoryview(np.ascontiguousarray(buf)).cast("B"), digest_size=16).hexdigest()


def _load() -> ctypes.CDLL:
    try:
        L = ctypes.CDLL(REF_GPU)
    except OSError:
        for cand in ("/usr/local/cuda/lib64/libcudart.so.12", "libcudart.so.12"):
            try:
                ctypes.CDLL(cand, mode=ctypes.RTLD_GLOBAL)
                break
            except OSError:
                continue
        L = ctypes.CDLL(REF_GPU)
    L.ref_alloc_managed.argtypes = [ctypes.c_size_t]
    L.ref_alloc_managed.restype = ctypes.c_void_p
    L.ref_free_managed.argtypes = [ctypes.c_void_p]
    L.ref_inplace_transpose_typed.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int]
    return L


def main() -> int:
    jobs = json.load(open(sys.argv[1]))
    out_path = sys.argv[2]
    L = _load()
    results = {}
    for job in jobs:
        code, eb = CODES[job["type"]]
        d1, d2, d3 = job["d1"], job["d2"], job["d3"]
        x = make_input(job["gen"], d1 * d2 * d3, eb, job["seed"])
        nbytes = x.size
        p = L.ref_alloc_managed(nbytes)
        if not p:
            results[job["name"]] = {"rc": -100}
            continue
        ctypes.memmove(p, x.ctypes.data, nbytes)
        rc = L.ref_inplace_transpose_typed(p, d1, d2, d3, code)
        y = np.empty_like(x)
        ctypes.memmove(y.ctypes.data, p, nbytes)
        res = {"rc": int(rc), "digest": digest(y)}
        if rc == 0 and job.get("time_reps"):
            # timing of further calls on the resident (already prefetched)
            # buffer; each call ends in cudaDeviceSynchronize, so the wall
            # time of a call is its launches, kernels and host work
            ts = []
            for _ in range(int(job["time_reps"])):
                t0 = time.perf_counter()
                L.ref_inplace_transpose_typed(p, d1, d2, d3, code)
                ts.append((time.perf_counter() - t0) * 1e3)
            ts.sort()
            res["ms_best"], res["ms_median"] = round(ts[0], 4), round(ts[len(ts) // 2], 4)
        L.ref_free_managed(p)
        if job.get("save"):
            y.tofile(job["save"])
        results[job["name"]] = res
        # written after every job, so a later failure still leaves the earlier results
        with open(out_path, "w") as f:
            json.dump(results, f)
    with open(out_path, "w") as f:
        json.dump(results, f)
    return 0


if __name__ == "__main__":
    sys.exit(main())
