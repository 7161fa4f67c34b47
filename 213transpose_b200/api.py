"""Python mirror of kaihsin/213transpose's C++ interface, on top of the C ABI.

Names, argument order and meaning follow the reference:

  inplace.transpose(data, d1, d2, d3)            include/transpose.h:17-18
  inplace.c2r.transpose(data, d1, d2, d3)        include/transpose.h:5-9
  inplace.r2c.transpose(data, d1, d2, d3)        include/transpose.h:11-15
  inplace.detail.rotate(fn, d3, d2, d1, data)    include/rotate.h:6-7
  inplace.detail.shuffle_fn(data, d3, d2, d1, fn) include/shuffle.h:5-6
  inplace.detail.col_shuffle_fn(fn, d3, d2, d1, data) include/col_shuffle.h:8-9
  inplace.detail.scatter_permute(fn, d3, d2, d1, data) include/permute.h:6-7
  inplace.detail.c2r.skinny_transpose(data, d1, d2, d3) include/skinny.h:9-10
  inplace.detail.r2c.skinny_transpose(data, d1, d2, d3) include/skinny.h:84-85
  functors inplace.detail.c2r.* / inplace.detail.r2c.* with the constructor
  arguments of include/equations.h and include/skinny.h.

`data` is a contiguous CUDA torch.Tensor (element size from its dtype, work on
its device's current stream) or a raw device pointer with elem_bytes=...
Where the reference exits or throws, these raise T213Error.
"""
from __future__ import annotations

import ctypes
from types import SimpleNamespace

from . import _lib
from ._lib import check, lib, params

_torch = None


def _t():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


def _resolve(data, elem_bytes=None, stream=None):
    """-> (pointer, element bytes, stream handle)"""
    if hasattr(data, "data_ptr"):
        torch = _t()
        if not data.is_cuda:
            raise ValueError("tensor must live on a CUDA device (use transpose_host for host tensors)")
        if not data.is_contiguous():
            raise ValueError("tensor must be contiguous")
        eb = data.element_size() if elem_bytes is None else int(elem_bytes)
        if stream is None:
            stream = torch.cuda.current_stream(data.device).cuda_stream
        elif hasattr(stream, "cuda_stream"):
            stream = stream.cuda_stream
        return ctypes.c_void_p(data.data_ptr()), eb, ctypes.c_void_p(int(stream))
    if elem_bytes is None:
        raise ValueError("elem_bytes is required with a raw pointer")
    if hasattr(stream, "cuda_stream"):
        stream = stream.cuda_stream
    return ctypes.c_void_p(int(data)), int(elem_bytes), ctypes.c_void_p(int(stream or 0))


class Functor:
    """An index functor of the decomposition: kind (include/t213.h t213_fn)
    plus the reference constructor's arguments."""

    kind = 0
    nparams = 0
    name = "functor"

    def __init__(self, *args):
        if len(args) != self.nparams:
            raise TypeError(f"{self.name} takes {self.nparams} arguments")
        self.params = tuple(int(a) for a in args)

    def __repr__(self):
        return f"{self.name}{self.params}"


def _fn(kind, nparams, name):
    return type(name, (Functor,), {"kind": kind, "nparams": nparams, "name": name})


# inplace::detail::c2r (include/equations.h, include/skinny.h)
_c2r_prerotator = _fn(1, 1, "c2r.prerotator")            # (b)
_c2r_postrotator = _fn(2, 1, "c2r.postrotator")          # (m)
_r2c_prerotator = _fn(3, 1, "r2c.prerotator")            # (m)
_r2c_postrotator = _fn(4, 2, "r2c.postrotator")          # (b, m)
_c2r_shuffle = _fn(10, 4, "c2r.shuffle")                 # (m, n, c, k)
_c2r_long_shuffle = _fn(11, 4, "c2r.long_shuffle")       # (m, n, c, k)
_r2c_shuffle = _fn(12, 4, "r2c.shuffle")                 # (m, n, c, k)
_c2r_fused_preop = _fn(20, 2, "c2r.fused_preop")         # (m, b)
_c2r_fused_postop = _fn(21, 3, "c2r.fused_postop")       # (m, n, c)
_r2c_fused_preop = _fn(22, 4, "r2c.fused_preop")         # (a, c, m, q)
_r2c_fused_postop = _fn(23, 2, "r2c.fused_postop")       # (m, b)
_c2r_postpermuter = _fn(30, 3, "c2r.postpermuter")       # (m, n, c)
_r2c_prepermuter = _fn(31, 3, "r2c.prepermuter")         # (m, n, c)


def _call_pass(cfn, fn: Functor, d3, d2, d1, data, elem_bytes=None, stream=None):
    p, eb, st = _resolve(data, elem_bytes, stream)
    prm = params(fn.params)
    check(cfn(fn.kind, prm, len(fn.params), p, int(d3), int(d2), int(d1), eb, st))


def rotate(fn, d3, d2, d1, data, *, elem_bytes=None, stream=None):
    """new[i][j] = old[(i + r(j)) mod d2][j] for every slice (src/rotate.cu:237-270)."""
    _call_pass(lib().t213_rotate, fn, d3, d2, d1, data, elem_bytes, stream)


def shuffle_fn(data, d3, d2, d1, fn, *, elem_bytes=None, stream=None):
    """new[i][j] = old[i][s_i(j)] (src/shuffle.cu:66-76, src/skinny.cu:237-280)."""
    _call_pass(lib().t213_row_shuffle, fn, d3, d2, d1, data, elem_bytes, stream)


def col_shuffle_fn(fn, d3, d2, d1, data, *, elem_bytes=None, stream=None):
    """new[i][j] = old[f(i,j)][j] (src/col_shuffle.cu:30-42, src/skinny.cu:282-309)."""
    _call_pass(lib().t213_col_shuffle, fn, d3, d2, d1, data, elem_bytes, stream)


def scatter_permute(fn, d3, d2, d1, data, *, elem_bytes=None, stream=None):
    """new[p(i)][*] = old[i][*] along precomputed cycles (src/permute.cu:116-137)."""
    _call_pass(lib().t213_scatter_permute, fn, d3, d2, d1, data, elem_bytes, stream)


def _shape_call(cfn, data, d1, d2, d3, elem_bytes=None, stream=None):
    p, eb, st = _resolve(data, elem_bytes, stream)
    check(cfn(p, int(d1), int(d2), int(d3), eb, st))


def transpose(data, d1, d2, d3, *, elem_bytes=None, stream=None):
    """In-place 213 transpose of a (d1,d2,d3) array (src/transpose.cu:99-124)."""
    _shape_call(lib().t213_transpose, data, d1, d2, d3, elem_bytes, stream)


def c2r_transpose(data, d1, d2, d3, *, elem_bytes=None, stream=None):
    """C2R on each d2 x d1 slice (src/transpose.cu:30-47)."""
    _shape_call(lib().t213_c2r_transpose, data, d1, d2, d3, elem_bytes, stream)


def r2c_transpose(data, d1, d2, d3, *, elem_bytes=None, stream=None):
    """R2C, the inverse of c2r_transpose(d1, d2) (src/transpose.cu:70-89)."""
    _shape_call(lib().t213_r2c_transpose, data, d1, d2, d3, elem_bytes, stream)


def skinny_c2r_transpose(data, d1, d2, d3, *, elem_bytes=None, stream=None):
    """Skinny C2R, d2 <= 32 (src/skinny.cu:313-333)."""
    _shape_call(lib().t213_skinny_c2r_transpose, data, d1, d2, d3, elem_bytes, stream)


def skinny_r2c_transpose(data, d1, d2, d3, *, elem_bytes=None, stream=None):
    """Skinny R2C, d2 <= 32 (src/skinny.cu:344-363)."""
    _shape_call(lib().t213_skinny_r2c_transpose, data, d1, d2, d3, elem_bytes, stream)


def transpose_with_plan(data, d1, d2, d3, plan, t=0, *, elem_bytes=None, stream=None):
    """The 213 transpose with an explicit plan family ('c2r', 'r2c', 'skinny',
    'blocks', 'bands', 'bands_t', 'identity' or 'auto') and block/band size t."""
    kind = _lib.PLAN_NAMES[plan] if isinstance(plan, str) else int(plan)
    p, eb, st = _resolve(data, elem_bytes, stream)
    check(lib().t213_transpose_with_plan(p, int(d1), int(d2), int(d3), eb, kind, int(t), st))


def permute(data, dims, perm, *, elem_bytes=None, stream=None):
    """In-place permutation of the axes of a rank-N array: dims[0] fastest,
    output axis j is input axis perm[j] (the reference's TensorUtil model,
    src/tensor_util.cpp:7-23,79-92); at most rank-1 213 transposes."""
    p, eb, st = _resolve(data, elem_bytes, stream)
    n = len(dims)
    if len(perm) != n:
        raise ValueError("dims and perm must have the same length")
    cd = (ctypes.c_int64 * max(1, n))(*[int(v) for v in dims])
    cp = (ctypes.c_int32 * max(1, n))(*[int(v) for v in perm])
    check(lib().t213_permute(p, n, cd, cp, eb, st))


def transpose_host(data, d1, d2, d3, *, elem_bytes=None, stream=None):
    """End-to-end transpose of a host buffer (torch CPU tensor, numpy array or
    raw pointer): copy in, transpose, copy out.  Synchronous."""
    if hasattr(data, "data_ptr") and not getattr(data, "is_cuda", False):
        ptr, eb = data.data_ptr(), data.element_size() if elem_bytes is None else elem_bytes
    elif hasattr(data, "ctypes"):
        ptr, eb = data.ctypes.data, data.itemsize if elem_bytes is None else elem_bytes
    else:
        ptr, eb = int(data), int(elem_bytes)
    st = ctypes.c_void_p(int(getattr(stream, "cuda_stream", stream) or 0))
    check(lib().t213_transpose_host(ctypes.c_void_p(ptr), int(d1), int(d2), int(d3), int(eb), st))


def describe(d1, d2, d3, elem_bytes, plan="auto", t=0) -> str:
    kind = _lib.PLAN_NAMES[plan] if isinstance(plan, str) else int(plan)
    buf = ctypes.create_string_buffer(1024)
    check(lib().t213_plan_describe(int(d1), int(d2), int(d3), int(elem_bytes), kind, int(t), buf, 1024))
    return buf.value.decode()


def plan_launches(d1, d2, d3, elem_bytes, plan="auto", t=0) -> int:
    kind = _lib.PLAN_NAMES[plan] if isinstance(plan, str) else int(plan)
    n = ctypes.c_int32(0)
    check(lib().t213_plan_launches(int(d1), int(d2), int(d3), int(elem_bytes), kind, int(t), ctypes.byref(n)))
    return int(n.value)


class pass_timing:
    """Per-pass CUDA-event timing of everything run while enabled."""

    @staticmethod
    def enable(on=True):
        check(lib().t213_pass_timing_enable(1 if on else 0))

    @staticmethod
    def reset():
        check(lib().t213_pass_timing_reset())

    @staticmethod
    def read(name):
        ms, n = ctypes.c_double(0), ctypes.c_int64(0)
        check(lib().t213_pass_timing_read(name.encode(), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value


class _Tuner:
    """The autotuner (t213_tune_shape, t213_tuner_*): per shape it times the
    applicable plan families, the winner's block or band size and the kernel
    variants of its passes, and caches the winner per exact shape and per
    shape class; the automatic plan choice (plan="auto") then uses it."""

    @staticmethod
    def tune(d1, d2, d3, elem_bytes, scratch=None, stream=None):
        """Tunes one shape on a scratch device buffer of the tensor's size
        (allocated here when not given); returns (plan name, block size)."""
        torch = _t()
        buf = scratch if scratch is not None else torch.empty(int(d1) * int(d2) * int(d3) * int(elem_bytes),
                                                              dtype=torch.uint8, device="cuda")
        kind, t = ctypes.c_int32(0), ctypes.c_int64(0)
        check(lib().t213_tune_shape(ctypes.c_void_p(buf.data_ptr()), int(d1), int(d2), int(d3), int(elem_bytes),
                                    _stream_of(stream), ctypes.byref(kind), ctypes.byref(t)))
        names = {v: k for k, v in _lib.PLAN_NAMES.items()}
        return names[int(kind.value)], int(t.value)

    @staticmethod
    def lookup(d1, d2, d3, elem_bytes):
        """(plan name, block size) cached for the shape, or None."""
        kind, t = ctypes.c_int32(0), ctypes.c_int64(0)
        rc = lib().t213_tuner_lookup(int(d1), int(d2), int(d3), int(elem_bytes), ctypes.byref(kind), ctypes.byref(t))
        if rc != _lib.OK:
            return None
        names = {v: k for k, v in _lib.PLAN_NAMES.items()}
        return names[int(kind.value)], int(t.value)

    @staticmethod
    def save(path):
        check(lib().t213_tuner_save(str(path).encode()))

    @staticmethod
    def load(path):
        check(lib().t213_tuner_load(str(path).encode()))

    @staticmethod
    def clear():
        check(lib().t213_tuner_clear())


tuner = _Tuner()


class Batch:
    """Many tensors transposed by one persistent, graph-captured launch
    (t213_batch_*).  `tensors` is a list of (data, d1, d2, d3) or
    (data, d1, d2, d3, elem_bytes[, plan]) tuples; data are CUDA tensors or raw
    device pointers (then elem_bytes is required)."""

    def __init__(self, tensors, tune=False):
        descs = []
        self._keep = []
        for t in tensors:
            data, d1, d2, d3 = t[:4]
            eb = t[4] if len(t) > 4 else None
            plan = t[5] if len(t) > 5 else "auto"
            p, eb, _ = _resolve(data, eb, 0)
            kind = _lib.PLAN_NAMES[plan] if isinstance(plan, str) else int(plan)
            descs.append(_lib.TensorDesc(p.value, int(d1), int(d2), int(d3), int(eb), kind))
            self._keep.append(data)
        self.count = len(descs)
        self._descs = (_lib.TensorDesc * max(1, self.count))(*descs)
        if tune:
            check(lib().t213_batch_tune(self._descs, self.count, _stream_of(None)))
        h = ctypes.c_void_p(0)
        check(lib().t213_batch_create(self._descs, self.count, ctypes.byref(h)))
        self._h = h

    def execute(self, stream=None):
        st = _stream_of(stream)
        check(lib().t213_batch_execute(self._h, st))

    def looped(self, stream=None):
        """The baseline: the plain call looped over the same list."""
        check(lib().t213_transpose_looped(self._descs, self.count, _stream_of(stream)))

    def status(self, stream=None) -> int:
        return int(lib().t213_batch_status(self._h, _stream_of(stream)))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(512)
        check(lib().t213_batch_describe(self._h, buf, 512))
        return buf.value.decode()

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().t213_batch_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving form (include/t213_serve.h): HBM-budget admission into a
    device arena, continuous dispatch onto a stream pool, p50/p99 latency."""

    def __init__(self, hbm_budget_bytes=150 * 10**9, max_inflight=64, streams=8):
        h = ctypes.c_void_p(0)
        check(lib().t213_server_create(int(hbm_budget_bytes), int(max_inflight), int(streams), ctypes.byref(h)))
        self._h = h

    @staticmethod
    def _requests(reqs):
        arr = (_lib.Request * max(1, len(reqs)))()
        for i, r in enumerate(reqs):
            kind = r.get("plan", "auto")
            kind = _lib.PLAN_NAMES[kind] if isinstance(kind, str) else int(kind)
            arr[i] = _lib.Request(int(r["d1"]), int(r["d2"]), int(r["d3"]), int(r["elem_bytes"]), kind,
                                  float(r.get("t", r.get("arrival_s", 0.0))), int(r.get("seed", i + 1)))
        return arr

    def run(self, reqs, capture=None):
        """Replays the schedule; returns (stats dict, checksums, latencies_ms).
        `capture` maps request indices to writable host buffers (numpy arrays
        or pinned torch tensors of the request's byte size) that receive the
        transposed tensor."""
        n = len(reqs)
        arr = self._requests(reqs)
        st = _lib.ServeStats()
        sums = (ctypes.c_uint64 * max(1, n))()
        lat = (ctypes.c_double * max(1, n))()
        outs = None
        if capture:
            outs = (ctypes.c_void_p * max(1, n))()
            for i, buf in capture.items():
                r = reqs[i]
                need = int(r["d1"]) * int(r["d2"]) * int(r["d3"]) * int(r["elem_bytes"])
                if hasattr(buf, "data_ptr"):
                    size, ptr = buf.numel() * buf.element_size(), buf.data_ptr()
                else:
                    size, ptr = buf.nbytes, buf.ctypes.data
                if size < need:
                    raise ValueError(f"capture buffer of request {i} holds {size} bytes, needs {need}")
                outs[i] = ptr
        check(lib().t213_server_run_capture(self._h, arr, n, ctypes.byref(st), sums, lat, outs))
        stats = {f: getattr(st, f) for f, _ in _lib.ServeStats._fields_}
        return stats, list(sums)[:n], list(lat)[:n]

    def expected_checksum(self, req) -> int:
        arr = self._requests([req])
        v = ctypes.c_uint64(0)
        check(lib().t213_server_expected_checksum(self._h, arr, ctypes.byref(v)))
        return int(v.value)

    def run_alone(self, req) -> int:
        arr = self._requests([req])
        v = ctypes.c_uint64(0)
        check(lib().t213_server_run_alone(self._h, arr, ctypes.byref(v)))
        return int(v.value)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().t213_server_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stream_of(stream):
    if stream is None:
        torch = _t()
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(int(getattr(stream, "cuda_stream", stream)))


def device_status(stream=None) -> int:
    v = ctypes.c_int32(0)
    check(lib().t213_device_status(_stream_of(stream), ctypes.byref(v)))
    return int(v.value)


def release_cache():
    check(lib().t213_release_cache())


inplace = SimpleNamespace(
    transpose=transpose,
    c2r=SimpleNamespace(transpose=c2r_transpose),
    r2c=SimpleNamespace(transpose=r2c_transpose),
    detail=SimpleNamespace(
        rotate=rotate,
        shuffle_fn=shuffle_fn,
        col_shuffle_fn=col_shuffle_fn,
        scatter_permute=scatter_permute,
        c2r=SimpleNamespace(
            prerotator=_c2r_prerotator, postrotator=_c2r_postrotator, shuffle=_c2r_shuffle,
            long_shuffle=_c2r_long_shuffle, postpermuter=_c2r_postpermuter,
            scatter_postpermuter=_r2c_prepermuter, fused_preop=_c2r_fused_preop,
            fused_postop=_c2r_fused_postop, skinny_transpose=skinny_c2r_transpose),
        r2c=SimpleNamespace(
            prerotator=_r2c_prerotator, postrotator=_r2c_postrotator, shuffle=_r2c_shuffle,
            prepermuter=_r2c_prepermuter, scatter_prepermuter=_c2r_postpermuter,
            fused_preop=_r2c_fused_preop, fused_postop=_r2c_fused_postop,
            skinny_transpose=skinny_r2c_transpose),
    ),
)
