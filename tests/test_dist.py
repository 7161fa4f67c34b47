"""The bench's multi-process path on the CPU: two gloo ranks on 127.0.0.1
rendezvous as torchrun would set them up, take the max of their step times,
aggregate the whole-job throughput, and leave the reference arm to rank 0."""
import contextlib
import importlib.util
import io
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    b = _bench()
    dist, r, w, local = b.init_dist(world, backend="gloo")
    try:
        b.barrier(dist, device="cpu")
        ms = b.max_over_ranks(dist, 10.0 + r, device="cpu")  # rank 1 is the slower one
        value = b.whole_job_gbps(w, 1 << 20, 4, ms)
        args = type("A", (), {"gpus": w, "steps": 1, "warmup": 0})()
        buf = io.StringIO()
        if r != 0:
            with contextlib.redirect_stdout(buf):
                b.run_reference(args)  # only rank 0 runs the reference arm
        out.put((r, w, ms, value, buf.getvalue()))
        b.barrier(dist, device="cpu")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2, 2]
    assert all(r[2] == pytest.approx(11.0) for r in res)  # the max over ranks
    want = 2 * 2 * (1 << 20) * 4 / (11.0e-3) / 1e9
    assert all(r[3] == pytest.approx(want) for r in res)
    assert res[1][4] == ""  # rank 1 printed nothing for the reference arm


def test_single_process_needs_no_rendezvous():
    b = _bench()
    assert b.init_dist(1) == (None, 0, 1, 0)
    assert b.max_over_ranks(None, 3.5) == 3.5
    assert b.whole_job_gbps(1, 805306368, 20, 11.0) == pytest.approx(2 * 805306368 * 20 / 11e-3 / 1e9)
