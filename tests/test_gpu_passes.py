"""Parity of the pass-level entry points (inplace::detail::rotate,
shuffle_fn, col_shuffle_fn, scatter_permute; include/rotate.h,
include/shuffle.h, include/col_shuffle.h, include/permute.h of the reference)
with the oracle's restatement of each pass, for every functor kind, on short
and tall matrices: tall ones take the cluster-local column kernel (strips
split over a thread-block cluster, halo rows per CTA), short ones the staged
single-CTA kernel.  Also functor parameters that do not belong to the matrix
(plain gather semantics must hold).  Bit-exact."""
import math

import numpy as np
import pytest

from conftest import from_device, to_device

pytestmark = pytest.mark.gpu

# (d3, m, n): m rows, n columns per slice
COL_SHAPES = [(2, 37, 53), (1, 900, 37), (2, 1537, 300), (1, 3000, 64), (1, 6151, 96), (2, 2048, 384),
              (1, 4096, 30), (3, 1001, 1001), (1, 12000, 40), (1, 40000, 16), (1, 100003, 8)]
ROW_SHAPES = [(2, 37, 53), (3, 97, 300), (1, 40, 7919), (2, 300, 2048), (1, 6, 60000), (2, 5, 200003)]
EBS = (4, 8, 16, 1, 2)


def params_for(kind, m, n, O):
    c = math.gcd(m, n)
    a, b = m // c, n // c
    if kind == 1:
        return (b,)
    if kind in (2, 3):
        return (m,)
    if kind == 4:
        return (b, m)
    if kind in (10, 11):
        k = O.ext_gcd(a, b)[1] if c > 1 else O.ext_gcd(m, n)[1]
        return (m, n, c, k)
    if kind == 12:
        return (m, n, c, 0)
    if kind in (20, 23):
        return (m, b)
    if kind == 21:
        return (m, n, c)
    if kind == 22:
        q = O.ext_gcd(b, a)[1] if c > 1 else O.ext_gcd(n, m)[1]
        return (a, c, m, q)
    if kind in (30, 31):
        return (m, n, c)
    raise ValueError(kind)


def run_pass(cuda, O, t213, which, kind, prm, d3, m, n, eb, seed=0):
    x = O.random_bits(d3 * m * n, eb, seed + kind)
    want = x.view(np.uint8).copy()
    getattr(O, which)(kind, prm, want, d3, m, n, eb)
    dev = to_device(cuda, x)
    fn = type("F", (t213.api.Functor,), {"kind": kind, "nparams": len(prm), "name": f"kind{kind}"})(*prm)
    gpu = {"rotate": lambda: t213.rotate(fn, d3, m, n, dev, elem_bytes=eb),
           "col_shuffle": lambda: t213.col_shuffle_fn(fn, d3, m, n, dev, elem_bytes=eb),
           "row_shuffle": lambda: t213.shuffle_fn(dev, d3, m, n, fn, elem_bytes=eb),
           "scatter_permute": lambda: t213.scatter_permute(fn, d3, m, n, dev, elem_bytes=eb)}[which]
    gpu()
    cuda.cuda.synchronize()
    got = from_device(dev)
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, f"{which} kind {kind} {prm} on {(d3, m, n, eb)}: {bad.size} bytes differ"


@pytest.mark.parametrize("eb", EBS)
@pytest.mark.parametrize("kind", (1, 2, 3, 4))
@pytest.mark.parametrize("shape", COL_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_rotate(cuda, oracle, t213, shape, kind, eb):
    d3, m, n = shape
    run_pass(cuda, oracle, t213, "rotate", kind, params_for(kind, m, n, oracle), d3, m, n, eb)


@pytest.mark.parametrize("eb", EBS)
@pytest.mark.parametrize("kind", (20, 21, 22, 23))
@pytest.mark.parametrize("shape", COL_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_col_shuffle(cuda, oracle, t213, shape, kind, eb):
    d3, m, n = shape
    run_pass(cuda, oracle, t213, "col_shuffle", kind, params_for(kind, m, n, oracle), d3, m, n, eb)


@pytest.mark.parametrize("variant", ("old", "local"))
@pytest.mark.parametrize("kind", (1, 2, 3, 4, 20, 21, 22, 23))
def test_col_kernels_agree(cuda, oracle, t213, monkeypatch, kind, variant):
    """Both column kernels, forced, on a mid-size matrix (the local kernel as
    a single CTA holding the whole strip plus its halo)."""
    monkeypatch.setenv("T213_COL_VARIANT", variant)
    d3, m, n = 2, 600, 200
    which = "rotate" if kind < 10 else "col_shuffle"
    for eb in (4, 8):
        run_pass(cuda, oracle, t213, which, kind, params_for(kind, m, n, oracle), d3, m, n, eb)


@pytest.mark.parametrize("shape", [(1, 3000, 64), (2, 2048, 384)], ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("wbytes,k", [(64, 0), (128, 2), (256, 0), (256, 16), (128, 5)])
def test_local_launch_shapes(cuda, oracle, t213, monkeypatch, shape, wbytes, k):
    """Strip widths and cluster sizes of the cluster-local kernel."""
    monkeypatch.setenv("T213_COL_LOCAL_WBYTES", str(wbytes))
    if k:
        monkeypatch.setenv("T213_COL_LOCAL_K", str(k))
    d3, m, n = shape
    for kind in (2, 21, 22):
        which = "rotate" if kind < 10 else "col_shuffle"
        run_pass(cuda, oracle, t213, which, kind, params_for(kind, m, n, oracle), d3, m, n, 4)


@pytest.mark.parametrize("kind,prm", [(21, (3000, 64, 1)), (21, (3000, 48, 8)), (22, (1000, 3, 3000, 2)),
                                      (22, (3000, 1, 3000, 0)), (20, (3000, 7)), (23, (3000, 5))])
def test_col_shuffle_foreign_params(cuda, oracle, t213, kind, prm):
    """Parameters that are not the decomposition's own for this matrix (a c
    that is not gcd(m, n'), a pre-permuter q that is no unit): the pass is
    still the plain gather new[i][j] = old[f(i,j)][j]."""
    run_pass(cuda, oracle, t213, "col_shuffle", kind, prm, 1, 3000, 64, 4)


@pytest.mark.parametrize("kind,prm", [(21, (2999, 64, 1)), (23, (3001, 7)), (20, (0, 3))])
def test_col_shuffle_rejects_other_m(cuda, t213, kind, prm):
    """A functor whose m is not the slice's row count is refused."""
    dev = cuda.zeros(3000 * 64 * 4, dtype=cuda.uint8, device="cuda")
    fn = type("F", (t213.api.Functor,), {"kind": kind, "nparams": len(prm), "name": f"kind{kind}"})(*prm)
    with pytest.raises(t213.T213Error) as e:
        t213.col_shuffle_fn(fn, 1, 3000, 64, dev, elem_bytes=4)
    assert e.value.status == 1


@pytest.mark.parametrize("eb", EBS)
@pytest.mark.parametrize("kind", (10, 11, 12))
@pytest.mark.parametrize("shape", ROW_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_row_shuffle(cuda, oracle, t213, shape, kind, eb):
    d3, m, n = shape
    run_pass(cuda, oracle, t213, "row_shuffle", kind, params_for(kind, m, n, oracle), d3, m, n, eb)


@pytest.mark.parametrize("variant,stage_kb", [("old", 0), ("pipe", 8), ("pipe", 24), ("pipe", 96), ("cluster", 0),
                                              ("scratch", 0)])
@pytest.mark.parametrize("kind", (10, 12))
def test_row_kernels(cuda, oracle, t213, monkeypatch, kind, variant, stage_kb):
    """The staged and the double-buffered row kernels, several unit sizes
    (one row per unit up to many), odd row lengths and row counts."""
    monkeypatch.setenv("T213_ROW_VARIANT", variant)
    if stage_kb:
        monkeypatch.setenv("T213_ROW_STAGE_KB", str(stage_kb))
    for d3, m, n, eb in ((2, 97, 300, 4), (1, 301, 1001, 8), (3, 40, 7919, 8), (1, 1000, 33, 16), (2, 77, 513, 2),
                         (1, 4, 70001, 4), (2, 3, 30011, 8)):
        run_pass(cuda, oracle, t213, "row_shuffle", kind, params_for(kind, m, n, oracle), d3, m, n, eb)


@pytest.mark.parametrize("eb", (4, 8, 16, 1))
@pytest.mark.parametrize("kind", (30, 31))
@pytest.mark.parametrize("shape", [(2, 37, 53), (1, 900, 37), (2, 1537, 300), (1, 6000, 32)],
                         ids=lambda s: "x".join(map(str, s)))
def test_scatter_permute(cuda, oracle, t213, shape, kind, eb):
    d3, m, n = shape
    run_pass(cuda, oracle, t213, "scatter_permute", kind, params_for(kind, m, n, oracle), d3, m, n, eb)
