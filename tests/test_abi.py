"""CPU tests of the boundary: the C-ABI library loads without a GPU, exports
every function its headers declare, and rejects bad arguments with status
codes (never exits, never throws).  The planner runs on the host and picks
the expected plan family for each configuration of the workload."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_function(t213):
    L = t213.lib()
    names = t213.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_static_library_and_cxx_header_present():
    hdr = open(os.path.join(ROOT, "include", "transpose.h")).read()
    for decl in ("template <typename T> void transpose(T* data, int d1, int d2, int d3);",):
        assert decl in hdr.replace("  ", " ")


def test_status_strings(t213):
    L = t213.lib()
    for s in range(8):
        assert L.t213_status_string(s)
    assert L.t213_version().startswith(b"213transpose_b200")


@pytest.mark.parametrize("args,status", [
    ((0, -1, 2, 1, 4), 1),      # negative dimension
    ((0, 3, 2, 1, 3), 2),       # 3-byte elements
    ((0, 3, 2, 1, 32), 2),      # 32-byte elements
    ((0, 3, 2, 1, 4), 1),       # NULL data with work to do
    ((6, 3, 2, 1, 4), 1),       # misaligned pointer for 4-byte elements
])
def test_transpose_rejects_bad_arguments(t213, args, status):
    L = t213.lib()
    ptr, d1, d2, d3, eb = args
    assert L.t213_transpose(ctypes.c_void_p(ptr), d1, d2, d3, eb, None) == status
    assert L.t213_last_error()


def test_empty_tensor_is_a_no_op(t213):
    L = t213.lib()
    for shape in ((0, 5, 2), (5, 0, 2), (5, 5, 0)):
        assert L.t213_transpose(None, *shape, 4, None) == 0


def test_pass_entry_points_validate_functors(t213):
    L = t213.lib()
    prm = (ctypes.c_int64 * 4)(0, 0, 0, 0)
    # rotator kind passed to the row shuffle, unknown kinds, negative params
    assert L.t213_row_shuffle(1, prm, 1, ctypes.c_void_p(256), 1, 4, 4, 4, None) == 1
    assert L.t213_rotate(99, prm, 1, ctypes.c_void_p(256), 1, 4, 4, 4, None) == 1
    assert L.t213_col_shuffle(3, prm, 1, ctypes.c_void_p(256), 1, 4, 4, 4, None) == 1
    neg = (ctypes.c_int64 * 4)(-1, 0, 0, 0)
    assert L.t213_scatter_permute(30, neg, 3, ctypes.c_void_p(256), 1, 4, 4, 4, None) == 1


def test_plan_kind_validation(t213):
    L = t213.lib()
    assert L.t213_transpose_with_plan(ctypes.c_void_p(256), 4, 4, 1, 4, 42, 0, None) == 1
    assert L.t213_transpose_with_plan(ctypes.c_void_p(256), 4, 4, 1, 4, 4, -3, None) == 1


CONFIG_PLANS = [
    # (d1, d2, d3, eb): expected plan family of the dispatcher
    ((8192, 6144, 4, 4), "blocks t=2048"),
    ((7919, 6151, 2, 8), "c2r"),
    ((512, 384, 16, 4), "slice: slice("),
    ((32, 1 << 24, 1, 4), "bands t="),
    ((1 << 24, 48, 1, 4), "bands_t t="),
    ((3, 1 << 22, 8, 4), "bands t="),
    ((1024, 1024, 1, 16), "blocks t=1024: tile_swap(t=1024)"),
    ((1, 1000, 3, 4), "identity"),
    ((1000, 1, 3, 8), "identity"),
]


@pytest.mark.parametrize("shape", [(7919, 6151, 2, 8), (8192, 6143, 2, 4), (6151, 7919, 2, 8)])
def test_tall_column_passes_use_the_cluster_local_kernel(t213, shape):
    """Coprime configurations take the cluster-local column gather with
    128-byte strips split over a cluster."""
    import re
    desc = t213.describe(*shape)
    m = re.search(r"\[local W=(\d+) cluster=(\d+)", desc)
    assert m, desc
    assert int(m.group(1)) * shape[3] == 128 and int(m.group(2)) >= 2, desc


@pytest.mark.parametrize("shape,prefix", CONFIG_PLANS, ids=lambda v: str(v))
def test_planner_choices(t213, shape, prefix):
    desc = t213.describe(*shape)
    assert desc.startswith(prefix), desc


def test_plan_families_on_cpu(t213):
    """Every family builds its pass list (and cycle tables) without a GPU."""
    d = t213.describe(512, 384, 2, 4, "c2r")
    assert d.startswith("c2r:") and d.count("gather") == 3
    d = t213.describe(384, 512, 2, 4, "r2c")
    assert d.startswith("r2c:") and d.count("gather") == 3
    d = t213.describe(7919, 6151, 1, 8, "r2c")
    assert d.count("gather") == 2  # coprime: no post-rotation
    d = t213.describe(600, 30, 1, 4, "skinny")
    assert d.startswith("skinny:")
    with pytest.raises(t213.T213Error):
        t213.describe(600, 300, 1, 4, "skinny")
    with pytest.raises(t213.T213Error):
        t213.describe(601, 300, 1, 4, "blocks", 7)


def test_launch_counts(t213):
    # blocks plan: tile swap + carry + walker; square: one launch
    assert t213.plan_launches(1024, 1024, 1, 16) == 1
    assert t213.plan_launches(8192, 6144, 4, 4) in (2, 3)
    assert t213.plan_launches(7919, 6151, 2, 8) == 2


def test_describe_names_the_peeled_column_kernel(t213):
    """Column passes over a pitch that is not a 16-byte multiple take the
    peeled cluster-local kernel for 4- and 8-byte elements; a 16-byte pitch
    keeps the plain one."""
    d = t213.describe(7919, 6151, 2, 8, "c2r")
    assert "[local W=16 cluster" in d and "peeled]" in d, d
    d = t213.describe(7919, 601, 1, 4, "r2c")
    assert "col_gather(fn=22)[local W=32" in d and "aw=16 peeled]" in d, d
    d = t213.describe(8192, 6143, 2, 4, "c2r")
    assert "col_gather(fn=21)[local W=32 cluster" in d and "peeled" not in d, d
