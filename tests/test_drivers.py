"""The drivers' raw output files (test_213inplace, gen_ans; same argv and
format as the reference's, src/test_213inplace.cu:66-90, src/gen_ans.cpp:21-43)
and the compare / dump tools of the CLI.  CPU: the tools on files written
here.  GPU: both drivers against the reference's own gen_ans output committed
under tests/golden (bit-exact)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "213transpose_b200", "bin")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def cli(*args):
    return subprocess.run([sys.executable, "-m", "213transpose_b200.cli", *map(str, args)], cwd=ROOT,
                          capture_output=True, text=True)


def test_compare_and_dump_tools(tmp_path):
    d1, d2, d3 = 7, 5, 3
    a = np.arange(d1 * d2 * d3, dtype=np.int32)
    b = a.copy()
    b[2 * d1 * d2 + 1 * d2 + 4] = -1  # slice 2, row i1 = 1, column i2 = 4
    pa, pb = tmp_path / "a.bin", tmp_path / "b.bin"
    a.tofile(pa)
    b.tofile(pb)
    r = cli("compare", pa, pa, d1, d2, d3, 4)
    assert r.returncode == 0 and json.loads(r.stdout)["mismatches"] == 0
    r = cli("compare", pa, pb, d1, d2, d3, 4)
    out = json.loads(r.stdout)
    assert r.returncode == 1 and out["mismatches"] == 1
    assert out["first"] == {"index": 2 * d1 * d2 + d2 + 4, "i2": 4, "i1": 1, "i3": 2}
    r = cli("compare", pa, pb, d1, d2, 2, 4)  # wrong size
    assert r.returncode != 0
    r = cli("dump", pa, d1, d2, d3, 4, "--slice", 1, "--rows", 2)
    assert r.returncode == 0 and r.stdout.split("\n")[0].split()[0] == str(d1 * d2)


def _driver_vs_golden(tmp_path, driver):
    for name in sorted(os.listdir(GOLDEN)):
        if not name.startswith("gen_ans_") or not name.endswith(".bin"):
            continue
        d1, d2, d3, ts = (int(v) for v in name[len("gen_ans_"):-len(".bin")].split("_"))
        out = tmp_path / f"{driver}_{name}"
        r = subprocess.run([os.path.join(BIN, driver), str(d1), str(d2), str(d3), str(ts), str(out)],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        c = cli("compare", out, os.path.join(GOLDEN, name), d1, d2, d3, ts)
        assert c.returncode == 0, (name, c.stdout, c.stderr)


@pytest.mark.gpu
def test_test_213inplace_matches_reference_gen_ans(tmp_path):
    """The GPU driver against the reference's own gen_ans output."""
    _driver_vs_golden(tmp_path, "test_213inplace")


def test_gen_ans_matches_reference_gen_ans(tmp_path):
    """This project's host answer generator (no GPU code) against the
    reference's own gen_ans output, byte for byte."""
    _driver_vs_golden(tmp_path, "gen_ans")
