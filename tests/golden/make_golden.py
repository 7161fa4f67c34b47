"""Generates the golden fixtures in this directory from the reference's own CPU
answer generator.

``gen_ans d1 d2 d3 type_size out`` (src/gen_ans.cpp:21-43, built from the
reference's sources by oracle/Makefile into oracle/_ref/gen_ans) writes the
213 transpose of the ramp data[i] = i as raw int32 (type_size 4) or int64
(otherwise) bytes.  Small shapes are committed as .bin files; larger ones are
recorded only by their SHA-256 in manifest.json.

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
GEN_ANS = os.path.join(ROOT, "oracle", "_ref", "gen_ans")

# (d1, d2, d3, type_size): committed as files
SMALL = [
    (7, 5, 3, 4), (33, 40, 2, 4), (64, 48, 4, 8), (3, 97, 2, 4), (100, 37, 1, 8),
    (97, 3, 2, 4), (35, 35, 1, 8), (120, 300, 1, 4), (1, 7, 2, 4), (64, 64, 2, 4),
    (600, 45, 1, 4), (40, 600, 1, 8), (2, 2, 1, 4), (31, 33, 3, 8), (256, 192, 1, 4),
]
# recorded by digest only
LARGE = [(512, 384, 16, 4), (1000, 999, 1, 8), (8192, 6, 3, 4), (96, 4096, 2, 8)]


def run_gen_ans(d1, d2, d3, ts, path):
    subprocess.run([GEN_ANS, str(d1), str(d2), str(d3), str(ts), path], check=True)


def main():
    if not os.path.exists(GEN_ANS):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-cpu"], check=True)
    manifest = {"generator": "reference gen_ans (src/gen_ans.cpp) on the ramp data[i]=i",
                "cases": []}
    for d1, d2, d3, ts in SMALL + LARGE:
        name = f"gen_ans_{d1}_{d2}_{d3}_{ts}.bin"
        small = (d1, d2, d3, ts) in SMALL
        if small:
            path = os.path.join(HERE, name)
            run_gen_ans(d1, d2, d3, ts, path)
            data = open(path, "rb").read()
        else:
            with tempfile.TemporaryDirectory() as td:
                path = os.path.join(td, name)
                run_gen_ans(d1, d2, d3, ts, path)
                data = open(path, "rb").read()
        manifest["cases"].append({"d1": d1, "d2": d2, "d3": d3, "type_size": ts,
                                  "file": name if small else None,
                                  "bytes": len(data),
                                  "sha256": hashlib.sha256(data).hexdigest()})
        print(name, len(data), "committed" if small else "digest only", file=sys.stderr)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
