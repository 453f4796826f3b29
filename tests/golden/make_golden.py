#!/usr/bin/env python3
"""Regenerates the golden fixtures in tests/golden/ from the reference tree.

Run in a container that has the reference tree, named by the environment
variable PYRO_REFERENCE_DIR (required). Nothing under tests/ reads the reference at
test time: the tests read only the JSON files this script writes.

* geometry_tables.json -- the reference's own integer tables, parsed as text
  from include/pyrochlore_geometry.hpp (nn1_dist, nn2_dist, nn3a_dist,
  nn3b_dist, nn1_pair_MN, pyro, fcc_Dy) and the 16-site cubic cell of
  PyroCubicCell (:12-32).
* xoshiro_streams.json -- draws of the reference's own RNG header
  include/XoshiroCpp.hpp (Xoroshiro128++ seeded through SplitMix64) through the
  libstdc++ normal and uniform distributions MC_runner uses, produced by the
  program oracle/make_ref.sh compiles from that header.
* philox_kat.json -- published known-answer vectors of Philox4x32-10
  (Random123 distribution, kat_vectors), the counter-based RNG of the GPU path.
"""
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("PYRO_REFERENCE_DIR", "")


def _strip_comments(src):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _parse_braces(text, start):
    """Parse a nested brace initialiser starting at text[start] == '{'.
    Returns (nested list of ints, index after the closing brace)."""
    assert text[start] == "{"
    out = []
    i = start + 1
    num = ""
    while i < len(text):
        ch = text[i]
        if ch == "{":
            sub, i = _parse_braces(text, i)
            out.append(sub)
            continue
        if ch in "-0123456789":
            num += ch
        else:
            if num:
                out.append(int(num))
                num = ""
            if ch == "}":
                return out, i + 1
        i += 1
    raise ValueError("unbalanced braces")


def parse_geometry(path):
    src = _strip_comments(open(path).read())
    tables = {}
    for name in ["nn1_dist", "nn2_dist", "nn3a_dist", "nn3b_dist", "nn1_pair_01", "nn1_pair_02",
                 "nn1_pair_03", "nn1_pair_12", "nn1_pair_13", "nn1_pair_23"]:
        m = re.search(r"\b%s\s*=\s*\{" % name, src)
        if not m:
            raise KeyError(name)
        val, _ = _parse_braces(src, m.end() - 1)
        tables[name] = val
    for name in ["pyro", "fcc_Dy"]:
        m = re.search(r"\bidx3_t\s+%s\s*\[\s*4\s*\]\s*=\s*\{" % name, src)
        val, _ = _parse_braces(src, m.end() - 1)
        tables[name] = val
    # PyroCubicCell: R_fcc and link_positions inside the factory (:16-21)
    body = src[src.index("PyroCubicCell()"):src.index("PrimitiveCell()")]
    for name in ["R_fcc", "link_positions"]:
        m = re.search(r"\b%s\s*\[\s*4\s*\]\s*=\s*\{" % name, body)
        val, _ = _parse_braces(body, m.end() - 1)
        tables["PyroCubicCell_" + name] = val
    return tables


def xoshiro_streams():
    subprocess.run([os.path.join(REPO, "oracle", "make_ref.sh")], check=True)
    exe = os.path.join(REPO, "oracle", "_ref", "xoshiro_golden")
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    rows = []
    for line in out.split("\n"):
        if not line.strip():
            continue
        seed, kind, idx, val = line.split()
        rows.append({"seed": int(seed), "kind": int(kind), "index": int(idx),
                     "value": int(val) if kind == "0" else float(val)})
    return rows


PHILOX_KAT = [
    # (counter[4], key[2], output[4]) -- Random123 kat_vectors, philox4x32 10 rounds
    ([0x00000000, 0x00000000, 0x00000000, 0x00000000], [0x00000000, 0x00000000],
     [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff], [0xffffffff, 0xffffffff],
     [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
]


def main():
    if not REF or not os.path.isdir(REF):
        sys.exit("set PYRO_REFERENCE_DIR to the reference tree")
    geo = parse_geometry(os.path.join(REF, "include", "pyrochlore_geometry.hpp"))
    geo["_source"] = "include/pyrochlore_geometry.hpp (parsed as text by tests/golden/make_golden.py)"
    with open(os.path.join(HERE, "geometry_tables.json"), "w") as f:
        json.dump(geo, f, indent=1)
    rows = xoshiro_streams()
    with open(os.path.join(HERE, "xoshiro_streams.json"), "w") as f:
        json.dump({"_source": "include/XoshiroCpp.hpp via oracle/ref_xoshiro_main.cpp", "draws": rows}, f)
    with open(os.path.join(HERE, "philox_kat.json"), "w") as f:
        json.dump({"_source": "Random123 kat_vectors, philox4x32 R=10",
                   "vectors": [{"ctr": c, "key": k, "out": o} for c, k, o in PHILOX_KAT]}, f, indent=1)
    print("wrote golden fixtures to", HERE)


if __name__ == "__main__":
    sys.exit(main())
