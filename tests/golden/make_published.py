"""Writes reference_published.json: the numbers the reference project
publishes for its own force path, read from its text files (the reference is
a Rust workspace that cannot be built here, so these printed results are the
golden values the oracle and the engine are pinned to).

Run from the repository root with the reference checked out at REF (default
/root/reference):  python tests/golden/make_published.py [REF]
"""

import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))


def line_of(path, pattern):
    with open(os.path.join(REF, path)) as f:
        for i, line in enumerate(f, 1):
            if re.search(pattern, line):
                return i, line
    raise SystemExit(f"{path}: no line matches {pattern!r}")


def main():
    out = {}
    i, line = line_of("todo.md", r"Release exit gate unchanged: max_s")
    m = re.search(r"max_s ([0-9.e-]+), rms_s ([0-9.e-]+)", line)
    out["exit_gate_n1e4"] = {
        "max_s": float(m.group(1)), "rms_s": float(m.group(2)),
        "printed_digits": {"max_s": 6, "rms_s": 8},
        "case": "tests/exit_gate.rs:11-24: plummer(10000, seed 2024), p = 5, eps = 1e-5, leaf 32, "
                "scaled errors against the direct sum",
        "source": f"todo.md:{i}"}
    i, line = line_of("PERF-ANALYSIS.md", r"Corrected walk stats at N=")
    with open(os.path.join(REF, "PERF-ANALYSIS.md")) as f:
        text = " ".join(f.read().splitlines()[i - 1:i + 2])
    pops = re.search(r"pops = ([0-9.]+)M", text).group(1)
    m2l = re.search(r"accepted\s+M2L pairs = ([0-9.]+)M", text).group(1)
    p2p = re.search(r"P2P leaf-pair calls = ([0-9.]+)M", text).group(1)
    leaves = re.search(r"leaves =\s*([0-9,]+)", text).group(1).replace(",", "")
    out["walk_stats_n1e6"] = {
        "pops_millions": float(pops), "m2l_pairs_millions": float(m2l), "p2p_calls_millions": float(p2p),
        "leaves": int(leaves), "printed_digits": {"pops_millions": 1, "m2l_pairs_millions": 1, "p2p_calls_millions": 2},
        "case": "crates/bench profile mode (crates/bench/src/main.rs:554-641): plummer(1e6, seed 42), p = 8, "
                "eps = 1e-5, leaf 16; P2P calls count leaf pairs apart from the self pairs",
        "source": f"PERF-ANALYSIS.md:{i}-{i + 2}"}
    with open(os.path.join(HERE, "reference_published.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
