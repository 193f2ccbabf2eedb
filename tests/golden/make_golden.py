"""Generates tests/golden/reference_examples.json from the reference tree.

Run where the reference tree is checked out, with its path as the first
argument or in the environment variable SCYCLE_REFERENCE.  The fixture holds facts derived from
the reference's shipped inputs -- the key/value settings of the
linear-elastic quasi-dynamic example examples/ex2.in as its own parser
reads them, and summary values of the PETSc-binary vector examples/ex3_z --
plus the root of the reference's known-answer residual TestRoots
(source/rootFinder.cpp:12-24), bracketed by plain bisection.  No reference
file is copied.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.infile import load_vector_double, load_vector_string, parse_lines, read_petsc_vecs  # noqa: E402
from oracle.fault import known_answer_resid  # noqa: E402


def main(ref):
    out = {}
    text = open(os.path.join(ref, "examples", "ex2.in")).read()
    entries = []
    for var, rhs, full in parse_lines(text):
        if not var or var.startswith("#") or var.startswith("%"):
            continue
        if full.startswith("["):
            vals = load_vector_string(full) if var == "timeIntInds" else load_vector_double(full)
            entries.append([var, "list", vals])
        elif rhs != "":
            entries.append([var, "scalar", rhs])
    out["ex2_settings"] = entries
    z = read_petsc_vecs(os.path.join(ref, "examples", "ex3_z"))
    v = z[0]
    out["ex3_z"] = dict(records=len(z), n=int(v.size), min=float(v.min()), max=float(v.max()),
                        sum=float(v.sum()), first=[float(x) for x in v[:5]],
                        col_first=[float(x) for x in v[755:760]], nz_guess=757, ny_guess=301)
    lo, hi = 0.0, 10.0
    assert known_answer_resid(lo) < 0 < known_answer_resid(hi)
    for _ in range(400):
        mid = 0.5 * (lo + hi)
        if known_answer_resid(mid) < 0:
            lo = mid
        else:
            hi = mid
    out["test_roots"] = dict(root=0.5 * (lo + hi), resid_at_root=float(known_answer_resid(0.5 * (lo + hi))))
    with open(os.path.join(HERE, "reference_examples.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SCYCLE_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference tree>  (or set SCYCLE_REFERENCE)")
    main(ref)
