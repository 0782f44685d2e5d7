"""Record the line count of every MATLAB source file of the xSPDE reference.

Usage: python make_reference_line_counts.py <reference checkout>
(or set XSPDE_REFERENCE).  Writes reference_line_counts.json beside this
script: {"path/within/project.m": lines}.  tests/test_citations_cpu.py uses it
to check that every file:line citation in this repository points inside the
file it names, without needing the reference checkout at test time.
"""
import json
import os
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("XSPDE_REFERENCE")
if not ref:
    sys.exit("usage: make_reference_line_counts.py <xSPDE reference checkout> (or set XSPDE_REFERENCE)")
out = {}
for dp, dn, fn in os.walk(ref):
    dn[:] = sorted(d for d in dn if not d.startswith("."))
    for f in sorted(fn):
        if f.endswith(".m"):
            path = os.path.join(dp, f)
            with open(path, errors="replace") as fh:
                out[os.path.relpath(path, ref)] = sum(1 for _ in fh)
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_line_counts.json")
with open(dst, "w") as f:
    json.dump(out, f, indent=0, sort_keys=True)
print("wrote", dst, len(out), "files")
