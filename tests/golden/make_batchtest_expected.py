"""Extract the reference's Batchtest golden error values into a fixture.

Reads Examples/Batchtest.m of the xSPDE reference checkout (path given as the
first argument, or in XSPDE_REFERENCE) as text and writes
batchtest_expected.json beside this script: {name: expected e(1)} for the 42
projects, in Batchtest order.  The reference accepts e(1) within a factor
1.001 of these values (Examples/Batchtest.m:81).
"""
import json
import os
import re
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("XSPDE_REFERENCE")
if not ref:
    sys.exit("usage: make_batchtest_expected.py <xSPDE reference checkout> (or set XSPDE_REFERENCE)")
src = open(os.path.join(ref, "Examples", "Batchtest.m")).read()
names = re.findall(r"e\{(\d+)\}\s*=\s*\w+;\s*n\{\d+\}\s*=\s*'([^']+)'", src)
body = src[src.index("e1 = ["):]
body = body[: body.index("];")]
vals = [float(x) for x in re.findall(r"[0-9.]+e[-+][0-9]+", body)]
assert len(names) == len(vals) == 42, (len(names), len(vals))
out = {n: v for (_, n), v in zip(names, vals)}
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "batchtest_expected.json")
with open(path, "w") as f:
    json.dump(out, f, indent=1)
print("wrote", path)
