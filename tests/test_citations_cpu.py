"""Every reference citation in this repository points inside the file it names.

Code, tests and notes cite the xSPDE reference as `name.m:a`, `name.m:a-b` or
`name.m:a,b` (optionally with a directory prefix).  The line counts of the
reference's MATLAB files are a committed fixture
(tests/golden/reference_line_counts.json, written by
make_reference_line_counts.py from a reference checkout), so this check needs
no checkout at test time.  A cited line beyond the end of its file, or a file
name the reference does not have, fails the test.
"""
import json
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CITE = re.compile(r"((?:[\w.'-]+/)*)([A-Za-z_]\w*\.m):(\d+)(?:-(\d+))?((?:,\s*\d+(?:-\d+)?)*)")
EXT = (".py", ".md", ".h", ".hpp", ".cpp", ".cu", ".cuh", ".c", ".m")


def _root_docs():
    """The top-level notes that are this library's documentation: README.md and the
    top-level .md files it names.  Other top-level .md files are records written
    around the build (reviews, surveys, run logs) that quote other documents'
    citations rather than make their own."""
    docs = {"README.md"}
    with open(os.path.join(ROOT, "README.md"), errors="replace") as f:
        docs |= set(re.findall(r"\b([A-Za-z][\w-]*\.md)\b", f.read()))
    return docs


def _tracked():
    try:
        out = subprocess.check_output(["git", "ls-files"], cwd=ROOT, text=True, stderr=subprocess.DEVNULL)
        files = out.split()
    except Exception:
        files = []
        for dp, dn, fn in os.walk(ROOT):
            # untracked trees: hidden and underscore folders, run outputs, installed packages
            dn[:] = [d for d in dn if not d.startswith((".", "_", "baseline")) and not d.endswith("_out")]
            files += [os.path.relpath(os.path.join(dp, f), ROOT) for f in fn]
    docs = _root_docs()
    return [f for f in files if f.endswith(EXT) and ("/" in f or not f.endswith(".md") or f in docs)]


def _counts():
    with open(os.path.join(ROOT, "tests", "golden", "reference_line_counts.json")) as f:
        counts = json.load(f)
    by_name = {}
    for path, n in counts.items():
        by_name.setdefault(os.path.basename(path), []).append((path, n))
    return by_name


def test_citations_fall_inside_the_cited_files():
    by_name = _counts()
    bad = []
    n_cites = 0
    for f in _tracked():
        full = os.path.join(ROOT, f)
        if not os.path.exists(full):
            continue
        with open(full, errors="replace") as fh:
            for ln, line in enumerate(fh, 1):
                for m in CITE.finditer(line):
                    prefix, name, a, b, extra = m.groups()
                    cands = by_name.get(name)
                    if not cands:
                        bad.append("%s:%d %s: no such reference file" % (f, ln, m.group(0)))
                        continue
                    if prefix:
                        narrowed = [c for c in cands if c[0].endswith(prefix + name)]
                        cands = narrowed or cands
                    lines = max(n for _, n in cands)
                    nums = [int(a)] + ([int(b)] if b else []) + [int(x) for x in re.findall(r"\d+", extra or "")]
                    n_cites += 1
                    if max(nums) > lines or (b and int(b) < int(a)):
                        bad.append("%s:%d %s: file has %d lines" % (f, ln, m.group(0), lines))
    assert n_cites > 100
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("cite,fragment", [
    ("Simulator/xpath.m:42", "p.method(a(1:f),w,p)"),
    ("Simulator/xnoise.m:33", "nc == 2"),
    ("Applications/SDE/MP.m:14", "p.iterations"),
    ("Simulator/xsim.m:95", "sqrt"),
])
def test_reference_anchor_lines_recorded(cite, fragment):
    """The anchors the C ABI header relies on exist with the recorded lengths
    (content is checked only where the reference checkout is present)."""
    path, line = cite.split(":")
    counts = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_line_counts.json")))
    assert int(line) <= counts[path]
    ref = os.environ.get("XSPDE_REFERENCE")
    if ref and os.path.isdir(ref):
        with open(os.path.join(ref, path), errors="replace") as fh:
            text = fh.read().splitlines()
        assert fragment in text[int(line) - 1]
