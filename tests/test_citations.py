"""Every `file.f90:line` citation in the sources, tests and documents names a Fortran file of
the reference checkout whose length covers the cited lines.  Runs when DSEM_REFERENCE_DIR names
the checkout; skipped otherwise."""
import collections
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("DSEM_REFERENCE_DIR", "")
CITE = re.compile(r"([A-Za-z0-9_./-]+\.f90):(\d+)(?:-(\d+))?((?:,\s*\d+(?:-\d+)?)*)")
SCANNED = ("dsem_b200", "oracle", "include", "tests", "bench.py", "__graft_entry__.py", "DESIGN.md",
           "INTEGRATION.md", "README.md", "BASELINE.md")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "src")), reason="reference checkout not given")
def test_fortran_citations_resolve():
    length = collections.defaultdict(list)  # file name -> [(path, lines)]
    for d, _, fs in os.walk(REF):
        for f in fs:
            if f.endswith(".f90"):
                p = os.path.join(d, f)
                with open(p, errors="replace") as fh:
                    length[f].append((p, sum(1 for _ in fh)))
    checked, bad = 0, []
    for entry in SCANNED:
        top = os.path.join(ROOT, entry)
        paths = [top] if os.path.isfile(top) else [
            os.path.join(d, f) for d, _, fs in os.walk(top) for f in fs
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp", ".md"))]
        for p in paths:
            with open(p, errors="replace") as fh:
                for ln, line in enumerate(fh, 1):
                    for m in CITE.finditer(line):
                        checked += 1
                        lines = [int(m.group(2))] + ([int(m.group(3))] if m.group(3) else [])
                        lines += [int(x) for x in re.findall(r"\d+", m.group(4) or "")]
                        cands = length.get(os.path.basename(m.group(1)), [])
                        if "/" in m.group(1):
                            cands = [c for c in cands if c[0].endswith(m.group(1))] or cands
                        if not any(max(lines) <= n for _, n in cands):
                            bad.append(f"{os.path.relpath(p, ROOT)}:{ln}: {m.group(0)}")
    assert checked > 100 and not bad, bad
