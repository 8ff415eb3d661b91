"""Every `name.m:line` citation in the source files points at lines that exist.

The kernels, the oracle and the tests cite the MATLAB reference file by file
and line so that each step can be audited against it.  This test reads the
reference checkout (the directory in $GBM3D_REFERENCE_ROOT, by default the
location in REF below) and fails for a citation whose file is
unknown or whose highest cited line is past the end of that file.  Without the
checkout it is skipped.
"""
import collections
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("GBM3D_REFERENCE_ROOT", "/root/reference")
CITE = re.compile(r"([A-Za-z0-9_]+\.m):(\d+(?:-\d+)?(?:,\d+(?:-\d+)?)*)")
# the source trees of the library, the oracle and the tests, and the
# top-level scripts
SOURCE_DIRS = ("gbm3d_b200", "oracle", "tests", "include")
SOURCE_EXT = (".py", ".cu", ".cuh", ".cpp", ".h", ".c")


def _reference_lines():
    index = collections.defaultdict(list)
    for dp, _, files in os.walk(REF):
        for f in files:
            if f.endswith(".m"):
                with open(os.path.join(dp, f), errors="replace") as fh:
                    index[f].append(sum(1 for _ in fh))
    return index


def _source_files():
    for f in sorted(os.listdir(ROOT)):
        if f.endswith(SOURCE_EXT):
            yield os.path.join(ROOT, f)
    for top in SOURCE_DIRS:
        for dp, dirs, files in os.walk(os.path.join(ROOT, top)):
            dirs[:] = [d for d in dirs if not d.startswith(("_", "."))]
            for f in sorted(files):
                if f.endswith(SOURCE_EXT):
                    yield os.path.join(dp, f)


def _citations():
    for p in _source_files():
        with open(p, errors="replace") as fh:
            for ln, line in enumerate(fh, 1):
                for m in CITE.finditer(line):
                    yield os.path.relpath(p, ROOT), ln, m.group(1), m.group(2)


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference checkout not present")
def test_every_cited_line_exists():
    index = _reference_lines()
    bad = []
    n = 0
    for path, ln, name, rng in _citations():
        n += 1
        hi = max(int(x) for x in re.findall(r"\d+", rng))
        lengths = index.get(name)
        if not lengths:
            bad.append(f"{path}:{ln}: {name} is not a file of the reference")
        elif all(hi > L for L in lengths):
            bad.append(f"{path}:{ln}: {name}:{rng} but the file has {max(lengths)} lines")
    assert n > 100, "citation scan found too few citations"
    assert not bad, "\n".join(bad)
