"""Every ``f/<file>:<lines>`` citation of the reference in this repository resolves.

The reference's file shapes (line counts and program-unit spans) are in
``tests/golden/reference_index.json``, written by
``tests/golden/make_reference_index.py`` from a checkout of the reference.  A
citation passes when its file exists there, every cited line lies inside the
file, and, when the citation sits next to the name of one of the cited file's
routines (``agauge`` ... ``f/agauge.f:7-205``), every cited line lies inside
that routine's span.
"""
from __future__ import annotations

import json
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INDEX = os.path.join(ROOT, "tests", "golden", "reference_index.json")

# product directories scanned in full; at the top level, the Python entry
# points and the markdown documents whose title names this package (planning
# notes and driver records quote the reference too, but are not product files)
SCAN_DIRS = ("lceqcd_b200", "include", "oracle", "tests", "profiles")
SKIP_DIRS = {"_build", "__pycache__", ".pytest_cache"}
EXTS = (".py", ".c", ".h", ".cu", ".cuh", ".hpp", ".cpp", ".md", ".txt")
SELF = os.path.abspath(__file__)  # holds deliberately bad examples

CITE_RE = re.compile(r"(?<![A-Za-z0-9_/.])(f/[A-Za-z0-9_./]+?\.(?:f|inc|h))"
                     r"(?::(\d+(?:-\d+)?(?:,\s?\d+(?:-\d+)?)*))?")


def _is_product_doc(path: str) -> bool:
    with open(path, encoding="utf-8", errors="replace") as fh:
        title = fh.readline()
    return title.startswith("#") and ("lceqcd_b200" in title or "lceqcd-b200" in title
                                      or "liblceqcd_gpu" in title)


def _repo_files():
    for name in sorted(os.listdir(ROOT)):
        p = os.path.join(ROOT, name)
        if os.path.isfile(p) and (name.endswith(".py") or (name.endswith(".md") and _is_product_doc(p))):
            yield p
    for d in SCAN_DIRS:
        for dirpath, dirnames, files in os.walk(os.path.join(ROOT, d)):
            dirnames[:] = [x for x in dirnames if x not in SKIP_DIRS and not x.startswith(".")]
            for name in files:
                p = os.path.join(dirpath, name)
                if name.endswith(EXTS) and os.path.abspath(p) != SELF:
                    yield p


def _ranges(spec: str):
    for part in spec.split(","):
        part = part.strip()
        if "-" in part:
            a, b = part.split("-")
            yield int(a), int(b)
        else:
            yield int(part), int(part)


def citations():
    out = []
    for path in _repo_files():
        with open(path, encoding="utf-8", errors="replace") as fh:
            for lineno, line in enumerate(fh, 1):
                for m in CITE_RE.finditer(line):
                    out.append((os.path.relpath(path, ROOT), lineno, line, m))
    return out


def _problems():
    with open(INDEX) as fh:
        index = json.load(fh)
    bad = []
    for rel, lineno, line, m in citations():
        fname, spec = m.group(1), m.group(2)
        where = f"{rel}:{lineno}: {m.group(0)}"
        if fname not in index:
            bad.append(f"{where}: no such reference file")
            continue
        info = index[fname]
        if spec is None:
            continue
        ranges = list(_ranges(spec))
        for a, b in ranges:
            if not (1 <= a <= b <= info["lines"]):
                bad.append(f"{where}: lines {a}-{b} outside the file ({info['lines']} lines)")
        # a routine of the cited file named just before the citation
        prefix = line[max(0, m.start() - 48):m.start()]
        named = [u for u in info["units"]
                 if re.search(r"(?<![A-Za-z0-9_])" + re.escape(u["name"]) + r"(?![A-Za-z0-9_])", prefix, re.I)]
        if len(named) == 1 and len(info["units"]) > 1:
            u = named[0]
            for a, b in ranges:
                if not (u["start"] <= a and b <= u["end"]):
                    bad.append(f"{where}: lines {a}-{b} outside {u['name']} ({u['start']}-{u['end']})")
    return bad


def test_index_present():
    with open(INDEX) as fh:
        index = json.load(fh)
    assert "f/agauge.f" in index and index["f/agauge.f"]["units"][0]["name"] == "agauge"


def test_repository_cites_the_reference():
    assert len(citations()) > 200


def test_every_citation_resolves():
    bad = _problems()
    assert not bad, f"{len(bad)} citations do not resolve:\n" + "\n".join(bad)


@pytest.mark.parametrize("text,ok", [
    ("`agauge` `f/agauge.f:7-205`", True),
    ("`f/renorm.f:205`", False),
    ("`randomconf` `f/confget.f:86-151`", True),
    ("`testconf` `f/confget.f:86-151`", False),
])
def test_checker_flags_bad_citations(text, ok, tmp_path):
    with open(INDEX) as fh:
        index = json.load(fh)
    m = CITE_RE.search(text)
    info = index[m.group(1)]
    ranges = list(_ranges(m.group(2)))
    inside = all(1 <= a <= b <= info["lines"] for a, b in ranges)
    named = [u for u in info["units"] if re.search(r"(?<![A-Za-z0-9_])" + u["name"] + r"(?![A-Za-z0-9_])",
                                                  text[:m.start()])]
    if len(named) == 1 and len(info["units"]) > 1:
        inside = inside and all(named[0]["start"] <= a and b <= named[0]["end"] for a, b in ranges)
    assert inside == ok
