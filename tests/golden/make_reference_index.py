"""Write tests/golden/reference_index.json: the shape of the reference's sources.

    python tests/golden/make_reference_index.py <path to the lceqcd checkout>

For every file under the checkout's ``f/`` directory (Fortran sources, the
``INCLUDE/*.inc`` blocks and ``luxury.h``) the index records its line count and
the line span of every program unit (``subroutine``/``function``/``program``
statement to its ``end`` statement).  No source text is stored: the index only
lets ``tests/test_citations.py`` check, without the reference present, that
every ``f/<file>:<line>`` citation in this repository lands inside the file and,
where the citation names a routine, inside that routine.
"""
from __future__ import annotations

import json
import os
import re
import sys

UNIT_RE = re.compile(r"^\s+(?:(?:real|integer|double\s+precision|complex|logical)\s*(?:\*\s*\d+)?\s+)?"
                     r"(subroutine|function|program)\s+([A-Za-z_][A-Za-z0-9_]*)", re.I)
END_RE = re.compile(r"^[\s\d]+end\s*(?:(?:subroutine|function|program)(?:\s+[A-Za-z0-9_]+)?)?\s*(?:!.*)?$", re.I)


def index_file(path: str) -> dict:
    with open(path, encoding="latin-1") as fh:
        lines = fh.read().split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    units = []
    cur = None
    for i, line in enumerate(lines, 1):
        if line[:1] in ("c", "C", "*", "!"):
            continue
        m = UNIT_RE.match(line)
        if m and cur is None:
            cur = {"name": m.group(2).lower(), "kind": m.group(1).lower(), "start": i}
            continue
        if cur is not None and END_RE.match(line):
            cur["end"] = i
            units.append(cur)
            cur = None
    return {"lines": len(lines), "units": units}


def main(argv: list[str]) -> int:
    if len(argv) != 2:
        print(__doc__)
        return 2
    root = os.path.join(argv[1], "f")
    out = {}
    for dirpath, _, files in os.walk(root):
        for name in sorted(files):
            if not (name.endswith(".f") or name.endswith(".inc") or name.endswith(".h")):
                continue
            p = os.path.join(dirpath, name)
            rel = os.path.relpath(p, argv[1]).replace(os.sep, "/")
            out[rel] = index_file(p)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_index.json")
    with open(dst, "w") as fh:
        json.dump(dict(sorted(out.items())), fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(f"wrote {dst}: {len(out)} files")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
