"""Generate tests/golden/ranlux_luxtst.json from the reference's own
known-answer block for RANLUX: the expected output of the luxtst program,
written as comments at f/luxtst.f:88-162 of derek-teaney/lceqcd.

Run in a checkout where the reference is available:
    python tests/golden/make_golden.py /path/to/lceqcd

The JSON records, for each case of the luxtst program (f/luxtst.f:10-66),
the call sequence and the printed numbers 1-5 and 101-105 (8 decimals), and
the 25-integer restart vector.  These are the only golden vectors the
reference repository holds.
"""
from __future__ import annotations

import json
import os
import re
import sys


def parse(path: str) -> dict:
    lines = open(path).read().splitlines()
    # the expected-output comment block starts after "OUTPUT FROM THE ABOVE TEST PROGRAM"
    start = next(i for i, l in enumerate(lines) if "OUTPUT FROM THE ABOVE TEST PROGRAM" in l)
    block = [l[1:] if l.startswith("!") else l for l in lines[start:]]
    nums = []
    restart = []
    grab_restart = False
    for l in block:
        s = l.strip()
        if "status saved" in s:
            grab_restart = True
            continue
        if grab_restart:
            ints = re.findall(r"-?\d+", s)
            if ints and all(len(x) > 3 for x in ints):
                restart.extend(int(x) for x in ints)
                if len(restart) >= 25:
                    grab_restart = False
                continue
        if re.fullmatch(r"(\d\.\d{8}\s*){5}", s):
            nums.append([float(x) for x in s.split()])
    cases = [
        {"setup": "default", "first": nums[0], "second": nums[1]},
        {"setup": "rluxgo(0,0,0,0)", "first": nums[2], "second": nums[3]},
        {"setup": "rluxgo(389,1,0,0)", "first": nums[4], "second": nums[5]},
        {"setup": "rluxgo(75,0,0,0)", "first": nums[6], "second": nums[7]},
        {"setup": "continue p=75", "first": nums[8], "second": nums[9]},
        {"setup": "rluxin(restart)", "first": nums[10], "second": nums[11]},
    ]
    return {
        "source": "f/luxtst.f:88-162 (expected output of the luxtst program)",
        "cases": cases,
        "restart": restart[:25],
    }


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the lceqcd checkout>")
    ref = sys.argv[1]
    data = parse(os.path.join(ref, "f", "luxtst.f"))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ranlux_luxtst.json")
    with open(out, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", out, len(data["cases"]), "cases")


if __name__ == "__main__":
    main()
