"""Record the reference's check-node tree schedules as a golden fixture.

Runs the reference's own generator (src/LDPCDec/min_find.pl, invoked as
min_find_wrap.pl does: ``min_find.pl <d> prod``) for every row weight and
writes ``min_find_trees.json``: for d <= 32 the full statement list
(node masks in hex), for 33..53 a SHA-256 of the statement list.

    python tests/golden/make_tree_golden.py <reference checkout>
"""
import hashlib
import json
import os
import re
import subprocess
import sys

STMT = [
    (re.compile(r"SIMD_CLASS m([0-9a-f]+) = tanh\( grp_min\[(\d+)\*SIMD_PER_Z \+ i\] \* 0\.5 \);"), "in"),
    (re.compile(r"SIMD_CLASS m([0-9a-f]+) = m([0-9a-f]+) \* m([0-9a-f]+);"), "op"),
    (re.compile(r"m([0-9a-f]+) = min\( Max_val, m([0-9a-f]+) \);"), "clamp"),
    (re.compile(r"fin_min\[(\d+)\*SIMD_PER_Z \+ i\] = 2\.0\*atanh\( m([0-9a-f]+) \);"), "out"),
]


def parse(text):
    out = []
    for line in text.splitlines():
        line = line.strip()
        for rx, kind in STMT:
            m = rx.fullmatch(line)
            if m:
                g = m.groups()
                if kind == "in":
                    out.append(["in", g[0], int(g[1])])
                elif kind == "op":
                    out.append(["op", g[0], g[1], g[2]])
                elif kind == "clamp":
                    out.append(["clamp", g[0]])
                else:
                    out.append(["out", int(g[0]), g[1]])
                break
    return out


def main():
    ref = sys.argv[1]
    gen = os.path.join(ref, "src", "LDPCDec", "min_find.pl")
    res = {"full": {}, "sha256": {}}
    for d in range(2, 54):
        txt = subprocess.run(["perl", gen, str(d), "prod"], capture_output=True, text=True, check=True).stdout
        stm = parse(txt)
        if d <= 32:
            res["full"][str(d)] = stm
        res["sha256"][str(d)] = hashlib.sha256(json.dumps(stm).encode()).hexdigest()
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "min_find_trees.json")
    with open(dst, "w") as f:
        json.dump(res, f, separators=(",", ":"))
        f.write("\n")


if __name__ == "__main__":
    main()
