"""Extract the reference's static mirror/glide table (src/mirror_table.jl) into
tests/golden/mirror_table.json.

The table was generated by the reference from Crystalline.jl's operation lists
(scripts/compute_mirror_table.jl), so it pins, for every space group, the
centring vectors and -- per mirror/glide normal -- the translation of the first
such operation in Crystalline's order.  The space-group tests compare the
library's generated operation tables against it.

Run with the path of the reference's src/mirror_table.jl:
    python tests/golden/make_mirror_fixture.py <reference checkout>/src/mirror_table.jl
"""
import json
import os
import re
import sys
from fractions import Fraction


def parse_vecs(s):
    out = []
    for m in re.finditer(r"\[([^\[\]]*)\]", s):
        body = m.group(1).strip()
        if not body:
            continue
        vals = [v.strip() for v in body.split(",")]
        row = []
        for v in vals:
            if "//" in v:
                a, b = v.split("//")
                row.append(str(Fraction(int(a), int(b))))
            else:
                row.append(str(Fraction(int(v))))
        out.append(row)
    return out


def main(path):
    text = open(path).read()
    table = {}
    pat = re.compile(r"^\s*(\d+)\s*=>\s*MirrorAdaptationEntry\((.*)\),\s*$", re.M)
    for m in pat.finditer(text):
        sg = int(m.group(1))
        body = m.group(2)
        # fields: n_mirrors, normals, translations, centering, centering_vecs, ...
        depth, parts, cur = 0, [], ""
        for ch in body:
            if ch == "[":
                depth += 1
            elif ch == "]":
                depth -= 1
            if ch == "," and depth == 0:
                parts.append(cur.strip())
                cur = ""
            else:
                cur += ch
        parts.append(cur.strip())
        n_mirrors = int(parts[0])
        normals = [[int(Fraction(x)) for x in v] for v in parse_vecs(parts[1])]
        trans = parse_vecs(parts[2])
        centering = parts[3].lstrip(":")
        cvecs = parse_vecs(parts[4])
        # remaining fields: all_axial, det_T, mirror_reduction, centering_multiplier,
        # effective_reduction, has_glide
        table[sg] = {"n_mirrors": n_mirrors, "normals": normals, "translations": trans,
                     "centering": centering, "centering_vecs": cvecs,
                     "all_axial": parts[5] == "true", "det_T": int(parts[6]),
                     "mirror_reduction": int(parts[7]), "centering_multiplier": int(parts[8]),
                     "effective_reduction": int(parts[9]), "has_glide": parts[10] == "true"}
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mirror_table.json")
    with open(out, "w") as f:
        json.dump({str(k): table[k] for k in sorted(table)}, f, indent=0, sort_keys=True)
    print(f"wrote {len(table)} entries to {out}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_mirror_fixture.py <reference checkout>/src/mirror_table.jl")
    main(sys.argv[1])
