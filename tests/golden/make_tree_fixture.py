"""Extract the reference's recursive-tree survey (test/debug_tree_output.log, written by
the reference's test/debug_tree.jl at N = 64^3) into tests/golden/tree_survey_64.json.

For each space group of the survey (16-74, 75-142, 195-230) the log lists |G| (the
number of operations get_ops returns, centring included), the centring class of the
pure translations (P, I/C/A, F), the reduction ratio N^3 / (total leaf volume) of the
recursive parity tree, and that ratio times the centring index.  The tree depends on
the operations' translations, so the ratios pin the operation tables as well as the
tree construction.

Run with the path of the reference's test/debug_tree_output.log:
    python tests/golden/make_tree_fixture.py <reference checkout>/test/debug_tree_output.log
"""
import json
import os
import re
import sys

ROW = re.compile(r"^\s*(\d+)\s+\S+\s+(\d+)\s+(\S+)\s+([\d.]+)×\s+([\d.]+)×\s+(\d+)×\s+([\d.]+)%")


def main(path):
    rows = {}
    for line in open(path, encoding="utf-8"):
        m = ROW.match(line)
        if m and m.group(1) not in rows:
            rows[m.group(1)] = {"G": int(m.group(2)), "centering": m.group(3), "ratio": float(m.group(4)),
                                "ratio_x_cent": float(m.group(5))}
    out = {"N": [64, 64, 64], "source": "test/debug_tree_output.log", "groups": rows}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tree_survey_64.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=0, sort_keys=True)
    print(f"{len(rows)} groups -> {dst}")


if __name__ == "__main__":
    main(sys.argv[1])
