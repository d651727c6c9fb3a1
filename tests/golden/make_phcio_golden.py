"""Pin the text readers of phcpack_b200.phcio against the reference's own
example systems (src/Demo of the PHCpack tree): every file is parsed, the
product of the degrees is compared with the total degree the file states,
and the solution lists that files carry are read back (by variable name)
and the end points at t = 1 evaluated in the parsed system; the
m-homogeneous Bezout numbers the files state for a partition of the
variables are recomputed (phcpack_b200.rootcounts).  The summary goes to
tests/golden/phcio_demo.json; tests/test_phcio.py checks it.

Run from the repository root with the reference tree at hand:
    python tests/golden/make_phcio_golden.py <reference tree>
"""
import json
import os
import re
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", ".."))
from phcpack_b200 import phcio, homotopy as hm, rootcounts  # noqa: E402


def stated_total_degree(text):
    m = re.search(r"total degree\s*:([^\n]*)", text)
    if not m:
        return None
    nums = re.findall(r"\d+", m.group(1).replace(",", ""))
    return int(nums[-1]) if nums else None


def rel_residual(polys, x):
    worst = 0.0
    for p in polys:
        v, a = 0j, 0.0
        for mono, c in p:
            t = c
            for j, e in mono:
                t = t * x[j] ** e
            v += t
            a += abs(t)
        worst = max(worst, abs(v) / (1.0 + a))
    return worst


def main(root):
    demo = os.path.join(root, "src", "Demo")
    out = {}
    for f in sorted(os.listdir(demo)):
        text = open(os.path.join(demo, f), errors="replace").read()
        rec = {}
        try:
            polys, sym = phcio.parse_system(text)
        except phcio.ParseError as e:
            out[f] = {"parsed": False, "error": str(e)[:120]}
            continue
        rec["parsed"] = True
        rec["neq"], rec["nvar"] = len(polys), len(sym)
        rec["terms"] = [len(p) for p in polys]
        rec["degrees"] = [hm.degree(p) for p in polys]
        rec["total_degree"] = int(np.prod(rec["degrees"]))
        rec["stated_total_degree"] = stated_total_degree(text)
        mh = []
        for m in re.finditer(r"(\d+)-homogeneous Bezout number\s*:\s*([\d,]+)\s*\n\s*with partition\s*:\s*(\{.*\})",
                             text):
            sets = [st.split() for st in re.findall(r"\{([^{}]*)\}", m.group(3)) if st.strip()]
            if sorted(v for st in sets for v in st) != sorted(sym):
                continue  # a partition line that does not list every variable
            part = [[sym.index(v) for v in st] for st in sets]
            mh.append({"m": int(m.group(1)), "partition": sets, "stated": int(m.group(2).replace(",", "")),
                       "computed": rootcounts.bezout_number(polys, part)})
        if mh:
            rec["mhom_bezout"] = mh
        k = text.find("THE SOLUTIONS")
        if k >= 0:
            body = text[k:].split("\n", 1)[1]
            try:
                sols = phcio.parse_solutions(body, symbols=sym)
                at1 = [s for s in sols if abs(s["t"] - 1.0) < 1e-12 and np.all(np.isfinite(s["x"]))]
                res = [rel_residual(polys, s["x"]) for s in at1]
                rec["solutions"] = len(sols)
                rec["solutions_at_t1"] = len(at1)
                rec["at_t1_residuals_below_1e-8"] = int(sum(r <= 1e-8 for r in res))
                rec["max_residual_at_t1"] = float(max(res)) if res else None
            except Exception as e:  # recorded, checked by the test
                rec["solutions_error"] = str(e)[:120]
        out[f] = rec
    path = os.path.join(os.path.dirname(__file__), "phcio_demo.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=0, sort_keys=True)
    print(path, len(out))


if __name__ == "__main__":
    main(sys.argv[1]) if len(sys.argv) > 1 else sys.exit("usage: " + sys.argv[0] + " <reference tree>")
