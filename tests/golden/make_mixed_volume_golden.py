"""Pin phcpack_b200.rootcounts.mixed_volume against the mixed volumes that
the reference's example systems state (src/Demo of the PHCpack tree, the
"mixed volume : N" lines).  Every file with a stated mixed volume and at most
MAXVAR variables is parsed, its supports are written to
tests/golden/mixed_volume_demo.json with the stated number and the computed
one (each in a child process, skipped after TIME_LIMIT seconds);
tests/test_rootcounts_mv.py checks the file and recomputes the smaller
systems from the stored supports.

Run from the repository root with the reference tree at hand:
    python tests/golden/make_mixed_volume_golden.py <reference tree>
"""
import json
import os
import re
import subprocess
import sys
import time

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", ".."))
from phcpack_b200 import phcio, rootcounts  # noqa: E402

MAXVAR = 12
TIME_LIMIT = 30


def stated_mixed_volume(text):
    m = re.search(r"mixed volume\s*:\s*([\d,]+)", text)
    return int(m.group(1).replace(",", "")) if m else None


def one(path, nvar):
    """Child process: the mixed volume of one file, printed as JSON."""
    polys, sym = phcio.parse_system(open(path, errors="replace").read())
    t0 = time.time()
    got = rootcounts.mixed_volume(polys, len(sym))
    print(json.dumps(dict(computed=got, seconds=round(time.time() - t0, 2))))


def main(ref):
    demo = os.path.join(ref, "src", "Demo")
    out = {}
    for name in sorted(os.listdir(demo)):
        path = os.path.join(demo, name)
        if not os.path.isfile(path):
            continue
        text = open(path, errors="replace").read()
        mv = stated_mixed_volume(text)
        if mv is None:
            continue
        try:
            polys, sym = phcio.parse_system(text)
        except Exception as e:  # noqa: BLE001 - a reader error is recorded, not fatal
            out[name] = dict(stated=mv, error=str(e))
            continue
        if len(sym) > MAXVAR or len(polys) != len(sym):
            continue
        supports = [s.tolist() for s in rootcounts._supports(polys, len(sym))]
        rec = dict(stated=mv, nvar=len(sym), supports=supports)
        try:
            r = subprocess.run([sys.executable, __file__, "--one", path], capture_output=True, text=True,
                               timeout=TIME_LIMIT)
            rec.update(json.loads(r.stdout.strip().splitlines()[-1]))
        except subprocess.TimeoutExpired:
            rec["skipped"] = f"over {TIME_LIMIT} s"
        out[name] = rec
        print(f"{name:12s} stated {mv:6d} computed {rec.get('computed', -1):6d} "
              f"({rec.get('seconds', rec.get('skipped'))})", flush=True)
    with open(os.path.join(os.path.dirname(__file__), "mixed_volume_demo.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--one":
        one(sys.argv[2], None)
    else:
        main(sys.argv[1]) if len(sys.argv) > 1 else sys.exit("usage: " + sys.argv[0] + " <reference tree>")
