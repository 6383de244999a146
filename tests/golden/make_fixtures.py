"""Regenerate tests/golden/example_inputs.json from the reference's example inputs.

The reference keeps its example parameters in examples/inputs/*.json (flat
{"key": {"value": v, "unit": u}} files read by CabanaDEM::Inputs).  This script collects
them, keyed by file stem, into one fixture so that tests running where the reference is
not mounted use the same parameters.  Run:  python tests/golden/make_fixtures.py [ref_root]
(ref_root defaults to $CABANADEM_REFERENCE, else the read-only mount /root/reference).
"""
import glob
import json
import os
import sys


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CABANADEM_REFERENCE", "/root/reference")
    if not os.path.isdir(os.path.join(ref, "examples", "inputs")):
        sys.exit("make_fixtures: no examples/inputs under %s (pass the reference checkout)" % ref)
    out = {}
    for path in sorted(glob.glob(os.path.join(ref, "examples", "inputs", "*.json"))):
        with open(path) as f:
            out[os.path.splitext(os.path.basename(path))[0]] = json.load(f)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "example_inputs.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", dst, "with", len(out), "inputs")


if __name__ == "__main__":
    main()
