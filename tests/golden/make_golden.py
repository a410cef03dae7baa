"""Regenerates the golden fixtures of this directory from the reference sources.

Run with the environment variable REFERENCE_ROOT set to a checkout of the
reference (lavenklau/homo3d).  The fixtures are committed; tests never read the
reference at run time.

  ke_lame72.json : the integer tables 72*K_lambda and 72*K_mu that the reference
                   hard-codes in homogenization/templateMatrix.cpp:8-61
                   (Ke = lambda*K_lambda + mu*K_mu), read from the source text.
"""
import json
import os
import re
import sys

ROOT = os.environ.get("REFERENCE_ROOT")


def _table(src, name):
    m = re.search(r"char\s+%s\s*\[\s*\]\s*=\s*\{(.*?)\};" % name, src, re.S)
    if not m:
        raise ValueError("table %s not found" % name)
    vals = [int(v) for v in re.findall(r"-?\d+", m.group(1))]
    if len(vals) != 576:
        raise ValueError("table %s has %d entries" % (name, len(vals)))
    return vals


def main():
    if not ROOT:
        sys.exit("set REFERENCE_ROOT to a checkout of lavenklau/homo3d")
    path = os.path.join(ROOT, "homogenization", "templateMatrix.cpp")
    src = open(path).read()
    out = {
        "source": "homogenization/templateMatrix.cpp:8-61",
        "layout": "row-major 24x24, DOF 3*node+component, node i at (i%2, i/2%2, i/4)",
        "kelam72": _table(src, "kelam72"),
        "kemu72": _table(src, "kemu72"),
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ke_lame72.json")
    with open(dst, "w") as f:
        json.dump(out, f)
    print("wrote", dst)


if __name__ == "__main__":
    sys.exit(main())
