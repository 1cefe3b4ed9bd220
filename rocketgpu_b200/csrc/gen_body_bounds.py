"""Generates rg_body_bounds.inc: every car body's stored mesh bounds (centre from the car's origin and half extent, uu),
indexed by CarConfig::body, the data the respawn-spot picker tests other cars' bodies against (reference
CarBodyMeshBounds, include/rocketgpu/detail/step/env_step.hpp:6546-6553, fed from the reference's
tools/data/car_body_mesh_bounds.tsv through its include/rocketgpu/detail/car_body_bounds.inc).

Each decimal is rounded once, exactly, to the nearest float (ties to even), and written with nine significant digits,
which read back to that float.
Run:  python rocketgpu_b200/csrc/gen_body_bounds.py <reference>/tools/data/car_body_mesh_bounds.tsv \
          > rocketgpu_b200/csrc/rg_body_bounds.inc
"""
from fractions import Fraction
import sys

import numpy as np


def nearest_float(text: str) -> np.float32:
    exact = Fraction(text)
    c = np.float32(float(exact))
    best = None
    for cand in (np.nextafter(c, np.float32(-np.inf)), c, np.nextafter(c, np.float32(np.inf))):
        err = abs(Fraction(float(cand)) - exact)
        even = (int(np.array(cand).view(np.uint32)) & 1) == 0
        key = (err, not even)
        if best is None or key < best[0]:
            best = (key, cand)
    return best[1]


def literal(text: str) -> str:
    f = nearest_float(text)
    s = "%.9g" % float(f)
    assert np.float32(float(s)) == f
    if "." not in s and "e" not in s:
        s += ".0"
    return s + "f"


def main(path: str) -> None:
    rows = [line.rstrip("\n").split("\t") for line in open(path) if line and line[0] != "#"]
    assert rows[0][:2] == ["body", "handling_preset"] and all(len(r) == 8 for r in rows), "unexpected table header"
    rows = rows[1:]
    out = ["// Generated by gen_body_bounds.py from the reference's car body mesh bounds table. Do not edit.",
           "// One row per CarConfig::body: mesh centre from the car's origin (x, y, z) and half extent (x, y, z), uu.",
           "RG_BODY_BOUNDS_TABLE(kBodyMeshBounds, %d) = {" % len(rows)]
    for r in rows:
        out.append("    {%s},  // %s" % (", ".join(literal(v) for v in r[2:]), r[0]))
    out.append("};")
    sys.stdout.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main(sys.argv[1])
