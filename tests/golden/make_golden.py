"""Regenerates the golden fixtures in tests/golden/ from the reference.

Run where the reference sources are present (--reference, or the environment
variable NDG_REFERENCE_DIR)
after `make -C oracle`:

    python tests/golden/make_golden.py [--reference /path/to/NDG_cuda]

* legendre_n16.json: the Legendre-Gauss N = 16 nodes and weights that the
  reference's own test pins (tests/polynomials_test.cu:187-226), read from
  that file as text.
* ref_*.npz: solution arrays of the reference's own CPU path
  (oracle/_ref/libndgref.so) after a number of RK3 steps on generated zones,
  with the zone parameters, dt and final time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle  # noqa: E402
from tests import meshgen  # noqa: E402

# name: (res, N, boundary, periodic, steps)
CASES = {
    "ref_periodic_r16_n4_s200": (16, 4, meshgen.WALL, True, 200),
    "ref_periodic_r8_n8_s20": (8, 8, meshgen.WALL, True, 20),
    "ref_wall_r8_n6_s30": (8, 6, meshgen.WALL, False, 30),
    "ref_outflow_r4_n5_s10": (4, 5, meshgen.OUTFLOW, False, 10),
}


def legendre_literals(reference: str) -> dict:
    path = os.path.join(reference, "tests", "polynomials_test.cu")
    text = open(path).read()
    block = text[text.index('TEST_CASE("LegendrePolynomials"'):]

    def array(name: str) -> list[float]:
        m = re.search(r"std::array<double, N_test\+1> " + name + r" \{([^}]*)\}", block)
        return [float(v) for v in m.group(1).replace("\n", " ").split(",")]

    return {"N": 16, "source": "tests/polynomials_test.cu:187-226", "nodes": array("nodes"), "weights": array("weights")}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("NDG_REFERENCE_DIR"),
                    help="root of the reference checkout (default: $NDG_REFERENCE_DIR)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("the reference checkout is needed: --reference or NDG_REFERENCE_DIR")
    with open(os.path.join(HERE, "legendre_n16.json"), "w") as f:
        json.dump(legendre_literals(args.reference), f, indent=1)
    if not pyoracle.ref_available():
        raise SystemExit("oracle/_ref/libndgref.so is missing: run make -C oracle first")
    for name, (res, N, bc, periodic, steps) in CASES.items():
        zone = meshgen.uniform_zone(res, boundary=bc, x_periodic=periodic, y_periodic=periodic)
        ref = pyoracle.RefSolver(zone, N)
        ref.initial_conditions()
        dt = ref.delta_t()
        t = ref.run(steps)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), res=res, N=N, boundary=bc, periodic=periodic, steps=steps,
                            dt=dt, time=t, p=ref.field("p"), u=ref.field("u"), v=ref.field("v"))
        print(name, "dt", dt, "t", t)


if __name__ == "__main__":
    main()
