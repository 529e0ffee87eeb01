"""Regenerate the golden fixtures under tests/golden/ (run in a container that
has the reference sources mounted).

ref_xoro.txt  -- output of oracle/_ref/ref_xoro: the reference's own
                 xoroshiro128+ engine (ModelG/xoroshiro128plus.h) driven through
                 NoiseGenerator's construction (NoiseGenerator.h:68-81) and the
                 libstdc++ distributions it uses.  Pins the oracle's restated
                 serial stream.
o4_known.json -- the O(4) rotation known answers written in
                 ModelG/O4AlgebraSignTest.cxx:20-39 (comments at :24, :31, :38),
                 and the fixed inputs of ModelG/O4AlgebraTester.cxx:48-81.
hcrit1.json   -- equilibrium <phi_0> of the Model A heat bath read from
                 ModelG/hcrit1_N032_m-04813_h010000_l10000_averages_ave.out:1
                 (parameters decoded from the file name: N=32, m^2=-4.813,
                 H=0.01, lambda=10).

Usage:  python tests/golden/make_golden.py --ref <reference ModelG directory>
"""
import argparse
import json
import math
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's ModelG directory")
    a = ap.parse_args()
    subprocess.check_call(["make", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={a.ref}"])
    out = subprocess.check_output([os.path.join(REPO, "oracle", "_ref", "ref_xoro")], text=True)
    with open(os.path.join(HERE, "ref_xoro.txt"), "w") as f:
        f.write(out)

    s = 1.0 / math.sqrt(2.0)
    known = {
        "source": "ModelG/O4AlgebraSignTest.cxx:20-39",
        "cases": [
            {"A": [math.pi / 4, 0, 0], "V": [0, 0, 0], "phi": [1, 0, 0, 0], "expect": [s, -s, 0, 0]},
            {"A": [0, 0, 0], "V": [0, 0, math.pi / 4], "phi": [0, 1, 0, 0], "expect": [0, s, -s, 0]},
            {"A": [0, 0, 0], "V": [0, 0, math.pi / 4], "phi": [0, 0, 1, 0], "expect": [0, s, s, 0]},
        ],
        "tester_inputs": {
            "source": "ModelG/O4AlgebraTester.cxx:48-81",
            "rotation": {"A": [1, 2, 3], "V": [4, 5, 6], "phi": [0.5, 0.5, 0.5, 0.5]},
        },
    }
    with open(os.path.join(HERE, "o4_known.json"), "w") as f:
        json.dump(known, f, indent=1)

    fname = os.path.join(a.ref, "hcrit1_N032_m-04813_h010000_l10000_averages_ave.out")
    with open(fname) as fh:
        cols = [float(x) for x in fh.read().split()]
    with open(os.path.join(HERE, "hcrit1.json"), "w") as f:
        json.dump({"source": "ModelG/hcrit1_N032_m-04813_h010000_l10000_averages_ave.out:1",
                   "N": 32, "mass0": -4.813, "H": 0.01, "lambda": 10.0,
                   "phi0_mean": cols[0], "phi0_err": cols[1], "tau_column": cols[2]}, f, indent=1)


if __name__ == "__main__":
    main()
