"""Generate tests/golden/reference_units.npz from the reference's own outputs.

The reference ships, beside its unit-scaling scripts (tests/test_units/
test_ac.py, test_dp.py, test_eps.py), the curves those scripts produced:
graphene 4096 x 4096 (a = 0.142 nm, t = 3.0 eV, the cell of
tests/test_units/test_lindhard.py:7-16), rescale 9, one random state, 1024
time steps:

* ac / omegas_ac: Analyzer.calc_ac_cond of Solver.calc_corr_ac_cond
  (correct_spin = True), shape (4, 1024);
* dp / omegas_dp: Analyzer.calc_dyn_pol at q = (1/a) (0.8660254, 0.5, 0);
* eps / omegas_eps: Analyzer.calc_epsilon at q = (4.122280922013927, 2.38, 0).

This script copies those arrays, unchanged, into one fixture.  Run it in a
container that holds the reference tree:

    python tests/golden/make_golden_units.py --ref <reference tree>
"""

import argparse
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["ac", "omegas_ac", "dp", "omegas_dp", "eps", "omegas_eps"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference source tree")
    args = ap.parse_args()
    src = os.path.join(args.ref, "tests", "test_units", "tbpm")
    arrays = {k: np.load(os.path.join(src, k + ".npy")) for k in NAMES}
    out = os.path.join(HERE, "reference_units.npz")
    np.savez(out, **arrays)
    print(out, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
