"""Converged omega fields of the BCC sweep fixture, solved by the oracle.

Writes tests/golden/bcc_sweep_omega.npz with the FP64 oracle's Anderson
solutions (Im-3m symmetry imposed) of sweep points 0 and 11 at the golden
cell parameters, starting from seeded tanh-sphere guesses.  The CPU golden
test restarts the oracle from these fields (a few iterations) and compares
f_Helmholtz, mu, pressure and stress with the reference's printed values.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from pscf_b200 import groups as G  # noqa: E402
from tests.cases import diblock, sphere_guess  # noqa: E402


def main():
    gold = json.load(open(os.path.join(HERE, "golden.json")))
    out = {}
    for i in (0, 11):
        B = gold["bcc_sweep"][i]
        fA = B["block_length"][0]
        s = diblock(3, [20, 20, 20], "cubic", B["cell_param"], fA=fA, chiN=15.0)
        o = O.Oracle(s)
        M, t = G.grid_ops("I m -3 m", [20, 20, 20])
        o.set_symmetry(M, t)
        w, rho, r = o.iterate_am(sphere_guess(s, fA, width=0.05), error_max=1e-11, max_itr=400)
        print(i, r, flush=True)
        out["point%d" % i] = w
    np.savez_compressed(os.path.join(HERE, "bcc_sweep_omega.npz"), **out)


if __name__ == "__main__":
    main()
