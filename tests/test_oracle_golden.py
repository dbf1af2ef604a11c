"""The FP64 oracle reproduces the reference's own converged outputs.

Golden values are the reference's printed results (10 significant digits)
extracted by tests/golden/make_golden.py; fields of the BCC sweep come from
tests/golden/make_bcc_fixture.py.  Agreement is required to 1e-10, i.e. the
print precision plus the convergence tolerance.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from pscf_b200 import groups as G
from tests.cases import diblock, lamellar_guess

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))
TOL = 1e-10


def _check(r, g):
    assert r["converged"]
    assert abs(r["f_helmholtz"] - g["f_Helmholtz"][0]) < TOL
    assert abs(r["mu_chain"][0] - g["mu_chain"][0]) < TOL
    assert abs(r["pressure"] - g["pressure"][0]) < TOL
    assert abs(r["stress"][0]) < TOL


def test_lamellar_outfile_golden():
    g = GOLD["lamellar_outfile"]
    s = diblock(1, [32], "lamellar", g["cell_param"], fA=g["block_length"][0], chiN=g["chi"][0])
    o = O.Oracle(s)
    M, t = G.grid_ops("-1", [32])
    o.set_symmetry(M, t)
    w, rho, r = o.iterate_am(lamellar_guess(s), error_max=1e-11, max_itr=500)
    _check(r, g)
    assert abs(O.free_energy_fh(s) - g["f_homo"][0]) < TOL


def test_lamellar_without_star_weights_differs_by_fp32_normalisation():
    """Without the single-precision star normalisation of the reference
    basis (src/basis_mod.f90:920) the field term differs by exactly the
    N=2 star weight: F_plain - F_ref = (1 - r2) * (non-uniform field term)."""
    g = GOLD["lamellar_outfile"]
    s = diblock(1, [32], "lamellar", g["cell_param"], fA=0.5, chiN=g["chi"][0])
    o = O.Oracle(s)
    w, rho, r = o.iterate_am(lamellar_guess(s), error_max=1e-11, max_itr=500)
    sf = np.float32(np.sqrt(np.float32(2.0)))
    r2 = float(sf) * float(sf) / 2.0
    chi = g["chi"][0]
    uniform = chi * 0.25 - 7.5 * 0.5 * 2  # k = 0 star: rho_A chi rho_B - sum omega rho
    field = r["f_helmholtz"] - (r["mu_chain"][0] - 1.0)
    predicted = r["f_helmholtz"] - (1 - r2) * (field - uniform)
    assert abs(predicted - g["f_Helmholtz"][0]) < TOL
    assert abs(r["f_helmholtz"] - g["f_Helmholtz"][0]) > 5e-8


@pytest.mark.parametrize("point", [0, 11])
def test_bcc_sweep_golden(point):
    g = GOLD["bcc_sweep"][point]
    fix = np.load(os.path.join(HERE, "golden", "bcc_sweep_omega.npz"))
    s = diblock(3, [20, 20, 20], "cubic", g["cell_param"], fA=g["block_length"][0], chiN=g["chi"][0])
    o = O.Oracle(s)
    M, t = G.grid_ops("I m -3 m", [20, 20, 20])
    o.set_symmetry(M, t)
    w, rho, r = o.iterate_am(fix["point%d" % point], error_max=5e-11, max_itr=20)
    _check(r, g)
    assert abs(O.free_energy_fh(s) - g["f_homo"][0]) < TOL
