"""Linear response (RESPONSE) on the GPU against the numpy oracle
(oracle/response.py, itself pinned to the reference's RPA table)."""
import numpy as np
import pytest

from oracle import response as R
from pscf_b200 import groups as G
from pscf_b200.engine import FP32, FP64, Engine, EngineError
from pscf_b200.response import drho_domega_full, drho_domega_id, perturbation_basis, response_sweep
from pscf_b200.system import Chain, System
from tests.cases import diblock, lamellar_guess, omega_guess, rel_err

pytestmark = pytest.mark.gpu

S_RPA = {0.5: 0.2166259738636831, 1.0: 2.119413868946634, 2.0: 4.233487531254821}


def _sym_omega(s, group, seed):
    w = omega_guess(s, seed, 2.0)
    return np.stack([G.symmetrize(w[a], group, s.ngrid) for a in range(2)])


def _compare(s, w, kvec, k_group, ktrans=0.0, tol=1e-10):
    basis = perturbation_basis(k_group, s.ngrid)
    e = Engine([s], FP64)
    e.density(w[None])
    got = drho_domega_id(e, 0, kvec, basis, ktrans)
    want = R.Response(s, w).drho_domega_id(kvec, ktrans, basis)[:3]
    for g, x in zip(got, want):
        assert rel_err(g, x) < tol
    e.close()
    return got


def test_response_lamellar_matches_oracle():
    s = diblock(1, [16], "lamellar", [1.7], fA=0.4, chiN=14.0, ds=0.05)
    _compare(s, lamellar_guess(s, 3.0), [0.3], "1")


def test_response_lamellar_transverse_k_matches_oracle():
    s = diblock(1, [16], "lamellar", [1.7], fA=0.4, chiN=14.0, ds=0.05)
    Gb = s.unit_cell()[0]
    kvec = [0.2, 0.35]
    kt = R.transverse_ksq(1, Gb, kvec)
    assert kt > 0
    _compare(s, lamellar_guess(s, 3.0), kvec[:1], "1", kt)


def test_response_hexagonal_matches_oracle():
    s = diblock(2, [8, 8], "hexagonal", [1.9], fA=0.3, chiN=16.0, ds=0.05)
    _compare(s, _sym_omega(s, "p 6 m m", 3), [0.2, 0.1], "p 1")


def test_response_cubic_general_k_matches_oracle():
    s = diblock(3, [4, 4, 4], "cubic", [1.9], fA=0.3, chiN=16.0, ds=0.05)
    _compare(s, omega_guess(s, 4, 1.5), [0.1, 0.2, 0.3], "P 1")


def test_response_bcc_gamma_symmetric_basis_matches_oracle():
    s = diblock(3, [8, 8, 8], "cubic", [1.95], fA=0.25, chiN=20.0, ds=0.05)
    _compare(s, _sym_omega(s, "I m -3 m", 5), [0.0, 0.0, 0.0], "I m -3 m")


def test_response_homogeneous_melt_gives_reference_rpa():
    chi = 1.049
    s = System(dim=1, ngrid=[8], crystal_system="lamellar", cell_param=[4 * np.pi], kuhn=[1.0, 1.0],
               chi=[[0.0, chi], [chi, 0.0]], chains=[Chain([0, 1], [5.0, 5.0])], ds=0.05)
    e = Engine([s], FP64)
    e.density(np.zeros((1, 2, s.nr)))
    res = response_sweep(e, 0, [0.0], [0.5], 1, "1", s.nr)
    ev = res[0]["eval"]
    assert len(ev) == s.nr - 1
    for q, S in S_RPA.items():
        want = 1.0 / (2.0 * S)
        assert np.min(np.abs(ev - want)) / want < 1e-6
    # k = 1/2: q = 0.25, 0.75, 1.25, 1.75 (each twice), none divergent
    assert len(res[1]["eval"]) == s.nr
    e.close()


def test_response_requires_density_and_fp64():
    s = diblock(1, [16], "lamellar", [1.7], fA=0.4, ds=0.05)
    basis = perturbation_basis("1", s.ngrid)
    e = Engine([s], FP64)
    with pytest.raises(EngineError):
        drho_domega_id(e, 0, [0.1], basis)
    e.close()
    e = Engine([s], FP32)
    e.density(lamellar_guess(s)[None])
    with pytest.raises(EngineError):
        drho_domega_id(e, 0, [0.1], basis)
    e.close()
