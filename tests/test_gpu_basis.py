"""Fields in star coefficients on the device (pscfg_set_basis,
pscfg_density_basis): basis_to_kgrid and the inverse FFT of omega, the
density, the forward FFT and kgrid_to_basis of rho
(src/grid_basis_mod.f90:47-200, src/scf_mod.fp.f90:144-229), against the
grid entry point and the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from pscf_b200 import groups as G
from pscf_b200.basis import StarBasis
from pscf_b200.engine import Engine, FP64
from tests.cases import diblock, omega_guess, rel_err

pytestmark = pytest.mark.gpu

CASES = [("I m -3 m", 3, [20, 20, 20], "cubic", [3.9]),
         ("I a -3 d", 3, [16, 16, 16], "cubic", [3.7]),
         ("p 6 m m", 2, [24, 24], "hexagonal", [1.9]),
         ("-1", 1, [32], "lamellar", [1.7]),
         ("-1", 1, [27], "lamellar", [1.4]),
         # groups without inversion: cosine / sine pairs of stars share their
         # half-grid waves (I 41 3 2 also has sine-like closed stars)
         ("I 41 3 2", 3, [16, 16, 16], "cubic", [3.7]),
         ("1", 1, [32], "lamellar", [1.7])]


def _symmetric_omega(s, group, seed):
    w = omega_guess(s, seed, 2.0)
    return np.stack([G.symmetrize(w[a], group, list(s.ngrid)) for a in range(s.n_monomer)])


@pytest.mark.parametrize("group,dim,ngrid,crystal,cell", CASES)
def test_density_basis_matches_grid_path_and_oracle(group, dim, ngrid, crystal, cell):
    s = diblock(dim, ngrid, crystal, cell, fA=0.35, chiN=15.0, ds=0.02)
    b = StarBasis(group, ngrid)
    w = _symmetric_omega(s, group, 5)
    wb = np.stack([b.to_basis(w[a]) for a in range(2)])
    e = Engine([s], FP64)
    e.set_basis(0, b)
    rb, q = e.density_basis([wb])
    rho_g, q_g = e.density(w[None])
    o = O.Oracle(s)
    rho_ref, q_ref = o.density(w)
    rb_ref = np.stack([b.to_basis(rho_ref[a]) for a in range(2)])
    assert rel_err(q[0, :1], q_ref) < 1e-12 and rel_err(q_g[0, :1], q_ref) < 1e-12
    assert rel_err(rb[0], rb_ref) < 1e-12, rel_err(rb[0], rb_ref)
    np.testing.assert_allclose(rb[0], np.stack([b.to_basis(rho_g[0, a]) for a in range(2)]), rtol=0, atol=1e-13)
    e.close()


def test_density_basis_batched_instances_with_their_own_bases():
    """Two instances of one grid shape, each with its own group and star
    count, packed one after another."""
    ss = [diblock(3, [16, 16, 16], "cubic", [3.9], fA=0.3, chiN=15.0, ds=0.02),
          diblock(3, [16, 16, 16], "cubic", [3.7], fA=0.4, chiN=16.0, ds=0.02)]
    groups = ["I m -3 m", "I a -3 d"]
    bases = [StarBasis(g, [16, 16, 16]) for g in groups]
    assert bases[0].n_star != bases[1].n_star
    e = Engine(ss, FP64)
    wbs, refs = [], []
    for i, (s, g, b) in enumerate(zip(ss, groups, bases)):
        e.set_basis(i, b)
        w = _symmetric_omega(s, g, 11 + i)
        wbs.append(np.stack([b.to_basis(w[a]) for a in range(2)]))
        rho_ref, _ = O.Oracle(s).density(np.stack([b.to_grid(wbs[-1][a]) for a in range(2)]))
        refs.append(np.stack([b.to_basis(rho_ref[a]) for a in range(2)]))
    rb, q = e.density_basis(wbs)
    for i in range(2):
        assert rel_err(rb[i], refs[i]) < 1e-12, (i, rel_err(rb[i], refs[i]))
    e.close()


def test_density_basis_requires_tables():
    from pscf_b200.engine import EngineError
    s = diblock(1, [32], "lamellar", [1.7])
    e = Engine([s], FP64)
    e._n_star = [3]
    with pytest.raises(EngineError):
        e.density_basis([np.zeros((2, 3))])
    e.close()
