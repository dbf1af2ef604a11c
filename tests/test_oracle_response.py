"""The response oracle (oracle/response.py) pinned to the reference's RPA
numbers: in a homogeneous melt the SCF response reduces to the random-phase
approximation, whose structure factor the reference tabulates for an AB
diblock with N_A = N_B = 5, chi = 1.049 (attic/rpa/out, section of that
system: S_rpa(1,1) at q = 0.5, 1.0, 2.0).  For a plane-wave basis the
eigenvalues 1/lambda - chi of the incompressible response are
1/(2 S_rpa(q)) at q = |G + k|."""
import numpy as np

from oracle import response as R
from pscf_b200.system import Chain, System

S_RPA = {0.5: 0.2166259738636831, 1.0: 2.119413868946634, 2.0: 4.233487531254821}
CHI = 1.049


def homogeneous_diblock(ds=0.05):
    # lamellar cell of length 4 pi: G = m/2, so q = 0, 0.5, 1.0, 1.5, 2.0 on 8 points
    return System(dim=1, ngrid=[8], crystal_system="lamellar", cell_param=[4 * np.pi], kuhn=[1.0, 1.0],
                  chi=[[0.0, CHI], [CHI, 0.0]], chains=[Chain([0, 1], [5.0, 5.0])], ds=ds)


def test_response_oracle_matches_reference_rpa():
    s = homogeneous_diblock()
    r = R.Response(s, np.zeros((2, s.nr)))
    basis = [(np.array([i]), np.array([1.0 + 0j])) for i in range(s.nr)]
    smm, spm, spp, _ = r.drho_domega_id([0.0], 0.0, basis)
    ev, _ = R.drho_domega_full(smm, spm, spp, CHI, s.nr)
    assert len(ev) == s.nr - 1                      # the q = 0 eigenvalue diverges and is dropped
    for q, S in S_RPA.items():
        want = 1.0 / (2.0 * S)
        assert np.min(np.abs(ev - want)) / want < 1e-6, (q, ev, want)


def test_response_oracle_bloch_shift_is_a_relabelling():
    # a homogeneous melt: k = 0.5 (in units of 2 pi / L) gives q = 0.25, 0.75, ...
    # which equals k = 0 on a cell twice as long
    s = homogeneous_diblock()
    r = R.Response(s, np.zeros((2, s.nr)))
    basis = [(np.array([i]), np.array([1.0 + 0j])) for i in range(s.nr)]
    ev1, _ = R.drho_domega_full(*r.drho_domega_id([0.5], 0.0, basis)[:3], CHI, s.nr)
    s2 = System(dim=1, ngrid=[16], crystal_system="lamellar", cell_param=[8 * np.pi], kuhn=[1.0, 1.0],
                chi=[[0.0, CHI], [CHI, 0.0]], chains=[Chain([0, 1], [5.0, 5.0])], ds=0.05)
    r2 = R.Response(s2, np.zeros((2, s2.nr)))
    b2 = [(np.array([i]), np.array([1.0 + 0j])) for i in range(s2.nr)]
    ev2, _ = R.drho_domega_full(*r2.drho_domega_id([0.0], 0.0, b2)[:3], CHI, s2.nr)
    # every q = |m/2 + 1/4| of the first cell is a q = m'/4 of the second
    for e in ev1:
        assert np.min(np.abs(ev2 - e)) / abs(e) < 1e-9
