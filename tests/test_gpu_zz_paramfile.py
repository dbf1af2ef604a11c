"""A reference-style parameter file run on the GPU engine: ITERATE from a
basis-format omega file, then SWEEP in chi (src/pscf.fp.f90:520-700).  The
files written are the reference's (<prefix>0.out, 1.out, ... with their
omega and rho), and the last point equals a direct solve at its chi.
Collected after the other GPU files: it drives the whole host stack
(parameter files, sweep, response, the summary's decomposition) over the
kernels those files test."""
import numpy as np
import pytest

from pscf_b200 import field_io as F
from pscf_b200 import paramfile as P
from pscf_b200 import sweep as S
from pscf_b200.engine import Engine
from tests.cases import diblock, lamellar_guess

pytestmark = pytest.mark.gpu

TEXT = """ format  1  0

MONOMERS
N_monomer
                   2
kuhn
    1.0000000000E+00    1.0000000000E+00

CHAINS
N_chain
                   1
N_block
                   2
block_monomer
                   1                   2
block_length
    5.0000000000E-01    5.0000000000E-01

COMPOSITION
ensemble
                   0
phi_chain
    1.0000000000E+00

INTERACTION
interaction_type
               'chi'
chi
    1.5000000000E+01

UNIT_CELL
dim
                   1
crystal_system
          'lamellar'
N_cell_param
                   1
cell_param
    1.5000000000E+00

DISCRETIZATION
ngrid
                  32
chain_step
    1.0000000000E-02

BASIS
group_name
                '-1'

ITERATE
input_filename
          'in.omega'
output_prefix
              'out/'
max_itr
                 500
error_max
    1.0000000000E-10
domain
                   T
itr_algo
                'AM'
N_hist
                  20

SWEEP
s_max
    2.0000000000E+00
d_chi
    5.0000000000E-01
end_increments

FINISH
"""


def test_iterate_and_sweep_from_a_parameter_file(tmp_path):
    s = diblock(1, [32], "lamellar", [1.5], fA=0.5, chiN=15.0)
    F.write_field(str(tmp_path / "in.omega"), lamellar_guess(s), s, "-1")
    (tmp_path / "param").write_text(TEXT)
    st = P.run_param(str(tmp_path / "param"))
    assert st["result"]["converged"] and len(st["sweep"]) == 3
    for j, chi in enumerate((15.0, 15.5, 16.0)):
        d = S.read_out(str(tmp_path / "out" / f"{j}.out"))
        assert abs(d["chi"][0] - chi) < 1e-6, (j, d["chi"])
        assert (tmp_path / "out" / f"{j}.omega").exists() and (tmp_path / "out" / f"{j}.rho").exists()
    last, mid = st["sweep"][-1], st["sweep"][1]
    # an independent solve at chi = 16, started from the chi = 15.5 point
    s16 = diblock(1, [32], "lamellar", list(mid.system.cell_param), fA=0.5, chiN=16.0)
    e = Engine([s16])
    e.set_symmetry(0, "-1")
    _, _, r = e.iterate_am(mid.omega[None], error_max=1e-10, max_itr=1000, domain=True)
    e.close()
    assert r[0]["converged"]
    assert abs(last.result["f_helmholtz"] - r[0]["f_helmholtz"]) < 1e-8
    assert abs(last.system.cell_param[0] - r[0]["cell_param"][0]) < 1e-6
    d2 = S.read_out(str(tmp_path / "out" / "2.out"))
    assert abs(d2["f_Helmholtz"][0] - r[0]["f_helmholtz"]) < 1e-8


RESPONSE = """RESPONSE
k_group
                 '1'
kdim
                   1
kvec
    1.0000000000E-01
nkstep
                   1
dkvec
    2.0000000000E-01
n_eigval_out
                   4
n_eigvec_out
                   1
n_basis_out
                   4

FINISH
"""


def test_iterate_and_response_from_a_parameter_file(tmp_path):
    """ITERATE then RESPONSE (src/pscf.fp.f90:707-723) on the engine: the
    eigenvalues in <prefix>0.eval and 1.eval equal the oracle's response
    of the converged state at k = 0.1 and 0.3."""
    from tests.test_paramfile import _oracle_response_sweep
    s = diblock(1, [32], "lamellar", [1.5], fA=0.5, chiN=15.0)
    F.write_field(str(tmp_path / "in.omega"), lamellar_guess(s), s, "-1")
    (tmp_path / "param").write_text(TEXT.split("SWEEP\n")[0] + RESPONSE)
    st = P.run_param(str(tmp_path / "param"))
    assert st["result"]["converged"] and len(st["response"]) == 2
    want = _oracle_response_sweep(st["system"], st["omega"],
                                  dict(k_group="1", kvec0=[0.1], dkvec=[0.2], nkstep=1, n_eigval_out=4))
    for j, pt in enumerate(want):
        lines = open(tmp_path / "out" / f"{j}.eval").read().splitlines()
        ev = [float(x.split()[0]) for x in lines[3:]]
        # absolute as well as relative: the lowest eigenvalue of an ordered phase
        # at small k lies near the translation mode's zero
        np.testing.assert_allclose(ev, pt["eval"], rtol=1e-7, atol=1e-7)
        np.testing.assert_allclose(st["response"][j]["eval"], pt["eval"], rtol=1e-7, atol=1e-7)
        assert (tmp_path / "out" / f"{j}.evec.1").exists()
