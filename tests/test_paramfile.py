"""The reference's parameter files (pscf_b200.paramfile), on the CPU: the
system sections of the reference's own file (tests/golden/lamellar.out, a
copy of tools/python/tests/outfile/in, whose first part is the parameter
file of its run), a SWEEP section's increments, and the field conversion
commands on the reference's own field file."""
import os

import numpy as np
import pytest

from pscf_b200 import field_io as F
from pscf_b200 import paramfile as P

HERE = os.path.dirname(os.path.abspath(__file__))


def test_reference_file_system_and_iterate():
    param = P.read_param(os.path.join(HERE, "golden", "lamellar.out"))
    assert [n for n, _ in param][-2:] == ["ITERATE", "FINISH"]
    s, group = P.system_of(param)
    assert group == "-1" and s.dim == 1 and list(s.ngrid) == [32] and s.ds == 0.01
    assert s.crystal_system == "lamellar" and s.cell_param == [1.5161093081]
    assert s.chains[0].block_monomer == [0, 1] and s.chains[0].block_length == [0.5, 0.5]
    assert s.chi[0, 1] == s.chi[1, 0] == 15.000000011 and s.kuhn == [1.0, 1.0]
    it = P._iterate_params(dict(param)["ITERATE"])
    assert it == dict(input_filename="in.omega", output_prefix="out/", max_itr=20, error_max=1e-8, domain=True,
                      itr_algo="NR", N_cut=17)


PARAM = """ format  1  0

MONOMERS
N_monomer
                   3
kuhn
    1.0000000000E+00    1.1000000000E+00    0.9000000000E+00

CHAINS
N_chain
                   2
N_block
                   3
                   1
block_monomer
                   1                   2                   3
                   2
block_length
    3.0000000000E-01    4.0000000000E-01    3.0000000000E-01
    5.0000000000E-01

COMPOSITION
ensemble
                   0
phi_chain
    8.0000000000E-01
    2.0000000000E-01

INTERACTION
interaction_type
               'chi'
chi
    1.2000000000E+01
    2.0000000000E+01    1.5000000000E+01

UNIT_CELL
dim
                   2
crystal_system
         'hexagonal'
N_cell_param
                   1
cell_param
    1.9000000000E+00

DISCRETIZATION
ngrid
                  24                  24
chain_step
    1.0000000000E-02

BASIS
group_name
          'p 6 m m'

ITERATE
input_filename
          'in.omega'
output_prefix
              'out/'
max_itr
                 200
error_max
    1.0000000000E-08
domain
                   F
itr_algo
                'AM'
N_hist
                  10

SWEEP
s_max
    4.0000000000E+00
d_chi
    1.0000000000E+00
    0.0000000000E+00    5.0000000000E-01
d_block_length
   -1.0000000000E-02    0.0000000000E+00    1.0000000000E-02
    0.0000000000E+00
d_phi_chain
   -5.0000000000E-02    5.0000000000E-02
end_increments

FINISH
"""


def test_three_monomer_file_with_sweep(tmp_path):
    p = tmp_path / "param"
    p.write_text(PARAM)
    param = P.read_param(str(p))
    assert [n for n, _ in param][-3:] == ["ITERATE", "SWEEP", "FINISH"]
    s, group = P.system_of(param)
    assert group == "p 6 m m" and s.n_monomer == 3 and len(s.chains) == 2
    assert s.chains[0].block_monomer == [0, 1, 2] and s.chains[1].block_monomer == [1]
    assert s.chi[1, 0] == 12.0 and s.chi[2, 0] == 20.0 and s.chi[2, 1] == 15.0
    assert [c.phi for c in s.chains] == [0.8, 0.2]
    s_max, inc = P.increments_of(dict(param)["SWEEP"], s)
    assert s_max == 4.0
    assert inc.chi[1, 0] == 1.0 and inc.chi[2, 1] == 0.5 and inc.chi[2, 0] == 0.0
    assert inc.block_length == [[-0.01, 0.0, 0.01], [0.0]] and inc.phi_chain == [-0.05, 0.05]
    it = P._iterate_params(dict(param)["ITERATE"])
    assert it["itr_algo"] == "AM" and it["N_hist"] == 10 and it["domain"] is False


def test_field_conversion_commands(tmp_path):
    """FIELD_TO_RGRID, RGRID_TO_FIELD and RHO_TO_OMEGA on the reference's
    own rho file (group -1, 40 points): the grid file holds the field, the
    round trip restores every coefficient, and omega = chi rho."""
    import shutil
    h = F._read_header(open(os.path.join(HERE, "golden", "fieldfile_rho.txt")).read().splitlines())[0]
    shutil.copy(os.path.join(HERE, "golden", "fieldfile_rho.txt"), tmp_path / "rho")
    text = f""" format  1  0

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
    5.6000000000E-01    4.4000000000E-01

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
{h["cell_param"][0]:20.10E}

DISCRETIZATION
ngrid
                  40
chain_step
    1.0000000000E-02

BASIS
group_name
                '-1'

FIELD_TO_RGRID
input_filename
               'rho'
output_filename
             'rho.rg'

RGRID_TO_FIELD
input_filename
             'rho.rg'
output_filename
            'rho.back'

RHO_TO_OMEGA
input_filename
               'rho'
output_filename
             'omega'

FINISH
"""
    (tmp_path / "param").write_text(text)
    st = P.run_param(str(tmp_path / "param"))
    s = st["system"]
    _, rho = F.read_field(str(tmp_path / "rho"), s)
    _, _, rg = F.read_rgrid(str(tmp_path / "rho.rg"))
    assert np.max(np.abs(rg - rho)) < 5e-9                         # F18.9 grid values
    _, back = F.read_field(str(tmp_path / "rho.back"), s)
    assert np.max(np.abs(back - rho)) < 5e-9
    _, w = F.read_field(str(tmp_path / "omega"), s)
    np.testing.assert_allclose(w, s.chi @ rho, atol=1e-9)
    with pytest.raises(NotImplementedError):
        (tmp_path / "p2").write_text(text.replace("FIELD_TO_RGRID", "OUTPUT_WAVES", 1))
        P.run_param(str(tmp_path / "p2"))
