"""The reference's BCC sweep re-run through the sweep driver on the GPU
engine: ITERATE at f_A = 0.39, then SWEEP with block-length increments
(-0.01, +0.01) to s_max = 11 with cell relaxation (src/pscf.fp.f90:557-700,
src/sweep_mod.f90:407-600).  Every integer point is compared with the
reference's printed output files tools/python/tests/sweep/out/{0..11}.out
(tests/golden/golden.json), and the output files it writes parse back."""
import json
import os

import numpy as np
import pytest

from pscf_b200 import sweep as S
from pscf_b200.field_io import read_field
from tests.cases import diblock

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))["bcc_sweep"]


def test_bcc_sweep_through_the_driver(tmp_path):
    g0 = GOLD[0]
    s = diblock(3, [20, 20, 20], "cubic", g0["cell_param"], fA=0.39, chiN=15.0)
    w0 = np.load(os.path.join(HERE, "golden", "bcc_sweep_omega.npz"))["point0"]
    inc = S.Increments(block_length=[[-0.01, 0.01]])
    solve = S.am_solver("I m -3 m", error_max=1e-11, max_itr=600, n_hist=20, domain=True)
    it = dict(input_filename="in.omega", output_prefix="out/", max_itr=600, error_max=1e-11, domain=True,
              itr_algo="AM", N_hist=20)
    prefix = str(tmp_path / "out") + "/"
    pts = S.run_sweep(s, w0, inc, 11.0, solve, domain=True, out_prefix=prefix, group_name="I m -3 m",
                      iterate=it, n_star=int(g0["N_star"][0]))
    assert [round(p.s, 6) for p in pts] == [float(j) for j in range(12)]
    for j, (p, g) in enumerate(zip(pts, GOLD)):
        r = p.result
        # the reference stopped its Newton iterations at errors of 1e-10 to
        # 1e-8 (final_error of each file); these points are solved to 1e-11
        tol = 2e-10 + 2 * g["final_error"][0]
        assert abs(p.system.chains[0].block_length[0] - g["block_length"][0]) < 2e-11, j
        assert abs(p.system.cell_param[0] - g["cell_param"][0]) < 5e-10 + 5 * g["final_error"][0], j
        assert abs(r["f_helmholtz"] - g["f_Helmholtz"][0]) < tol, j
        assert abs(r["mu_chain"][0] - g["mu_chain"][0]) < tol, j
        assert abs(r["pressure"] - g["pressure"][0]) < tol, j
        d = S.read_out(f"{prefix}{j}.out")
        assert abs(d["f_Helmholtz"][0] - r["f_helmholtz"]) < 1e-10 * abs(r["f_helmholtz"])
        assert abs(d["f_homo"][0] - g["f_homo"][0]) < 1e-9
        assert d["cell_param"][0] == pytest.approx(p.system.cell_param[0], rel=1e-10)
    # the basis-format field files of the last point read back as its fields
    _, w11 = read_field(f"{prefix}11.omega", pts[-1].system)
    assert np.max(np.abs(w11 - pts[-1].omega)) < 1e-9 * np.max(np.abs(pts[-1].omega))
