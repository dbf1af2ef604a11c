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


def _oracle_decompose(system, group, omega, f_total):
    """_decompose with the oracle's density and propagators in place of the
    engine's (the CPU stand-in)."""
    from oracle import oracle as O
    from pscf_b200.sweep import divide_energy
    from pscf_b200.system import chain_grid
    w = np.asarray(omega, dtype=np.float64).reshape(system.n_monomer, system.nr)
    o = O.Oracle(system)
    rho, q = o.density(w)
    junctions = []
    for c, chain in enumerate(system.chains):
        qf, qr = o.propagators(c)
        bgn, _ = chain_grid(chain.block_length, system.ds)
        h, t = bgn[1], bgn[len(chain.block_length) - 1]
        junctions.append((qf[h], qr[h], qf[t], qr[t]))
    fb = F.field_basis(group, system)
    fc, ov = divide_energy(system, np.stack([fb.to_coeffs(x) for x in w]), np.stack([fb.to_coeffs(x) for x in rho]),
                           q, junctions, f_total)
    return dict(f_component=fc, overlap=ov, q_solvent=[])


_ENGINE_DECOMPOSE = P._decompose          # the product's, before the fixture below replaces it


@pytest.fixture(autouse=True)
def _decompose_on_the_oracle(monkeypatch):
    monkeypatch.setattr(P, "_decompose", _oracle_decompose)


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


_TWO_MONOMER = """ format  1  0

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
@CELL@

DISCRETIZATION
ngrid
                  40
chain_step
    1.0000000000E-02

BASIS
group_name
                '-1'

"""


def test_field_conversion_commands(tmp_path):
    """FIELD_TO_RGRID, RGRID_TO_FIELD and RHO_TO_OMEGA on the reference's
    own rho file (group -1, 40 points): the grid file holds the field, the
    round trip restores every coefficient, and omega = chi rho."""
    import shutil
    h = F._read_header(open(os.path.join(HERE, "golden", "fieldfile_rho.txt")).read().splitlines())[0]
    shutil.copy(os.path.join(HERE, "golden", "fieldfile_rho.txt"), tmp_path / "rho")
    text = _TWO_MONOMER.replace("@CELL@", f'{h["cell_param"][0]:20.10E}') + """FIELD_TO_RGRID
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
    for listing in ("OUTPUT_WAVES", "OUTPUT_GROUP", "OUTPUT_GROUP_CPP", "WRITE_GROUPS"):
        (tmp_path / "p2").write_text(text.replace("FIELD_TO_RGRID", listing, 1))
        with pytest.raises(NotImplementedError):
            P.run_param(str(tmp_path / "p2"))


def test_rescale_reference_volume(tmp_path, monkeypatch):
    """RESCALE (src/pscf.fp.f90:414-455, rescale_vref
    src/chemistry_mod.f90:1344-1361): v -> v / lambda divides kuhn by
    sqrt(lambda) and chi and omega by lambda and multiplies block lengths and
    solvent sizes by lambda, so chi N, omega N and b N^(1/2) stay; the
    ITERATE after it has no input_filename and starts from omega / lambda."""
    import shutil
    from pscf_b200.sweep import read_out
    from pscf_b200.system import Solvent
    base = PARAM.split("ITERATE")[0]
    s0, group = P.system_of(P.read_param_text(base + "FINISH\n"))
    s0.solvents = [Solvent(monomer=2, size=0.2, phi=0.0)]
    lam = 2.0
    s1 = P.rescale_vref(s0, lam)
    for c0, c1 in zip(s0.chains, s1.chains):
        np.testing.assert_allclose(np.sum(c1.block_length) * s1.chi, np.sum(c0.block_length) * s0.chi)
        np.testing.assert_allclose(np.sqrt(np.sum(c1.block_length)) * np.array(s1.kuhn),
                                   np.sqrt(np.sum(c0.block_length)) * np.array(s0.kuhn))
    assert s1.solvents[0].size == 0.4 and s0.solvents[0].size == 0.2       # the input is not modified
    # interaction_type 'chi_T': chi_A and chi_B scale, the temperature stays
    from pscf_b200.system import Chain, System
    t0 = System(dim=1, ngrid=[16], crystal_system="lamellar", cell_param=[1.7], kuhn=[1.0, 1.0],
                chi=np.zeros((2, 2)), chains=[Chain([0, 1], [0.5, 0.5])], ds=0.01,
                chi_A=[[0.0, 3000.0], [3000.0, 0.0]], chi_B=[[0.0, -2.0], [-2.0, 0.0]], temperature=200.0)
    t1 = P.rescale_vref(t0, 4.0)
    assert t1.temperature == 200.0 and t1.chi_A[0, 1] == 750.0 and t1.chi_B[0, 1] == -0.5
    assert abs(t1.chi[0, 1] - t0.chi[0, 1] / 4.0) < 1e-15 and t1.chains[0].block_length == [2.0, 2.0]
    it = P._iterate_params(dict(output_prefix=["out/"], max_itr=[10.0], error_max=[1e-8], domain=["F"],
                                itr_algo=["AM"], N_hist=[5.0]))
    assert it["input_filename"] is None
    # a file with RESCALE + ITERATE, run with a stand-in solver
    shutil.copy(os.path.join(HERE, "golden", "fieldfile_rho.txt"), tmp_path / "in.omega")
    h = F._read_header(open(tmp_path / "in.omega").read().splitlines())[0]
    cell = f"{h['cell_param'][0]:20.10E}"
    text = (_TWO_MONOMER.replace("@CELL@", cell) + "RESCALE\ninput_filename\n          'in.omega'\nvref_scale\n"
            "    4.0000000000E+00\n\nITERATE\noutput_prefix\n              'out/'\nmax_itr\n"
            "                 100\nerror_max\n    1.0000000000E-08\ndomain\n                   F\n"
            "itr_algo\n                'AM'\nN_hist\n                  10\n\nFINISH\n")
    (tmp_path / "param").write_text(text)
    seen = {}

    def fake_solver(it, group):
        def solve(system, w0):
            seen.update(system=system, w0=w0, it=it)
            r = dict(converged=True, itr=1, error=1e-9, f_helmholtz=1.0, pressure=2.0, stress=[0.0],
                     mu_chain=[3.0], cell_param=list(system.cell_param))
            return w0, w0, r
        return solve
    monkeypatch.setattr(P, "_solver", fake_solver)
    st = P.run_param(str(tmp_path / "param"))
    s = seen["system"]
    assert s.chains[0].block_length == [0.56 * 4.0, 0.44 * 4.0] and s.kuhn == [0.5, 0.5]
    assert abs(s.chi[0, 1] - 15.0 / 4.0) < 1e-15 and seen["it"]["input_filename"] == "in.omega"
    _, w = F.read_field(str(tmp_path / "in.omega"), s)
    np.testing.assert_array_equal(seen["w0"], w / 4.0)
    d = read_out(str(tmp_path / "out" / "out"))
    assert d["block_length"] == [2.24, 1.76] and d["input_filename"] == ["in.omega"]
    (tmp_path / "p2").write_text(text.replace("RESCALE\ninput_filename\n          'in.omega'\nvref_scale\n"
                                              "    4.0000000000E+00\n\n", ""))
    with pytest.raises(ValueError):
        P.run_param(str(tmp_path / "p2"))


def test_kgrid_to_rgrid(tmp_path):
    """KGRID_TO_RGRID (src/pscf.fp.f90:813-888): a wave-grid file of the
    reference's rho (Fortran list-directed '(re , im)' values) gives the
    same coordinate grid as FIELD_TO_RGRID of the basis file; each star's
    coefficient comes from its own wave (kgrid_to_basis), so a change at
    another wave of the star does not move it; a wrong grid raises."""
    import shutil
    h = F._read_header(open(os.path.join(HERE, "golden", "fieldfile_rho.txt")).read().splitlines())[0]
    shutil.copy(os.path.join(HERE, "golden", "fieldfile_rho.txt"), tmp_path / "rho")
    sys_text = _TWO_MONOMER.replace("@CELL@", f'{h["cell_param"][0]:20.10E}')
    (tmp_path / "p0").write_text(sys_text + "FINISH\n")
    s, group = P.system_of(P.read_param(str(tmp_path / "p0")))
    _, rho = F.read_field(str(tmp_path / "rho"), s)
    F.write_kgrid(str(tmp_path / "rho.kg"), rho, s, group)
    # the Fortran list-directed form of the same values
    lines = open(tmp_path / "rho.kg").read().splitlines()
    nh = len(lines) - (s.n[0] // 2 + 1)
    fort = lines[:nh] + [ln.replace("(", "(  ").replace(",", "     ,  ").replace(")", "     )").replace("E", "D")
                         for ln in lines[nh:]]
    (tmp_path / "rho.kgf").write_text("\n".join(fort) + "\n")
    text = sys_text + ("KGRID_TO_RGRID\ninput_filename\n             'rho.kgf'\noutput_filename\n"
                       "              'a.rg'\n\nFIELD_TO_RGRID\ninput_filename\n               'rho'\n"
                       "output_filename\n              'b.rg'\n\nFINISH\n")
    (tmp_path / "param").write_text(text)
    P.run_param(str(tmp_path / "param"))
    assert open(tmp_path / "a.rg").read() == open(tmp_path / "b.rg").read()
    _, spec = F.read_kgrid(str(tmp_path / "rho.kg"), s)
    fb = F.FieldBasis(group, s)
    c0 = fb.spectrum_to_coeffs(spec[0])
    st = next(x for x in fb.stars if len(x["idx"]) > 1)
    other = next(int(k) for k in st["idx"] if int(k) != st["wave"])
    bumped = spec[0].copy()
    bumped[other] += 0.5
    np.testing.assert_array_equal(fb.spectrum_to_coeffs(bumped), c0)
    s2, _ = P.system_of(P.read_param_text(sys_text.replace("                  40\n", "                  20\n")
                                          + "FINISH\n"))
    with pytest.raises(ValueError):
        F.read_kgrid(str(tmp_path / "rho.kg"), s2)


def _oracle_response_sweep(system, omega, rp):
    """response_sweep of pscf_b200.response with the oracle in place of the
    engine (the CPU stand-in for _response_sweep)."""
    from oracle import response as R
    from pscf_b200.response import perturbation_basis
    basis = perturbation_basis(rp["k_group"], system.ngrid)
    resp = R.Response(system, np.asarray(omega).reshape(system.n_monomer, system.nr))
    G = system.unit_cell()[0]
    out, k = [], np.array(rp["kvec0"], dtype=float)
    for _ in range(rp["nkstep"] + 1):
        kt = R.transverse_ksq(system.dim, G, k)
        smm, spm, spp = resp.drho_domega_id(k[:system.dim], kt, basis)[:3]
        ev, V = R.drho_domega_full(smm, spm, spp, float(system.chi[0, 1]), rp["n_eigval_out"])
        out.append({"kvec": k.copy(), "eval": ev, "evec": V, "n_basis": len(basis)})
        k = k + np.asarray(rp["dkvec"])
    return out


def test_fortran_e_format():
    assert P._fortran_e(1.0) == "     0.100000000E+01"
    assert P._fortran_e(-0.5) == "    -0.500000000E+00"
    assert P._fortran_e(0.0) == "     0.000000000E+00"
    assert P._fortran_e(9.9999999999) == "     0.100000000E+02"
    assert P._fortran_e(-1.234567891e-5) == "    -0.123456789E-04"
    assert P._fortran_e(1e-101) == "     0.100000000-100"


def test_response_command(tmp_path, monkeypatch):
    """RESPONSE (src/pscf.fp.f90:707-723; response_sweep and
    calc_drho_domega_full, src/response_mod.f90:309-389, 497-652): the
    section is read in the reference's order (no dkvec when nkstep = 0),
    needs an ITERATE (or SWEEP) just before it, and writes
    <prefix>j.eval (q_vec, N_basis, E20.9 eigenvalues) and
    <prefix>j.evec.k (the eigenvector's first n_basis_out coefficients,
    +v / -v for the two monomers) per k point.  The engine's response is
    stood in for by the oracle here; the GPU test runs the engine."""
    import shutil
    rp = P.response_params({"k_group": ["1"], "kdim": [1.0], "kvec0": [0.0], "nkstep": [0.0],
                            "n_eigval_out": [4.0], "n_eigvec_out": [1.0], "n_basis_out": [3.0]}, 1)
    assert rp["dkvec"] == [0.0] and rp["n_basis_out"] == 3
    assert P.response_params({"a": ["P 1"], "b": [2.0], "c": [0.1, 0.2], "d": [1.0], "e": [0.0, 0.1],
                              "f": [1.0, 1.0, 1.0]}, 1)["k_group"] == "1"
    with pytest.raises(ValueError):
        P.response_params({"k_group": ["1"], "kdim": [3.0]}, 1)
    shutil.copy(os.path.join(HERE, "golden", "fieldfile_rho.txt"), tmp_path / "in.omega")
    h = F._read_header(open(tmp_path / "in.omega").read().splitlines())[0]
    sys_text = _TWO_MONOMER.replace("@CELL@", f'{h["cell_param"][0]:20.10E}')
    iterate = ("ITERATE\ninput_filename\n          'in.omega'\noutput_prefix\n              'out/'\nmax_itr\n"
               "                 100\nerror_max\n    1.0000000000E-08\ndomain\n                   F\n"
               "itr_algo\n                'AM'\nN_hist\n                  10\n\n")
    response = ("RESPONSE\nk_group\n                 '1'\nkdim\n                   1\nkvec\n"
                "    1.0000000000E-01\nnkstep\n                   1\ndkvec\n    2.0000000000E-01\n"
                "n_eigval_out\n                   5\nn_eigvec_out\n                   2\nn_basis_out\n"
                "                   6\n\n")

    def fake_solver(it, group):
        def solve(system, w0):
            r = dict(converged=True, itr=1, error=1e-9, f_helmholtz=1.0, pressure=2.0, stress=[0.0],
                     mu_chain=[3.0], cell_param=list(system.cell_param))
            return w0, w0, r
        return solve
    monkeypatch.setattr(P, "_solver", fake_solver)
    monkeypatch.setattr(P, "_response_sweep", _oracle_response_sweep)
    (tmp_path / "param").write_text(sys_text + iterate + response + "FINISH\n")
    st = P.run_param(str(tmp_path / "param"))
    s = st["system"]
    _, w = F.read_field(str(tmp_path / "in.omega"), s)
    want = _oracle_response_sweep(s, w, dict(k_group="1", kvec0=[0.1], dkvec=[0.2], nkstep=1, n_eigval_out=5))
    for j, pt in enumerate(want):
        lines = open(tmp_path / "out" / f"{j}.eval").read().splitlines()
        assert lines[0].startswith("q_vec   =") and abs(float(lines[0].split()[2]) - (0.1 + 0.2 * j)) < 1e-12
        assert lines[1].split()[-1] == "40" and lines[2] == ""
        ev = [float(x.split()[0]) for x in lines[3:]]
        assert [int(x.split()[1]) for x in lines[3:]] == list(range(1, 6))
        np.testing.assert_allclose(ev, pt["eval"], rtol=1e-8)
        for k in (1, 2):
            el = open(tmp_path / "out" / f"{j}.evec.{k}").read().splitlines()
            i = el.index(next(x for x in el if x.startswith("N_star")))
            assert int(el[i + 1]) == 6
            rows = [[float(v) for v in x.split()[:2]] for x in el[i + 2:i + 8]]
            np.testing.assert_allclose([r[0] for r in rows], pt["evec"][:6, k - 1], rtol=1e-11, atol=1e-13)
            assert all(r[1] == -r[0] for r in rows)
        assert not os.path.exists(tmp_path / "out" / f"{j}.evec.3")
    # RESPONSE must follow ITERATE (or SWEEP) directly
    conv = "RHO_TO_OMEGA\ninput_filename\n          'in.omega'\noutput_filename\n          'w2'\n\n"
    for text in (sys_text + response, sys_text + iterate + conv + response):
        (tmp_path / "p2").write_text(text + "FINISH\n")
        with pytest.raises(RuntimeError):
            P.run_param(str(tmp_path / "p2"))


def test_response_after_sweep_uses_the_last_point(tmp_path, monkeypatch):
    """SWEEP leaves iterate_flag set (src/pscf.fp.f90:557-700), so a RESPONSE
    after it runs on the sweep's last system and field."""
    import shutil
    shutil.copy(os.path.join(HERE, "golden", "fieldfile_rho.txt"), tmp_path / "in.omega")
    h = F._read_header(open(tmp_path / "in.omega").read().splitlines())[0]
    sys_text = _TWO_MONOMER.replace("@CELL@", f'{h["cell_param"][0]:20.10E}')
    iterate = ("ITERATE\ninput_filename\n          'in.omega'\noutput_prefix\n              'out/'\nmax_itr\n"
               "                 100\nerror_max\n    1.0000000000E-08\ndomain\n                   F\n"
               "itr_algo\n                'AM'\nN_hist\n                  10\n\n")
    sweep = "SWEEP\ns_max\n    1.0000000000E+00\nd_chi\n    2.0000000000E+00\nend_increments\n\n"
    response = ("RESPONSE\nk_group\n                 '1'\nkdim\n                   1\nkvec\n"
                "    2.0000000000E-01\nnkstep\n                   0\nn_eigval_out\n                   3\n"
                "n_eigvec_out\n                   0\nn_basis_out\n                   0\n\n")
    seen = []

    def fake_solver(it, group):
        def solve(system, w0):
            seen.append(float(system.chi[0, 1]))
            r = dict(converged=True, itr=1, error=1e-9, f_helmholtz=1.0, pressure=2.0, stress=[0.0],
                     mu_chain=[3.0], cell_param=list(system.cell_param))
            return w0 * (1.0 + 0.01 * len(seen)), w0, r
        return solve
    got = {}

    def response_on_oracle(system, omega, rp):
        got.update(chi=float(system.chi[0, 1]), omega=np.array(omega))
        return _oracle_response_sweep(system, omega, rp)
    monkeypatch.setattr(P, "_solver", fake_solver)
    monkeypatch.setattr(P, "_response_sweep", response_on_oracle)
    (tmp_path / "param").write_text(sys_text + iterate + sweep + response + "FINISH\n")
    st = P.run_param(str(tmp_path / "param"))
    assert abs(got["chi"] - 17.0) < 1e-6 and abs(seen[-1] - 17.0) < 1e-6
    np.testing.assert_array_equal(got["omega"], st["sweep"][-1].omega)
    assert (tmp_path / "out" / "0.eval").exists() and not (tmp_path / "out" / "0.evec.1").exists()
    assert (tmp_path / "out" / "1.out").exists()


def test_nr_n_cut_is_passed_through(monkeypatch):
    """ITERATE with itr_algo 'NR' reads N_cut as the reference does (it is
    required there) and hands it to the solver unchanged, 0 included."""
    from pscf_b200 import sweep as S
    seen = {}
    monkeypatch.setattr(S, "nr_solver", lambda group, **kw: seen.update(kw) or (lambda system, w: None))
    for n_cut in (0, 17):
        it = P._iterate_params(dict(input_filename=["in.omega"], output_prefix=["out/"], max_itr=[20.0],
                                    error_max=[1e-8], domain=["T"], itr_algo=["NR"], N_cut=[float(n_cut)]))
        P._solver(it, "-1")
        assert seen["n_cut"] == n_cut and seen["domain"] is True
    with pytest.raises(ValueError):
        P._iterate_params(dict(input_filename=["in.omega"], output_prefix=["out/"], max_itr=[20.0],
                               error_max=[1e-8], domain=["T"], itr_algo=["NR"]))


def test_second_iterate_starts_from_the_current_omega(tmp_path, monkeypatch):
    """omega_flag (src/pscf.fp.f90:479-487): once an ITERATE has run, the
    next one reads no input_filename and starts from the current omega; a
    conversion command in between clears it."""
    import shutil
    shutil.copy(os.path.join(HERE, "golden", "fieldfile_rho.txt"), tmp_path / "in.omega")
    h = F._read_header(open(tmp_path / "in.omega").read().splitlines())[0]
    sys_text = _TWO_MONOMER.replace("@CELL@", f'{h["cell_param"][0]:20.10E}')
    tail = ("output_prefix\n              'out/'\nmax_itr\n                 100\nerror_max\n    1.0000000000E-08\n"
            "domain\n                   F\nitr_algo\n                'AM'\nN_hist\n                  10\n\n")
    first = "ITERATE\ninput_filename\n          'in.omega'\n" + tail
    again = "ITERATE\n" + tail
    starts = []

    def fake_solver(it, group):
        def solve(system, w0):
            starts.append(np.array(w0))
            r = dict(converged=True, itr=1, error=1e-9, f_helmholtz=1.0, pressure=2.0, stress=[0.0],
                     mu_chain=[3.0], cell_param=list(system.cell_param))
            return w0 + 1.0, w0, r
        return solve
    monkeypatch.setattr(P, "_solver", fake_solver)
    (tmp_path / "param").write_text(sys_text + first + again + "FINISH\n")
    P.run_param(str(tmp_path / "param"))
    np.testing.assert_array_equal(starts[1], starts[0] + 1.0)
    from pscf_b200.sweep import read_out
    d = read_out(str(tmp_path / "out" / "out"))
    assert d["input_filename"] == ["in.omega"]
    conv = "FIELD_TO_RGRID\ninput_filename\n          'in.omega'\noutput_filename\n          'x.rg'\n\n"
    (tmp_path / "p2").write_text(sys_text + first + conv + again + "FINISH\n")
    with pytest.raises(ValueError):
        P.run_param(str(tmp_path / "p2"))


def test_divide_energy_uniform_fields():
    """divide_energy (src/scf_mod.fp.f90:588-709) on uniform fields a, b
    of a diblock f_A, N = 1: q is exp(-a s) along the A block, so at the
    junction qf qr / Q = 1 and f_head = -log qf - a f_A = 0, f_tail = 0;
    overlap_AB = f_A f_B; f_excess = f_total + 1 - chi f_A f_B."""
    from oracle import oracle as O
    from pscf_b200.sweep import divide_energy
    from pscf_b200.system import Chain, System, chain_grid
    s = System(dim=1, ngrid=[16], crystal_system="lamellar", cell_param=[1.7], kuhn=[1.0, 1.0],
               chi=[[0.0, 14.0], [14.0, 0.0]], chains=[Chain([0, 1], [0.4, 0.6], phi=1.0)], ds=0.01)
    w = np.stack([np.full(16, 2.0), np.full(16, -0.5)])
    o = O.Oracle(s)
    rho, q = o.density(w)
    qf, qr = o.propagators(0)
    h = chain_grid([0.4, 0.6], 0.01)[0][1]
    fb = F.FieldBasis("-1", s)
    fc, ov = divide_energy(s, np.stack([fb.to_coeffs(x) for x in w]), np.stack([fb.to_coeffs(x) for x in rho]), q,
                           [(qf[h], qr[h], qf[h], qr[h])], 3.0)
    assert abs(fc[1]) < 1e-12 and abs(fc[2]) < 1e-12
    assert abs(ov[0, 1] - 0.4 * 0.6) < 1e-12 and abs(fc[0] - 14.0 * 0.24) < 1e-11
    assert abs(fc[3] - (3.0 + 1.0 - 14.0 * 0.24)) < 1e-11


def test_decompose_section_in_iterate_and_sweep_files(tmp_path, monkeypatch):
    """The summary of the current reference writes DECOMPOSE between THERMO
    and STATISTICS (output_summary, src/pscf.fp.f90:1162-1174): overlap_AB,
    f_enthalpy, f_head, f_tail, f_excess, for the ITERATE file and every
    sweep point."""
    import shutil
    from pscf_b200.sweep import read_out
    shutil.copy(os.path.join(HERE, "golden", "fieldfile_rho.txt"), tmp_path / "in.omega")
    h = F._read_header(open(tmp_path / "in.omega").read().splitlines())[0]
    sys_text = _TWO_MONOMER.replace("@CELL@", f'{h["cell_param"][0]:20.10E}')
    iterate = ("ITERATE\ninput_filename\n          'in.omega'\noutput_prefix\n              'out/'\nmax_itr\n"
               "                 100\nerror_max\n    1.0000000000E-08\ndomain\n                   F\n"
               "itr_algo\n                'AM'\nN_hist\n                  10\n\n")
    sweep = "SWEEP\ns_max\n    1.0000000000E+00\nd_chi\n    2.0000000000E+00\nend_increments\n\n"

    def fake_solver(it, group):
        def solve(system, w0):
            r = dict(converged=True, itr=1, error=1e-9, f_helmholtz=1.25, pressure=2.0, stress=[0.0],
                     mu_chain=[3.0], cell_param=list(system.cell_param))
            return w0, w0, r
        return solve
    monkeypatch.setattr(P, "_solver", fake_solver)
    (tmp_path / "param").write_text(sys_text + iterate + sweep + "FINISH\n")
    st = P.run_param(str(tmp_path / "param"))
    for j in (0, 1):
        lines = open(tmp_path / "out" / f"{j}.out").read().splitlines()
        i = lines.index("DECOMPOSE           ")
        assert lines[i - 1] == "" and lines.index("STATISTICS          ") > i > lines.index("THERMO              ")
        assert [x.strip() for x in lines[i + 1:i + 11:2]] == ["overlap_AB", "f_enthalpy", "f_head", "f_tail", "f_excess"]
        d = read_out(str(tmp_path / "out" / f"{j}.out"))
        pt = st["sweep"][j]
        want = _oracle_decompose(pt.system, "-1", pt.omega, 1.25)
        assert abs(d["overlap_AB"][0] - want["overlap"][0, 1]) < 1e-9 * max(1.0, abs(want["overlap"][0, 1]))
        np.testing.assert_allclose([d[k][0] for k in ("f_enthalpy", "f_head", "f_tail", "f_excess")],
                                   want["f_component"], rtol=1e-9, atol=1e-10)


class _OracleEngine:
    """The engine's interface as _decompose uses it (density with q padded
    to MAX_CHAIN, q_solvent, propagators, close), served by the oracle."""

    def __init__(self, systems, precision):
        from oracle import oracle as O
        self.s = systems[0]
        self.o = O.Oracle(self.s)

    def density(self, omega):
        from pscf_b200.system import MAX_CHAIN, MAX_SOLVENT
        rho, q = self.o.density(np.asarray(omega)[0])
        qq = np.zeros((1, MAX_CHAIN))
        qq[0, :len(q)] = q
        self.q_solvent = np.zeros((1, MAX_SOLVENT))
        for i, v in enumerate(self.s.solvents):
            w = np.asarray(omega)[0, v.monomer]
            self.q_solvent[0, i] = np.mean(np.exp(-v.size * w))      # solvent_density's Q
        return rho[None], qq

    def propagators(self, inst=0, chain=0):
        return self.o.propagators(chain)

    def close(self):
        pass


def test_decompose_through_the_engine_interface(monkeypatch):
    """The product's _decompose (not the stand-in used above), with the
    engine class replaced by the oracle behind the same interface: its
    slice bookkeeping, junction choice and solvent partition functions
    give the stand-in's values, for a triblock with a solvent."""
    import pscf_b200.engine as EN
    from pscf_b200.system import Chain, Solvent, System
    monkeypatch.setattr(EN, "Engine", _OracleEngine)
    s = System(dim=1, ngrid=[16], crystal_system="lamellar", cell_param=[1.7], kuhn=[1.0, 1.1, 0.9],
               chi=np.array([[0, 12.0, 20.0], [12.0, 0, 15.0], [20.0, 15.0, 0]]),
               chains=[Chain([0, 1, 2], [0.3, 0.4, 0.3], phi=0.8)], solvents=[Solvent(1, 0.2, phi=0.2)], ds=0.01)
    w = 1.5 * np.cos(2 * np.pi * np.arange(16) / 16)[None, :] * np.array([[1.0], [-0.5], [0.3]])
    got = _ENGINE_DECOMPOSE(s, "-1", w, 2.5)
    want = _oracle_decompose(s, "-1", w, 2.5)
    np.testing.assert_allclose(got["f_component"], want["f_component"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(got["overlap"], want["overlap"], rtol=1e-12, atol=1e-14)
    assert abs(got["q_solvent"][0] - np.mean(np.exp(-0.2 * w[1]))) < 1e-15
