"""Sweep driver and output summary files (pscf_b200.sweep), on the CPU.

The summary writer is pinned to two of the reference's own output files
(tests/golden/sweep/0.out, lamellar.out, copied by make_outfile_fixture.py):
written from the values they hold, they come back byte for byte.  The
sweep's step schedule, continuation and backtracking (src/pscf.fp.f90:557-700,
src/sweep_mod.f90:407-600) are checked with a stand-in solver."""
import os

import numpy as np
import pytest

from pscf_b200 import sweep as S
from pscf_b200.system import Chain, Solvent, System
from tests.cases import diblock

HERE = os.path.dirname(os.path.abspath(__file__))


def _from_out(path):
    """System, result, iterate and statistics dicts of an output file."""
    d = S.read_out(path)
    M = int(d["N_monomer"][0])
    nch = int(d["N_chain"][0])
    nblk = [int(x) for x in d["N_block"]]
    mon, lens = [int(x) - 1 for x in d["block_monomer"]], d["block_length"]
    chains, k = [], 0
    for j in range(nch):
        chains.append(Chain(mon[k:k + nblk[j]], lens[k:k + nblk[j]], phi=d["phi_chain"][j]))
        k += nblk[j]
    chi = np.zeros((M, M))
    k = 0
    for a in range(1, M):
        for b in range(a):
            chi[a, b] = chi[b, a] = d["chi"][k]
            k += 1
    dim = int(d["dim"][0])
    s = System(dim=dim, ngrid=[int(x) for x in d["ngrid"]], crystal_system=d["crystal_system"][0],
               cell_param=d["cell_param"], kuhn=d["kuhn"], chi=chi, chains=chains, ds=d["chain_step"][0])
    res = dict(f_helmholtz=d["f_Helmholtz"][0], pressure=d["pressure"][0], stress=d["stress"],
               mu_chain=d["mu_chain"])
    it = dict(input_filename=d["input_filename"][0], output_prefix=d["output_prefix"][0],
              max_itr=int(d["max_itr"][0]), error_max=d["error_max"][0], domain=d["domain"][0] == "T",
              itr_algo=d["itr_algo"][0], N_cut=int(d["N_cut"][0]) if "N_cut" in d else 0,
              N_hist=int(d["N_hist"][0]) if "N_hist" in d else 0)
    st = dict(n_star=int(d["N_star"][0]), final_error=d["final_error"][0], iterations=int(d["iterations"][0]),
              basis_time=d["basis_time"][0], scf_time=d["scf_time"][0])
    return s, d["group_name"][0], res, it, st, d


@pytest.mark.parametrize("name", ["sweep/0.out", "lamellar.out"])
def test_output_summary_reproduces_reference_files(tmp_path, name):
    src = os.path.join(HERE, "golden", name)
    s, group, res, it, st, d = _from_out(src)
    assert abs(S.free_energy_fh(s) - d["f_homo"][0]) < 1e-9
    out = tmp_path / "x.out"
    S.write_out(str(out), s, group, res, it, st)
    # (the lamellar file carries one extra empty line at its end)
    assert open(out).read().rstrip("\n") == open(src).read().rstrip("\n")


def test_free_energy_fh_blend():
    chains = [Chain([0, 1], [0.4, 0.6], phi=0.7), Chain([0], [0.5], phi=0.2)]
    s = System(dim=1, ngrid=[8], crystal_system="lamellar", cell_param=[1.0], kuhn=[1.0, 1.0],
               chi=[[0, 14.0], [14.0, 0]], chains=chains, solvents=[Solvent(1, 0.1, phi=0.1)], ds=0.01)
    rA = 0.7 * 0.4 + 0.2
    rB = 0.7 * 0.6 + 0.1
    f = 0.7 * (np.log(0.7) - 1) + 0.2 / 0.5 * (np.log(0.2) - 1) + 0.1 / 0.1 * (np.log(0.1) - 1) + 14.0 * rA * rB
    assert abs(S.free_energy_fh(s) - f) < 1e-13


def test_increment_parameters_by_ensemble_and_domain():
    s = diblock(1, [16], "lamellar", [1.7], fA=0.4, chiN=15.0)
    inc = S.Increments(chi=[[0, 1.0], [1.0, 0]], block_length=[[-0.01, 0.01]], kuhn=[0.0, 0.1],
                       phi_chain=[0.5], mu_chain=[2.0], cell_param=[0.2])
    a = S.increment_parameters(s, inc, 0.5, domain=True)
    assert a.chi[0, 1] == 15.5 and a.chains[0].block_length == [0.395, 0.605] and a.kuhn == [1.0, 1.05]
    assert a.chains[0].phi == 1.25 and a.chains[0].mu == s.chains[0].mu and a.cell_param == [1.7]
    b = S.increment_parameters(s, inc, 0.5, domain=False)
    assert abs(b.cell_param[0] - 1.8) < 1e-15
    s.ensemble = 1
    c = S.increment_parameters(s, inc, 0.5, domain=True)
    assert c.chains[0].mu == s.chains[0].mu + 1.0 and c.chains[0].phi == s.chains[0].phi
    assert s.chains[0].block_length == [0.4, 0.6]                 # the input is not modified


def test_continuation_orders():
    h = S.History()
    f = lambda s: np.array([1.0 + 2.0 * s - 0.5 * s * s, -3.0 * s * s])
    cell = lambda s: [2.0 + 0.25 * s * s]
    h.update(0.0, f(0.0), cell(0.0), True)
    w, c = h.continuation(0.1, True, [9.9])
    np.testing.assert_allclose(w, f(0.0))
    np.testing.assert_allclose(c, cell(0.0))
    h.update(0.1, f(0.1), cell(0.1), True)
    w, _ = h.continuation(0.9, True, [9.9])
    lin = f(0.0) + (f(0.1) - f(0.0)) * 10.0                          # first order through s = 0, 0.1
    np.testing.assert_allclose(w, lin, rtol=1e-12)
    h.update(1.0, f(1.0), cell(1.0), True)
    w, c = h.continuation(1.0, True, [9.9])                          # second order: exact for a quadratic
    np.testing.assert_allclose(w, f(2.0), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(c, cell(2.0), rtol=1e-12)
    _, c = h.continuation(1.0, False, [9.9])
    assert c == [9.9]


def _fake_solver(fail_at=()):
    """Converges to omega = f(parameters) unless the current block length
    is in fail_at; records the starting fields it was given."""
    calls = []

    def solve(system, omega):
        L = system.chains[0].block_length[0]
        target = np.array([[L, L * L], [1.0 - L, 0.5]])
        calls.append((L, np.array(omega)))
        ok = not any(abs(L - x) < 1e-9 for x in fail_at)
        res = dict(converged=ok, itr=3, error=1e-11, f_helmholtz=L, pressure=1.0, stress=[0.0],
                   mu_chain=[0.0], cell_param=list(system.cell_param))
        return target, target * 0.5, res
    return solve, calls


def test_sweep_schedule_outputs_and_backtracking(tmp_path):
    s0 = diblock(1, [16], "lamellar", [1.7], fA=0.40, chiN=15.0)
    inc = S.Increments(block_length=[[-0.01, 0.01]])
    solve, calls = _fake_solver()
    it = dict(max_itr=20, error_max=1e-10, domain=False, itr_algo="AM", N_hist=20)
    pts = S.run_sweep(s0, np.zeros((2, 16)), inc, 3.0, solve, domain=False, out_prefix=str(tmp_path / "out") + "/",
                      iterate=it, n_star=9)
    Ls = [round(c[0], 8) for c in calls]
    assert Ls == [0.40, 0.399, 0.39, 0.38, 0.37]                    # s = 0, 0.1, 1, 2, 3
    # the first steps are the single-precision 0.1 and 0.9 of the reference
    assert abs(calls[2][0] - (0.40 - 0.01 * (float(np.float32(0.1)) + float(np.float32(0.9))))) < 1e-15
    assert [round(p.s, 6) for p in pts] == [0.0, 1.0, 2.0, 3.0]
    for j in range(4):
        d = S.read_out(str(tmp_path / "out" / f"{j}.out"))
        assert abs(d["block_length"][0] - (0.40 - 0.01 * j)) < 3e-10 and d["N_star"] == [9.0]
    # the third point (s = 2) is predicted to second order from s = 0.1, 1 (first order) ...
    # every prediction is exact here: the target is quadratic in s
    s1 = float(np.float32(0.1)) + float(np.float32(0.9))
    L = lambda s: 0.40 - 0.01 * (s - 1.0 + s1)
    tgt = lambda s: np.array([[L(s), L(s) ** 2], [1.0 - L(s), 0.5]])
    np.testing.assert_allclose(calls[4][1], tgt(3.0), atol=1e-12)
    # a failure at s = 2 halves the unit step: s = 1.5, 2, 2.5, 3
    solve, calls = _fake_solver(fail_at=[0.38])
    with pytest.raises(RuntimeError):
        S.run_sweep(s0, np.zeros((2, 16)), inc, 3.0, solve, domain=False)
    solve, calls = _fake_solver(fail_at=[0.385])
    pts = S.run_sweep(s0, np.zeros((2, 16)), inc, 3.0, solve, domain=False)
    assert [round(c[0], 8) for c in calls] == [0.40, 0.399, 0.39, 0.38, 0.37]
    solve, calls = _fake_solver(fail_at=[])
    first = [True]

    def flaky(system, omega):
        w, r, res = solve(system, omega)
        if abs(system.chains[0].block_length[0] - 0.38) < 1e-8 and first[0]:
            first[0] = False
            res = dict(res, converged=False)
        return w, r, res
    pts = S.run_sweep(s0, np.zeros((2, 16)), inc, 3.0, flaky, domain=False)
    assert [round(c[0], 8) for c in calls] == [0.40, 0.399, 0.39, 0.38, 0.385, 0.38, 0.375, 0.37]
    assert [round(p.s, 6) for p in pts] == [0.0, 1.0, 2.0, 3.0]


def test_temperature_interaction_sweep_and_summary(tmp_path):
    """interaction_type 'chi_T' (chi = chi_A / T + chi_B): a temperature
    increment moves chi with it (increment_parameters,
    src/sweep_mod.f90:418-421), and the summary prints chi_A, chi_B and the
    temperature under INTERACTION and the resulting chi under THERMO
    (output_interaction, src/chemistry_mod.f90:1274-1326; output_summary,
    src/pscf.fp.f90:1157-1159)."""
    chi_A = np.array([[0.0, 3000.0], [3000.0, 0.0]])
    chi_B = np.array([[0.0, -2.0], [-2.0, 0.0]])
    s = System(dim=1, ngrid=[16], crystal_system="lamellar", cell_param=[1.7], kuhn=[1.0, 1.0], chi=np.zeros((2, 2)),
               chains=[Chain([0, 1], [0.5, 0.5])], ds=0.01, chi_A=chi_A, chi_B=chi_B, temperature=200.0)
    assert abs(s.chi[0, 1] - (3000.0 / 200.0 - 2.0)) < 1e-14
    t = S.increment_parameters(s, S.Increments(temperature=-10.0), 0.5, domain=True)
    assert t.temperature == 195.0 and abs(t.chi[0, 1] - (3000.0 / 195.0 - 2.0)) < 1e-13
    assert s.temperature == 200.0
    res = dict(f_helmholtz=2.0, pressure=3.0, stress=[1e-12], mu_chain=[4.0])
    it = dict(max_itr=10, error_max=1e-8, domain=True, itr_algo="AM", N_hist=20)
    st = dict(n_star=9, final_error=1e-9, iterations=5)
    S.write_out(str(tmp_path / "t.out"), t, "-1", res, it, st)
    lines = open(tmp_path / "t.out").read().splitlines()
    d = S.read_out(str(tmp_path / "t.out"))
    assert d["interaction_type"] == ["chi_T"] and d["chi_A"] == [3000.0] and d["chi_B"] == [-2.0]
    assert d["temperature"] == [195.0] and abs(d["chi"][0] - t.chi[1, 0]) < 1e-9
    assert lines.index("chi                 ") > lines.index("THERMO              ")


def test_sweep_reproduces_the_reference_sweep_files(tmp_path, monkeypatch):
    """The reference's own sweep (tools/python/tests/sweep/out/0.out ...
    11.out: BCC 20^3, block length 0.39 -> 0.28 in steps of -0.01, cell
    relaxed at every point), replayed with a stand-in solver that returns
    each point's own results: every file comes back line for line but for
    the two timings.  This pins the step schedule (the single-precision
    first steps: 0.38000000022, ...), the parameters written, f_homo and
    the layout against the reference's own output."""
    ref = [_from_out(os.path.join(HERE, "golden", "sweep", f"{j}.out")) for j in range(12)]
    s0, group, _, it, st0, _ = ref[0]
    by_length = {round(r[0].chains[0].block_length[0], 9): r for r in ref}

    def solve(system, omega):
        got = by_length.get(round(system.chains[0].block_length[0], 9))
        if got is None:                        # s = 0.1: not written
            return omega, omega, dict(converged=True, itr=1, error=1e-9, f_helmholtz=0.0, pressure=0.0,
                                      stress=[0.0], mu_chain=[0.0], cell_param=list(system.cell_param))
        s, _, res, _, st, _ = got
        r = dict(res, converged=True, itr=st["iterations"], error=st["final_error"], cell_param=list(s.cell_param))
        return omega, omega, r
    from pscf_b200 import field_io
    monkeypatch.setattr(field_io, "write_field", lambda *a, **k: None)
    pts = S.run_sweep(s0, np.zeros((2, s0.nr)), S.Increments(block_length=[[-0.01, 0.01]]), 11.0, solve,
                      domain=True, out_prefix=str(tmp_path / "out") + "/", group_name=group, iterate=it,
                      n_star=st0["n_star"])
    assert len(pts) == 12
    for j in range(12):
        want = open(os.path.join(HERE, "golden", "sweep", f"{j}.out")).read().splitlines()
        got = open(tmp_path / "out" / f"{j}.out").read().splitlines()
        assert len(got) == len(want)
        skip = {want.index(x) + 1 for x in want if x.strip() in ("basis_time", "scf_time")}
        for k, (a, b) in enumerate(zip(got, want)):
            if k not in skip:
                assert a == b, (j, k, a, b)


def test_grand_canonical_summary_prints_the_solution_phi(tmp_path):
    """Grand ensemble (ensemble = 1): COMPOSITION holds mu_chain, and THERMO
    the chains' phi = Q exp(mu) (mu_phi_chain, src/scf_mod.fp.f90:768-785)
    with f_homo of those phi (output_summary, src/pscf.fp.f90:1130-1150)."""
    chains = [Chain([0, 1], [0.4, 0.6], mu=1.5), Chain([0], [0.5], mu=-0.25)]
    s = System(dim=1, ngrid=[16], crystal_system="lamellar", cell_param=[1.7], kuhn=[1.0, 1.0],
               chi=[[0, 12.0], [12.0, 0]], chains=chains, ds=0.01, ensemble=1)
    q = [0.123, 1.9]
    res = dict(f_helmholtz=2.0, pressure=3.0, stress=[1e-12], mu_chain=[1.5, -0.25], q=q)
    it = dict(max_itr=10, error_max=1e-8, domain=True, itr_algo="AM", N_hist=20)
    S.write_out(str(tmp_path / "g.out"), s, "-1", res, it, dict(n_star=9, final_error=1e-9, iterations=5))
    d = S.read_out(str(tmp_path / "g.out"))
    phi = [q[0] * np.exp(1.5), q[1] * np.exp(-0.25)]
    np.testing.assert_allclose(d["phi_chain"], phi, rtol=1e-10)
    np.testing.assert_allclose(d["mu_chain"], [1.5, -0.25])
    sp = S.grand_phi(s, res)
    assert [c.phi for c in sp.chains] == phi and s.chains[0].phi == 1.0       # the input is not modified
    assert abs(d["f_homo"][0] - S.free_energy_fh(sp)) < 1e-9 * abs(S.free_energy_fh(sp))


def test_canonical_solvent_mu_from_its_partition_function(tmp_path):
    """Canonical ensemble with a solvent: THERMO prints mu_solvent =
    log(phi / Q_solvent) (mu_phi_solvent, src/scf_mod.fp.f90:803-820) when
    the result carries the solvent's Q."""
    s = System(dim=1, ngrid=[16], crystal_system="lamellar", cell_param=[1.7], kuhn=[1.0, 1.0],
               chi=[[0, 12.0], [12.0, 0]], chains=[Chain([0, 1], [0.4, 0.6], phi=0.9)],
               solvents=[Solvent(1, 0.1, phi=0.1)], ds=0.01)
    res = dict(f_helmholtz=2.0, pressure=3.0, stress=[1e-12], mu_chain=[1.5], q_solvent=[0.8])
    it = dict(max_itr=10, error_max=1e-8, domain=True, itr_algo="AM", N_hist=20)
    S.write_out(str(tmp_path / "s.out"), s, "-1", res, it, dict(n_star=9, final_error=1e-9, iterations=5))
    d = S.read_out(str(tmp_path / "s.out"))
    assert abs(d["mu_solvent"][0] - np.log(0.1 / 0.8)) < 1e-10
    assert d["phi_solvent"] == [0.1] and d["solvent_size"] == [0.1]
