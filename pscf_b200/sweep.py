"""Parameter sweeps with continuation, and the output summary file.

The reference's SWEEP command (src/pscf.fp.f90:557-700) solves a sequence of
systems along a line in parameter space: a continuation variable s runs from
0 to s_max, every parameter with a nonzero increment changes by step x its
increment (increment_parameters, src/sweep_mod.f90:407-454), and the next
omega (and, when the cell relaxes, the cell) is predicted from up to three
previous solutions by polynomial extrapolation in s (update_history /
continuation, :467-600).  The first step is 0.1, the second the rest of the
way to s = 1, then whole steps; a point that does not converge is undone
and the unit step halved, down to 1/16.  At integer s the output summary
(output_summary, src/pscf.fp.f90:1056-1188) and the fields are written.

Each point is solved by a caller-supplied solve(system, omega) -- the
engine's Anderson mixing (am_solver) or Newton iteration (nr_solver) --
on the grid fields; continuation is linear, so extrapolating grid fields is
the same as extrapolating the reference's star coefficients.
"""
from __future__ import annotations

import copy
import dataclasses
import os
import time
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from .system import System


@dataclasses.dataclass
class Increments:
    """Increments per unit s (input_increments, src/sweep_mod.f90:120-300);
    None leaves a parameter fixed.  block_length is per chain, chi the full
    symmetric matrix."""
    kuhn: Optional[Sequence[float]] = None
    chi: Optional[np.ndarray] = None
    temperature: Optional[float] = None     # interaction_type 'chi_T': d(temperature)
    block_length: Optional[Sequence[Sequence[float]]] = None
    phi_chain: Optional[Sequence[float]] = None
    mu_chain: Optional[Sequence[float]] = None
    phi_solvent: Optional[Sequence[float]] = None
    mu_solvent: Optional[Sequence[float]] = None
    solvent_size: Optional[Sequence[float]] = None
    cell_param: Optional[Sequence[float]] = None


def increment_parameters(system: System, inc: Increments, step: float, domain: bool) -> System:
    """A copy of `system` with every swept parameter moved by step x its
    increment (src/sweep_mod.f90:407-454): phi in the canonical ensemble, mu
    in the grand one; the cell only when it is not relaxed."""
    s = copy.deepcopy(system)
    if inc.kuhn is not None:
        s.kuhn = [k + step * d for k, d in zip(s.kuhn, inc.kuhn)]
    if s.temperature is not None:
        # chi_T: the temperature moves and chi follows (chi_A / T + chi_B)
        if inc.temperature is not None:
            s.temperature = s.temperature + step * inc.temperature
        s.chi = s.chi_A / s.temperature + s.chi_B
    elif inc.chi is not None:
        s.chi = s.chi + step * np.asarray(inc.chi, dtype=np.float64)
    for j, c in enumerate(s.chains):
        if inc.block_length is not None:
            c.block_length = [L + step * d for L, d in zip(c.block_length, inc.block_length[j])]
        if s.ensemble == 0 and inc.phi_chain is not None:
            c.phi += step * inc.phi_chain[j]
        if s.ensemble == 1 and inc.mu_chain is not None:
            c.mu += step * inc.mu_chain[j]
    for j, v in enumerate(s.solvents):
        if s.ensemble == 0 and inc.phi_solvent is not None:
            v.phi += step * inc.phi_solvent[j]
        if s.ensemble == 1 and inc.mu_solvent is not None:
            v.mu += step * inc.mu_solvent[j]
        if inc.solvent_size is not None:
            v.size += step * inc.solvent_size[j]
    if not domain and inc.cell_param is not None:
        s.cell_param = [c + step * d for c, d in zip(s.cell_param, inc.cell_param)]
    return s


class History:
    """Stack of the last N_HIST = 3 solutions (s, omega, cell) and the
    zeroth-, first- or second-order prediction from it
    (src/sweep_mod.f90:467-600)."""
    N_HIST = 3

    def __init__(self):
        self.s: List[float] = []
        self.omega: List[np.ndarray] = []
        self.cell: List[List[float]] = []

    def update(self, s: float, omega: np.ndarray, cell_param: Sequence[float], domain: bool) -> None:
        self.s.insert(0, float(s))
        self.omega.insert(0, np.array(omega, dtype=np.float64))
        self.cell.insert(0, list(cell_param))
        del self.s[self.N_HIST:], self.omega[self.N_HIST:], self.cell[self.N_HIST:]

    def continuation(self, step: float, domain: bool, cell_param: Sequence[float]):
        """(omega, cell_param) predicted for s = s_1 + step."""
        d = len(self.s)
        if d > 2:
            ds2 = self.s[1] - self.s[0]
            ds3 = self.s[2] - self.s[0]
            A2 = step * (ds3 / ds2) / (ds3 - ds2)
            A3 = step * (ds2 / ds3) / (ds2 - ds3)
            B2 = step ** 2 / (ds2 * (ds2 - ds3))
            B3 = step ** 2 / (ds3 * (ds3 - ds2))
            C = [0.0, A2 + B2, A3 + B3]
            C[0] = 1.0 - C[1] - C[2]
        elif d == 2:
            C2 = step / (self.s[1] - self.s[0])
            C = [1.0 - C2, C2]
        elif d == 1:
            C = [1.0]
        else:
            raise RuntimeError("continuation with an empty history")
        omega = sum(c * w for c, w in zip(C, self.omega))
        cell = list(cell_param)
        if domain:
            cell = [sum(c * cl[b] for c, cl in zip(C, self.cell)) for b in range(len(cell))]
        return omega, cell


def free_energy_fh(system: System) -> float:
    """Flory-Huggins free energy per monomer of the homogeneous mixture
    (free_energy_FH, src/scf_mod.fp.f90:903-941)."""
    f = 0.0
    rho = np.zeros(system.n_monomer)
    for c in system.chains:
        if c.phi > 1.0e-8:
            f += (c.phi / c.length) * (np.log(c.phi) - 1.0)
        for m, L in zip(c.block_monomer, c.block_length):
            rho[m] += c.phi * L / c.length
    for v in system.solvents:
        if v.phi > 1.0e-8:
            f += (v.phi / v.size) * (np.log(v.phi) - 1.0)
        rho[v.monomer] += v.phi
    M = system.n_monomer
    for i in range(M - 1):
        for j in range(i + 1, M):
            f += system.chi[i, j] * rho[i] * rho[j]
    return float(f)


# --- output summary (io_mod conventions: label padded to 20 characters on
# its own line, then the data: I20, ES20.10, L20, or a quoted string
# right-justified in 20) ---------------------------------------------------

def _lab(name: str) -> str:
    return f"{name:<20}"


def _int(v) -> str:
    return f"{int(v):20d}"


def _real(v) -> str:
    return f"{float(v):20.10E}"


def _str(v: str) -> str:
    return f"{chr(39) + v + chr(39):>20}"


def grand_phi(system: System, result: Dict) -> System:
    """The system with the volume fractions of a grand-canonical solution,
    phi = Q exp(mu) for chains (mu_phi_chain, src/scf_mod.fp.f90:768-785)
    and solvents (solvent_density, :251-295), from the result's q and
    q_solvent; a canonical system is returned as it is."""
    if system.ensemble != 1:
        return system
    s = copy.deepcopy(system)
    for c, q in zip(s.chains, result.get("q", [])):
        c.phi = float(q) * float(np.exp(c.mu))
    for v, q in zip(s.solvents, result.get("q_solvent", [])):
        v.phi = float(q) * float(np.exp(v.mu))
    return s


def divide_energy(system: System, omega_c: np.ndarray, rho_c: np.ndarray, Q: Sequence[float], junctions,
                  f_total: float):
    """Components of the free energy per monomer and the overlap integrals
    of a solution (divide_energy, src/scf_mod.fp.f90:588-709):

      overlap(a, b) = sum over stars rho_a rho_b,
      f_enthalpy    = sum_{a<b} chi_ab overlap(a, b),
      f_head        = -<qf qr log qf / Q> phi / N at the chain's first
                      junction (block_bgn(2)) - (omega . rho of its first
                      block's monomer) phi,
      f_tail        = the same with log qr at its last junction
                      (block_bgn(N_block)) and the last block's monomer,
      f_excess      = f_Helmholtz + sum phi / N - the three above,

    summed over chains, the averages over the grid points where qf and qr
    are both positive.  omega_c, rho_c: basis coefficients [M][n_star] in
    the reference's convention; Q: the chains' partition functions;
    junctions: per chain (qf, qr at the first junction, qf, qr at the last)
    as grid arrays.  Returns (f_component [4], overlap [M][M])."""
    M = system.n_monomer
    ov = np.zeros((M, M))
    enthalpy = 0.0
    for a in range(M):
        for b in range(a + 1, M):
            ov[a, b] = ov[b, a] = float(np.dot(rho_c[a], rho_c[b]))
            enthalpy += float(system.chi[a, b]) * ov[a, b]
    fhead = ftail = 0.0
    nr = None
    for c, q, (qfh, qrh, qft, qrt) in zip(system.chains, Q, junctions):
        w = c.phi / sum(c.block_length)
        nr = len(qfh)
        m = (qfh > 0.0) & (qrh > 0.0)
        fhead -= float(np.sum(qfh[m] * qrh[m] / q * np.log(qfh[m]))) * w
        m = (qft > 0.0) & (qrt > 0.0)
        ftail -= float(np.sum(qft[m] * qrt[m] / q * np.log(qrt[m]))) * w
    if nr:
        fhead /= nr
        ftail /= nr
    for c in system.chains:
        b0, b1 = c.block_monomer[0], c.block_monomer[-1]
        fhead -= float(np.dot(omega_c[b0], rho_c[b0])) * c.phi
        ftail -= float(np.dot(omega_c[b1], rho_c[b1])) * c.phi
    fjct = f_total + sum(c.phi / sum(c.block_length) for c in system.chains) - enthalpy - fhead - ftail
    return np.array([enthalpy, fhead, ftail, fjct]), ov


def write_out(path: str, system: System, group_name: str, result: Dict, iterate: Dict, stats: Dict) -> None:
    """The reference's output summary file: the input-file sections of the
    system, FINISH, then THERMO, DECOMPOSE (when the result carries
    f_component and overlap, from divide_energy) and STATISTICS.  result:
    f_helmholtz, pressure, stress, mu_chain and, when present, mu_solvent
    (canonical; without it, log(phi / q_solvent) when the result carries
    the solvents' q_solvent); the grand ensemble prints phi = Q exp(mu)
    from the result's q (and q_solvent), and f_homo of those phi;
    iterate: input_filename, output_prefix, max_itr, error_max, domain,
    itr_algo and N_cut or N_hist; stats: n_star, final_error, iterations,
    basis_time, scf_time."""
    s = system
    L: List[str] = [" format  1  0", "", _lab("MONOMERS"), _lab("N_monomer"), _int(s.n_monomer),
                    _lab("kuhn"), "".join(_real(k) for k in s.kuhn)]
    L += ["", _lab("CHAINS"), _lab("N_chain"), _int(len(s.chains))]
    if s.chains:
        L += [_lab("N_block")] + [_int(len(c.block_length)) for c in s.chains]
        L += [_lab("block_monomer")] + ["".join(_int(m + 1) for m in c.block_monomer) for c in s.chains]
        L += [_lab("block_length")] + ["".join(_real(b) for b in c.block_length) for c in s.chains]
    if s.solvents:
        L += ["", _lab("SOLVENTS"), _lab("N_solvent"), _int(len(s.solvents)),
              _lab("solvent_monomer"), "".join(_int(v.monomer + 1) for v in s.solvents),
              _lab("solvent_size"), "".join(_real(v.size) for v in s.solvents)]
    L += ["", _lab("COMPOSITION"), _lab("ensemble"), _int(s.ensemble)]
    if s.ensemble == 0:
        if s.chains:
            L += [_lab("phi_chain")] + [_real(c.phi) for c in s.chains]
        if s.solvents:
            L += [_lab("phi_solvent")] + [_real(v.phi) for v in s.solvents]
    else:
        if s.chains:
            L += [_lab("mu_chain")] + [_real(c.mu) for c in s.chains]
        if s.solvents:
            L += [_lab("mu_solvent")] + [_real(v.mu) for v in s.solvents]
    lower = lambda m: ["".join(_real(m[k, j]) for j in range(k)) for k in range(1, s.n_monomer)]
    if s.temperature is None:
        L += ["", _lab("INTERACTION"), _lab("interaction_type"), _str("chi"), _lab("chi")] + lower(s.chi)
    else:
        L += ["", _lab("INTERACTION"), _lab("interaction_type"), _str("chi_T"), _lab("chi_A")] + lower(s.chi_A)
        L += [_lab("chi_B")] + lower(s.chi_B) + [_lab("temperature"), _real(s.temperature)]
    L += ["", _lab("UNIT_CELL"), _lab("dim"), _int(s.dim), _lab("crystal_system"), _str(s.crystal_system),
          _lab("N_cell_param"), _int(len(s.cell_param)), _lab("cell_param"),
          "".join(_real(c) for c in s.cell_param)]
    L += ["", _lab("DISCRETIZATION"), _lab("ngrid"), "".join(_int(n) for n in s.ngrid),
          _lab("chain_step"), _real(s.ds)]
    L += ["", _lab("BASIS"), _lab("group_name"), _str(group_name)]
    it = iterate
    L += ["", _lab("ITERATE"), _lab("input_filename"), _str(it.get("input_filename", "in.omega")),
          _lab("output_prefix"), _str(it.get("output_prefix", "out/")), _lab("max_itr"), _int(it["max_itr"]),
          _lab("error_max"), _real(it["error_max"]), _lab("domain"), f"{'T' if it['domain'] else 'F':>20}",
          _lab("itr_algo"), _str(it["itr_algo"])]
    if it["itr_algo"] == "NR":
        L += [_lab("N_cut"), _int(it["N_cut"])]
    elif it["itr_algo"] == "AM":
        L += [_lab("N_hist"), _int(it["N_hist"])]
    L += ["", _lab("FINISH")]
    r = result
    sp = grand_phi(s, r)                                # phi of the solution in the grand ensemble
    L += ["", _lab("THERMO"), _lab("f_Helmholtz"), _real(r["f_helmholtz"]), _lab("f_homo"),
          _real(free_energy_fh(sp)), _lab("pressure"), _real(r["pressure"])]
    if s.ensemble == 0:
        if s.chains:
            L += [_lab("mu_chain")] + [_real(m) for m in r["mu_chain"][:len(s.chains)]]
        mus = r.get("mu_solvent")
        if mus is None and "q_solvent" in r:
            # mu = log(phi / Q) (mu_phi_solvent, src/scf_mod.fp.f90:803-820)
            mus = [float(np.log(v.phi / q)) for v, q in zip(s.solvents, r["q_solvent"])]
        if s.solvents and mus is not None:
            L += [_lab("mu_solvent")] + [_real(m) for m in mus[:len(s.solvents)]]
    else:
        if s.chains:
            L += [_lab("phi_chain")] + [_real(c.phi) for c in sp.chains]
        if s.solvents:
            L += [_lab("phi_solvent")] + [_real(v.phi) for v in sp.solvents]
    L += [_lab("stress"), "".join(_real(x) for x in r["stress"][:len(s.cell_param)])]
    if s.temperature is not None:                       # chi printed when it follows T
        L += [_lab("chi")] + lower(s.chi)
    if "f_component" in r and "overlap" in r:
        # DECOMPOSE (output_summary, src/pscf.fp.f90:1162-1174)
        ov, fc = r["overlap"], r["f_component"]
        L += ["", _lab("DECOMPOSE"), _lab("overlap_AB"), _real(ov[0][1])]
        if s.n_monomer == 3:
            L += [_lab("overlap_BC"), _real(ov[1][2]), _lab("overlap_CA"), _real(ov[2][0])]
        L += [_lab("f_enthalpy"), _real(fc[0]), _lab("f_head"), _real(fc[1]), _lab("f_tail"), _real(fc[2]),
              _lab("f_excess"), _real(fc[3])]
    st = stats
    L += ["", _lab("STATISTICS"), _lab("N_star"), _int(st["n_star"]), _lab("final_error"),
          _real(st["final_error"]), _lab("iterations"), _int(st["iterations"]), _lab("basis_time"),
          _real(st.get("basis_time", 0.0)), _lab("scf_time"), _real(st.get("scf_time", 0.0))]
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")


SECTIONS = ("MONOMERS", "CHAINS", "SOLVENTS", "COMPOSITION", "INTERACTION", "UNIT_CELL", "DISCRETIZATION",
            "BASIS", "ITERATE", "FINISH", "THERMO", "DECOMPOSE", "STATISTICS")


def read_out(path: str) -> Dict[str, List]:
    """Labels of an output summary file with their values (numbers as
    floats, quoted strings and T/F as strings), in file order; section
    names map to []."""
    out: Dict[str, List] = {}
    key = None
    for line in open(path).read().splitlines()[1:]:
        t = line.strip()
        if not t:
            continue
        if t in SECTIONS:
            out[t] = []
            key = None
            continue
        toks = t.split()
        try:
            vals = [float(x.replace("D", "E")) for x in toks]
        except ValueError:
            if key is not None and (t.startswith("'") or t in ("T", "F")):
                vals = [t.strip("'")]
            else:
                key = t
                out[key] = []
                continue
        if key is not None:
            out[key] += vals
    return out


# --- solvers ---------------------------------------------------------------

def am_solver(group: Optional[str] = None, **am_kwargs) -> Callable:
    """solve(system, omega) by the engine's Anderson mixing (one engine per
    point: the contour discretisation follows the block lengths)."""
    from .engine import Engine, FP64

    def solve(system: System, omega: np.ndarray):
        e = Engine([copy.deepcopy(system)], FP64)
        try:
            if group:
                e.set_symmetry(0, group)
            w, rho, res = e.iterate_am(np.asarray(omega)[None], **am_kwargs)
        finally:
            e.close()
        return w[0], rho[0], res[0]
    return solve


def nr_solver(group: str, n_cut: Optional[int] = None, max_batch: int = 64, **nr_kwargs) -> Callable:
    """solve(system, omega) by Newton iteration with the batched
    finite-difference Jacobian (pscf_b200.newton)."""
    from .basis import StarBasis
    from .newton import EngineProvider, iterate_nr

    def solve(system: System, omega: np.ndarray):
        basis = StarBasis(group, system.ngrid, system.unit_cell()[0])
        prov = EngineProvider(system, group, max_batch=max_batch)
        try:
            return iterate_nr(prov, basis, system, np.asarray(omega), n_cut=n_cut, **nr_kwargs)
        finally:
            prov.engine.close()
    return solve


@dataclasses.dataclass
class SweepPoint:
    s: float
    system: System
    omega: np.ndarray
    rho: np.ndarray
    result: Dict
    seconds: float


def run_sweep(system: System, omega: np.ndarray, inc: Increments, s_max: float, solve: Callable,
              domain: bool, out_prefix: Optional[str] = None, group_name: Optional[str] = None,
              iterate: Optional[Dict] = None, n_star: int = 0, min_step: float = 1.0 / 16.0,
              log: Callable[[str], None] = lambda msg: None, start=None,
              decompose: Optional[Callable] = None) -> List[SweepPoint]:
    """ITERATE at s = 0, then SWEEP to s_max (src/pscf.fp.f90:557-700).
    Returns the converged points at integer s (s = 0 first); with
    out_prefix, writes <prefix><j>.out (and <prefix><j>.omega / .rho in the
    basis format when group_name is given) for each of them.  start:
    (omega, rho, result) of an already converged s = 0 point, which is then
    neither solved again nor written.  Raises RuntimeError when a point
    fails at the smallest unit step or at s = 0.  decompose(system, omega,
    result) -> dict(f_component, overlap), when given, adds the DECOMPOSE
    section to every file written."""
    def emit(j, pt):
        if not out_prefix:
            return
        d = os.path.dirname(out_prefix)
        if d:
            os.makedirs(d, exist_ok=True)
        r = pt.result
        if decompose is not None:
            r = dict(r, **decompose(pt.system, pt.omega, r))
        stats = dict(n_star=n_star, final_error=r["error"], iterations=r["itr"], basis_time=0.0,
                     scf_time=pt.seconds)
        write_out(f"{out_prefix}{j}.out", pt.system, group_name or "", r, iterate or {}, stats)
        if group_name:
            from .field_io import write_field
            write_field(f"{out_prefix}{j}.omega", pt.omega, pt.system, group_name)
            write_field(f"{out_prefix}{j}.rho", pt.rho, pt.system, group_name)

    # the first two steps are 0.1 and 0.9 of the unit step as the reference
    # writes them, default-real (single precision) literals
    f01, f09 = float(np.float32(0.1)), float(np.float32(0.9))
    t0 = time.perf_counter()
    w, rho, r = solve(system, omega) if start is None else start
    if not r["converged"]:
        raise RuntimeError("the first point (s = 0) did not converge")
    sys0 = copy.deepcopy(system)
    if domain:
        sys0.cell_param = list(r["cell_param"])
    points = [SweepPoint(0.0, sys0, w, rho, r, time.perf_counter() - t0)]
    if start is None:
        emit(0, points[0])
    hist = History()
    hist.update(0.0, w, sys0.cell_param, domain)
    cur = sys0
    s = 0.0
    i = 0
    step_unit = 1.0
    converged = True
    while True:
        if i == 0:
            step = f01 * step_unit
        elif i == 1:
            step = f09 * step_unit if converged else step_unit - s
        else:
            step = step_unit
        s += step
        nxt = increment_parameters(cur, inc, step, domain)
        w0, cell = hist.continuation(step, domain, nxt.cell_param)
        nxt.cell_param = cell
        t0 = time.perf_counter()
        w, rho, r = solve(nxt, w0)
        dt = time.perf_counter() - t0
        converged = bool(r["converged"])
        log(f"s = {s:.4f}: {'converged' if converged else 'not converged'} after {r['itr']} iterations")
        if converged:
            i += 1
            if domain:
                nxt.cell_param = list(r["cell_param"])
            cur = nxt
            hist.update(s, w, cur.cell_param, domain)
            if abs(s - round(s)) < 0.001:
                pt = SweepPoint(s, copy.deepcopy(cur), w, rho, r, dt)
                points.append(pt)
                emit(int(round(s)), pt)
        elif step_unit > min_step + 0.001:
            s -= step                     # back to the last solution, half the unit step
            step_unit *= 0.5
            continue
        else:
            raise RuntimeError(f"sweep failed to converge at s = {s:.4f} with the smallest step")
        if s + 0.001 >= s_max:
            break
    return points
