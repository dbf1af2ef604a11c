"""The reference's parameter files, read and run on the engine.

A parameter file (doc/user-man/param.rst; read by the main program,
src/pscf.fp.f90:200-720) is a version line and a sequence of sections, each
a name on its own line followed by `label` / value lines in the io_mod
layout -- the same layout as the first part of an output summary:

  MONOMERS, CHAINS, SOLVENTS, COMPOSITION, INTERACTION, UNIT_CELL,
  DISCRETIZATION, BASIS  -- the system;
  RESCALE                -- read an omega file and change the monomer
                            reference volume (the next ITERATE starts
                            from that field);
  ITERATE                -- solve from a basis-format omega file, or,
                            without input_filename, from the current omega
                            (RESCALE's, or the last ITERATE's or SWEEP's);
  SWEEP                  -- continuation to s_max with d_<name> increments,
                            ended by end_increments;
  RESPONSE               -- eigenvalues and eigenvectors of the linear
                            response of the converged state along a line
                            of k points;
  FIELD_TO_RGRID, RGRID_TO_FIELD, KGRID_TO_RGRID, RHO_TO_OMEGA
                         -- field conversions;
  FINISH.

read_param parses a file into its sections; system_of builds the System;
run_param executes the commands in order with the engine (Anderson mixing,
or Newton with the batched Jacobian for itr_algo 'NR'), writing the same
files as the reference: <output_prefix>out / omega / rho for ITERATE,
<output_prefix>0., 1., ... for a SWEEP, <output_prefix>j.eval and
j.evec.k for RESPONSE.  OUTPUT_WAVES and OUTPUT_GROUP are not run here.
"""
from __future__ import annotations

import os
import time
from typing import Dict, List, Tuple

import numpy as np

from .system import Chain, Solvent, System

SYSTEM_SECTIONS = ("MONOMERS", "CHAINS", "SOLVENTS", "COMPOSITION", "INTERACTION", "UNIT_CELL", "DISCRETIZATION",
                   "BASIS")
COMMANDS = ("ITERATE", "SWEEP", "RESPONSE", "FIELD_TO_RGRID", "RGRID_TO_FIELD", "KGRID_TO_RGRID", "RHO_TO_OMEGA",
            "RESCALE", "OUTPUT_WAVES", "OUTPUT_GROUP", "OUTPUT_GROUP_CPP", "WRITE_GROUPS", "FINISH")


def _values(line: str):
    """The values of a data line, or None for a label line."""
    t = line.strip()
    toks = t.split()
    try:
        return [float(x.replace("D", "E").replace("d", "e")) for x in toks]
    except ValueError:
        pass
    if t.startswith("'") or t in ("T", "F"):
        return [t.strip("'")]
    return None


def read_param(path: str) -> List[Tuple[str, Dict[str, List]]]:
    """Sections of a parameter file in file order: (name, {label: values});
    parsing stops at FINISH."""
    return read_param_text(open(path).read(), path)


def read_param_text(text: str, path: str = "<text>") -> List[Tuple[str, Dict[str, List]]]:
    """read_param of the file's text."""
    lines = text.splitlines()
    out: List[Tuple[str, Dict[str, List]]] = []
    cur = None
    key = None
    for raw in lines[1:]:
        t = raw.strip()
        if not t:
            continue
        if t in SYSTEM_SECTIONS or t in COMMANDS:
            cur = (t, {})
            out.append(cur)
            key = None
            if t == "FINISH":
                break
            continue
        if t == "end_increments":
            key = None
            continue
        vals = _values(t)
        if vals is None:
            key = t
            if cur is None:
                raise ValueError(f"{path}: {t!r} before the first section")
            cur[1][key] = []
        elif key is not None:
            cur[1][key] += vals
        else:
            raise ValueError(f"{path}: values {t!r} without a label")
    return out


def _sections(param) -> Dict[str, Dict[str, List]]:
    d: Dict[str, Dict[str, List]] = {}
    for name, body in param:
        if name in SYSTEM_SECTIONS:
            d.setdefault(name, {}).update(body)
    return d


def _lower(vals, M):
    m = np.zeros((M, M))
    k = 0
    for a in range(1, M):
        for b in range(a):
            m[a, b] = m[b, a] = vals[k]
            k += 1
    return m


def system_of(param) -> Tuple[System, str]:
    """(System, group name) of the system sections (monomer indices made
    0-based)."""
    d = _sections(param)
    mon, ch, comp, inter = d["MONOMERS"], d.get("CHAINS", {}), d["COMPOSITION"], d["INTERACTION"]
    cell, disc = d["UNIT_CELL"], d["DISCRETIZATION"]
    M = int(mon["N_monomer"][0])
    ens = int(comp["ensemble"][0])
    chains = []
    nch = int(ch.get("N_chain", [0])[0])
    if nch:
        nblk = [int(x) for x in ch["N_block"]]
        bm = [int(x) - 1 for x in ch["block_monomer"]]
        bl = ch["block_length"]
        k = 0
        for j in range(nch):
            c = Chain(bm[k:k + nblk[j]], bl[k:k + nblk[j]])
            if ens == 0:
                c.phi = comp["phi_chain"][j]
            else:
                c.mu = comp["mu_chain"][j]
            chains.append(c)
            k += nblk[j]
    solvents = []
    sv = d.get("SOLVENTS", {})
    for j in range(int(sv.get("N_solvent", [0])[0])):
        v = Solvent(monomer=int(sv["solvent_monomer"][j]) - 1, size=sv["solvent_size"][j])
        if ens == 0:
            v.phi = comp["phi_solvent"][j]
        else:
            v.mu = comp["mu_solvent"][j]
        solvents.append(v)
    kw = {}
    itype = inter["interaction_type"][0]
    if itype == "chi":
        chi = _lower(inter["chi"], M)
    elif itype == "chi_T":
        kw = dict(chi_A=_lower(inter["chi_A"], M), chi_B=_lower(inter["chi_B"], M),
                  temperature=inter["temperature"][0])
        chi = np.zeros((M, M))
    else:
        raise ValueError(f"interaction_type {itype!r}")
    dim = int(cell["dim"][0])
    s = System(dim=dim, ngrid=[int(x) for x in disc["ngrid"]], crystal_system=cell["crystal_system"][0],
               cell_param=cell["cell_param"], kuhn=mon["kuhn"], chi=chi, chains=chains, ds=disc["chain_step"][0],
               solvents=solvents, ensemble=ens, **kw)
    return s, d.get("BASIS", {}).get("group_name", [""])[0]


def increments_of(body: Dict[str, List], system: System):
    """(s_max, Increments) of a SWEEP section."""
    from .sweep import Increments
    M = system.n_monomer
    inc = Increments()
    for key, vals in body.items():
        if key == "s_max":
            continue
        if not key.startswith("d_"):
            raise ValueError(f"SWEEP: unknown entry {key!r}")
        name = key[2:]
        if name == "chi":
            inc.chi = _lower(vals, M)
        elif name == "block_length":
            rows, k = [], 0
            for c in system.chains:
                n = len(c.block_length)
                rows.append(list(vals[k:k + n]))
                k += n
            inc.block_length = rows
        elif name in ("temperature",):
            inc.temperature = vals[0]
        elif name in ("kuhn", "phi_chain", "mu_chain", "phi_solvent", "mu_solvent", "solvent_size", "cell_param"):
            setattr(inc, name, list(vals))
        else:
            raise ValueError(f"SWEEP: no increments of {name!r}")
    return body["s_max"][0], inc


def rescale_vref(system: System, scale: float) -> System:
    """The same system with the monomer reference volume v -> v / scale
    (rescale_vref, src/chemistry_mod.f90:1344-1361): kuhn / sqrt(scale),
    chi (or chi_A and chi_B) / scale, block lengths and solvent sizes
    x scale.  The caller divides omega by scale."""
    import copy
    s = copy.deepcopy(system)
    s.kuhn = [k / np.sqrt(scale) for k in s.kuhn]
    if s.temperature is not None:
        s.chi_A = s.chi_A / scale
        s.chi_B = s.chi_B / scale
        s.chi = s.chi_A / float(s.temperature) + s.chi_B
    else:
        s.chi = np.asarray(s.chi, dtype=np.float64) / scale
    for c in s.chains:
        c.block_length = [L * scale for L in c.block_length]
    for v in s.solvents:
        v.size = v.size * scale
    return s


def _iterate_params(body):
    # an ITERATE after RESCALE has no input_filename: it starts from the rescaled field
    it = dict(input_filename=body["input_filename"][0] if "input_filename" in body else None,
              output_prefix=body["output_prefix"][0],
              max_itr=int(body["max_itr"][0]), error_max=body["error_max"][0], domain=body["domain"][0] == "T",
              itr_algo=body["itr_algo"][0])
    if it["itr_algo"] == "NR":
        if "N_cut" not in body:
            raise ValueError("ITERATE: itr_algo 'NR' needs N_cut")
        it["N_cut"] = int(body["N_cut"][0])
    elif it["itr_algo"] == "AM":
        it["N_hist"] = int(body.get("N_hist", [20])[0])
    else:
        raise ValueError(f"itr_algo {it['itr_algo']!r}")
    return it


def response_params(body: Dict[str, List], dim: int) -> Dict:
    """The RESPONSE section, read in the order response_startup and
    response_sweep read it (src/response_mod.f90:182, 329-342): k_group,
    kdim, kvec0 (kdim values), nkstep, dkvec (kdim values, present only
    when nkstep > 0), n_eigval_out, n_eigvec_out, n_basis_out.  The labels
    are comments there and are not checked here either."""
    vals = [v for vs in body.values() for v in vs]
    pos = [0]

    def take(n=1):
        if pos[0] + n > len(vals):
            raise ValueError("RESPONSE: section ends early")
        out = vals[pos[0]:pos[0] + n]
        pos[0] += n
        return out
    k_group = str(take()[0])
    if dim == 1 and k_group.strip() == "P 1":
        k_group = "1"
    kdim = int(take()[0])
    if kdim not in (dim, dim + 1):
        raise ValueError(f"RESPONSE: kdim must equal dim or dim+1, got {kdim}")
    kvec0 = [float(x) for x in take(kdim)]
    nkstep = int(take()[0])
    dkvec = [float(x) for x in take(kdim)] if nkstep > 0 else [0.0] * kdim
    n_eigval_out, n_eigvec_out, n_basis_out = (int(x) for x in take(3))
    return dict(k_group=k_group, kdim=kdim, kvec0=kvec0, nkstep=nkstep, dkvec=dkvec, n_eigval_out=n_eigval_out,
                n_eigvec_out=n_eigvec_out, n_basis_out=n_basis_out)


def _fortran_e(v: float, w: int = 20, d: int = 9) -> str:
    """Fortran Ew.d: 0.ddd...E+xx, right-justified in w columns (a
    three-digit exponent drops the E)."""
    v = float(v)
    if v == 0.0:
        body = "0." + "0" * d + "E+00"
    else:
        m, e = f"{abs(v):.{d - 1}E}".split("E")
        e = int(e) + 1
        digits = m.replace(".", "")
        ex = f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else f"{'+' if e >= 0 else '-'}{abs(e):03d}"
        body = ("-" if v < 0 else "") + "0." + digits + ex
    return f"{body:>{w}}"


def write_eval(path: str, kvec: List[float], n_basis: int, evals) -> None:
    """Eigenvalue file of one k point (calc_drho_domega_full,
    src/response_mod.f90:597-605): q_vec (three components), N_basis, an
    empty line, then one 'eval  k' line per eigenvalue (E20.9, I5)."""
    k3 = list(kvec) + [0.0] * (3 - len(kvec))
    out = [f"{'q_vec   =':<20}" + "".join(f"{x:20.10E}" for x in k3[:3]),
           f"{'N_basis =':<20}" + f"{n_basis:20d}", ""]
    out += [_fortran_e(x) + "  " + f"{k:5d}" for k, x in enumerate(evals, 1)]
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def _response_sweep(system: System, omega, rp: Dict):
    """The response at every k point of the sweep, on the engine (fp64):
    the ideal-gas propagation of the converged state and the incompressible
    response (pscf_b200.response)."""
    from .engine import FP64, Engine
    from .response import response_sweep
    e = Engine([system], FP64)
    try:
        e.density(np.asarray(omega, dtype=np.float64).reshape(1, system.n_monomer, system.nr))
        return response_sweep(e, 0, rp["kvec0"], rp["dkvec"], rp["nkstep"], rp["k_group"], rp["n_eigval_out"])
    finally:
        e.close()


def _decompose(system: System, group: str, omega, f_total: float) -> Dict:
    """f_component and overlap of a solution for the DECOMPOSE section
    (sweep.divide_energy), and the solvents' partition functions q_solvent
    (for mu_solvent, or phi in the grand ensemble): one density of omega on
    the engine (fp64), the chains' propagators at their first and last
    junctions, and the reference-convention coefficients of omega and rho."""
    from . import field_io as F
    from .engine import FP64, Engine
    from .sweep import divide_energy, grand_phi
    from .system import chain_grid
    M, nr = system.n_monomer, system.nr
    w = np.asarray(omega, dtype=np.float64).reshape(M, nr)
    e = Engine([system], FP64)
    try:
        rho, q = e.density(w.reshape(1, M, nr))
        q_solvent = [float(x) for x in e.q_solvent[0, :len(system.solvents)]]
        system = grand_phi(system, dict(q=q[0, :len(system.chains)], q_solvent=q_solvent))
        junctions = []
        for c, chain in enumerate(system.chains):
            qf, qr = e.propagators(0, c)
            bgn, _ = chain_grid(chain.block_length, system.ds)
            if qf.shape[0] != bgn[-1] + 1:
                raise RuntimeError(f"chain {c}: {qf.shape[0]} stored slices, {bgn[-1] + 1} expected")
            h, t = bgn[1], bgn[len(chain.block_length) - 1]
            junctions.append((qf[h], qr[h], qf[t], qr[t]))
    finally:
        e.close()
    fb = F.field_basis(group, system)
    omega_c = np.stack([fb.to_coeffs(x) for x in w])
    rho_c = np.stack([fb.to_coeffs(x) for x in rho[0]])
    fc, ov = divide_energy(system, omega_c, rho_c, q[0, :len(system.chains)], junctions, f_total)
    return dict(f_component=fc, overlap=ov, q_solvent=q_solvent)


def _solver(it, group):
    from .sweep import am_solver, nr_solver
    if it["itr_algo"] == "AM":
        return am_solver(group or None, error_max=it["error_max"], max_itr=it["max_itr"], n_hist=it["N_hist"],
                         domain=it["domain"])
    # N_cut = 0: no differenced columns, the Debye response alone
    # (N_corner = 0, iterate_NR_startup, src/iterate_mod.fp.f90:200-225)
    return nr_solver(group, n_cut=it["N_cut"], error_max=it["error_max"], max_itr=it["max_itr"],
                     domain=it["domain"])


def run_param(path: str, workdir: str = None, log=lambda msg: None) -> Dict:
    """Run the commands of a parameter file; file names are relative to
    workdir (default: the file's directory).  Returns the last system, the
    converged fields and results (ITERATE) and the sweep points (SWEEP)."""
    from . import field_io as F
    from .sweep import run_sweep, write_out
    param = read_param(path)
    wd = workdir or os.path.dirname(os.path.abspath(path))
    at = lambda name: name if os.path.isabs(name) else os.path.join(wd, name)
    system, group = system_of(param)
    state: Dict = {"system": system}
    names = [n for n, _ in param]
    for k, (name, body) in enumerate(param):
        if name in SYSTEM_SECTIONS:
            continue
        if name == "FINISH":
            break
        # iterate_flag: set by ITERATE, kept by SWEEP, cleared by every other
        # command; omega_flag (a current omega exists): set by ITERATE and
        # RESCALE, kept by SWEEP and RESPONSE, cleared by the conversions and
        # listings (src/pscf.fp.f90:174-175, 414-1017)
        iterate_flag = state.get("iterate_flag", False)
        if name not in ("ITERATE", "SWEEP"):
            state["iterate_flag"] = False
        if name not in ("ITERATE", "SWEEP", "RESPONSE", "RESCALE"):
            state["omega_flag"] = False
        if name == "RESCALE":
            # src/pscf.fp.f90:414-455: read omega, change v, then omega / scale
            lam = body["vref_scale"][0]
            _, w = F.read_field(at(body["input_filename"][0]), system, group)
            system = rescale_vref(system, lam)
            state.update(omega_cur=w / lam, omega_file=body["input_filename"][0], omega_flag=True)
            continue
        if name == "ITERATE":
            it = _iterate_params(body)
            if it["input_filename"] is None:
                # the reference reads input_filename only while no omega is current
                if not state.get("omega_flag"):
                    raise ValueError("ITERATE without input_filename needs an omega from RESCALE or an ITERATE before it")
                w0 = state["omega_cur"]
                it["input_filename"] = state["omega_file"]
            else:
                _, w0 = F.read_field(at(it["input_filename"]), system, group)
                state["omega_file"] = it["input_filename"]
            t0 = time.perf_counter()
            w, rho, r = _solver(it, group)(system, w0)
            dt = time.perf_counter() - t0
            if it["domain"]:
                system.cell_param = list(r["cell_param"])
            nxt = names[k + 1] if k + 1 < len(names) else ""
            prefix = at(it["output_prefix"]) + ("0." if nxt == "SWEEP" else "")
            d = os.path.dirname(prefix)
            if d:
                os.makedirs(d, exist_ok=True)
            n_star = len(F.field_basis(group, system).stars) if group else 0
            stats = dict(n_star=n_star, final_error=r["error"], iterations=r["itr"], basis_time=0.0, scf_time=dt)
            dec = _decompose(system, group, w, r["f_helmholtz"]) if group and system.chains else {}
            write_out(prefix + "out", system, group, dict(r, **dec), it, stats)
            if group:
                F.write_field(prefix + "omega", w, system, group)
                F.write_field(prefix + "rho", rho, system, group)
            log(f"ITERATE: {'converged' if r['converged'] else 'not converged'} after {r['itr']} iterations")
            state.update(iterate=it, omega=w, rho=rho, result=r, n_star=n_star, iterate_flag=True, omega_cur=w,
                         omega_flag=True)
        elif name == "SWEEP":
            if "result" not in state or not state["result"]["converged"]:
                raise RuntimeError("SWEEP needs a converged ITERATE before it")
            it = state["iterate"]
            s_max, inc = increments_of(body, system)
            pts = run_sweep(system, state["omega"], inc, s_max, _solver(it, group), it["domain"],
                            out_prefix=at(it["output_prefix"]), group_name=group or None, iterate=it,
                            n_star=state["n_star"], log=log,
                            start=(state["omega"], state["rho"], state["result"]),
                            decompose=(lambda s_, w_, r_: _decompose(s_, group, w_, r_["f_helmholtz"]))
                            if group and system.chains else None)
            state["sweep"] = pts
            system = pts[-1].system
            state["omega"] = state["omega_cur"] = pts[-1].omega
        elif name == "RESPONSE":
            # src/pscf.fp.f90:707-723 and response_sweep, src/response_mod.f90:309-389
            if not iterate_flag:
                raise RuntimeError("RESPONSE needs an ITERATE before it")
            rp = response_params(body, system.dim)
            pts = _response_sweep(system, state["omega"], rp)
            prefix = at(state["iterate"]["output_prefix"])
            d = os.path.dirname(prefix)
            if d:
                os.makedirs(d, exist_ok=True)
            for j, pt in enumerate(pts):
                write_eval(f"{prefix}{j}.eval", pt["kvec"], pt["n_basis"], pt["eval"])
                nb = min(rp["n_basis_out"], pt["n_basis"])
                for k in range(min(rp["n_eigvec_out"], len(pt["eval"]))):
                    v = pt["evec"][:nb, k]
                    F.write_coeffs(f"{prefix}{j}.evec.{k + 1}", np.stack([v, -v]), system, rp["k_group"])
            log(f"RESPONSE: {len(pts)} k points")
            state["response"] = pts
        elif name in ("FIELD_TO_RGRID", "RGRID_TO_FIELD", "KGRID_TO_RGRID", "RHO_TO_OMEGA"):
            src, dst = at(body["input_filename"][0]), at(body["output_filename"][0])
            if name == "KGRID_TO_RGRID":
                # wave grid -> basis coefficients -> coordinate grid (src/pscf.fp.f90:813-888)
                _, spec = F.read_kgrid(src, system)
                fb = F.field_basis(group, system)
                F.write_rgrid(dst, np.stack([fb.to_grid(fb.spectrum_to_coeffs(z)) for z in spec]), system, group)
            elif name == "FIELD_TO_RGRID":
                _, f = F.read_field(src, system, group)
                F.write_rgrid(dst, f, system, group)
            elif name == "RGRID_TO_FIELD":
                _, _, f = F.read_rgrid(src)
                b = F.star_basis(group, system.ngrid)
                f = np.stack([b.to_grid(b.to_basis(x)) for x in f])      # onto the group's fields
                F.write_field(dst, f, system, group)
            else:
                # omega_a = sum_b chi_ab rho_b: the pressure field set to zero
                _, rho = F.read_field(src, system, group)
                F.write_field(dst, system.chi @ rho, system, group)
        else:
            raise NotImplementedError(f"parameter-file command {name} is not run by this driver")
    state["system"] = system
    return state
