"""ctypes binding of the C ABI in include/pscf_gpu.h (libpscfgpu.so).

Method names follow the reference routines the ABI replaces:
``density`` (src/scf_mod.fp.f90:144-229), ``scf_stress`` (:451-550),
``free_energy`` (:834-886), ``iterate_am`` (src/iterate_mod.fp.f90:1042-1490),
``propagate`` (step_exp, src/step_mod.f90:146-176).

The library is the only compute path: if it cannot be loaded this module
raises, there is no CPU fallback.
"""
from __future__ import annotations

import copy
import ctypes as C
import os
from typing import List, Sequence

import numpy as np

from .system import (MAX_BLOCK, MAX_CELL_PARAM, MAX_CHAIN, MAX_MONOMER,
                     MAX_SOLVENT, System)

_HERE = os.path.dirname(os.path.abspath(__file__))
# PSCFG_LIB points the binding at another build of the same library (for
# example one compiled with different flags); default: the in-tree build.
LIB_PATH = os.environ.get("PSCFG_LIB") or os.path.join(_HERE, "_lib", "libpscfgpu.so")

FP64 = 0
FP32 = 1
MIXED = 2
CHECKPOINT = 0x100   # OR into the precision: sqrt(Ns) propagator checkpoints (PSCFG_CHECKPOINT)

OK, EINVAL, ECUDA, ENOMEM, ESTATE, ENOTCONV = 0, 1, 2, 3, 4, 5


class PscfgSystem(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("n", C.c_int * 3),
        ("n_monomer", C.c_int),
        ("n_chain", C.c_int),
        ("n_solvent", C.c_int),
        ("ensemble", C.c_int),
        ("n_block", C.c_int * MAX_CHAIN),
        ("block_monomer", (C.c_int * MAX_BLOCK) * MAX_CHAIN),
        ("block_length", (C.c_double * MAX_BLOCK) * MAX_CHAIN),
        ("kuhn", C.c_double * MAX_MONOMER),
        ("chi", (C.c_double * MAX_MONOMER) * MAX_MONOMER),
        ("phi_chain", C.c_double * MAX_CHAIN),
        ("mu_chain", C.c_double * MAX_CHAIN),
        ("solvent_monomer", C.c_int * MAX_SOLVENT),
        ("solvent_size", C.c_double * MAX_SOLVENT),
        ("phi_solvent", C.c_double * MAX_SOLVENT),
        ("mu_solvent", C.c_double * MAX_SOLVENT),
        ("chain_step", C.c_double),
        ("crystal_system", C.c_int),
        ("cell_param", C.c_double * MAX_CELL_PARAM),
    ]


class PscfgAmParam(C.Structure):
    _fields_ = [
        ("max_itr", C.c_int),
        ("n_hist", C.c_int),
        ("domain", C.c_int),
        ("error_max", C.c_double),
        ("switch_error", C.c_double),
        ("mix_max", C.c_double),
        ("restart", C.c_double),
        ("graph_check", C.c_int),
    ]


# pscfg_am_result.status (PSCFG_AM_*)
AM_STATUS = {0: "converged", 1: "running", 2: "nonfinite", 3: "diverged", 4: "maxiter", 5: "singular"}


class PscfgAmResult(C.Structure):
    _fields_ = [
        ("itr", C.c_int),
        ("itr_fp32", C.c_int),
        ("converged", C.c_int),
        ("status", C.c_int),
        ("error", C.c_double),
        ("f_helmholtz", C.c_double),
        ("pressure", C.c_double),
        ("stress", C.c_double * MAX_CELL_PARAM),
        ("cell_param", C.c_double * MAX_CELL_PARAM),
        ("q", C.c_double * MAX_CHAIN),
        ("mu_chain", C.c_double * MAX_CHAIN),
    ]


# Every symbol the header declares, with its ctypes signature.
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
SIGNATURES = {
    "pscfg_create": (C.c_int, [C.POINTER(PscfgSystem), C.c_int, C.c_int, C.POINTER(_vp)]),
    "pscfg_destroy": (None, [_vp]),
    "pscfg_last_error": (C.c_char_p, [_vp]),
    "pscfg_set_cell_param": (C.c_int, [_vp, C.c_int, _dp]),
    "pscfg_get_ksq": (C.c_int, [_vp, C.c_int, _dp]),
    "pscfg_density": (C.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "pscfg_density_device": (C.c_int, [_vp, _vp, _vp, _dp, _dp]),
    "pscfg_stress": (C.c_int, [_vp, _dp]),
    "pscfg_free_energy": (C.c_int, [_vp, _dp, _dp]),
    "pscfg_iterate_am": (C.c_int, [_vp, _dp, C.POINTER(PscfgAmParam), _dp, C.POINTER(PscfgAmResult)]),
    "pscfg_propagate": (C.c_int, [_vp, C.c_int, _dp, C.c_double, C.c_double, _dp, _dp, C.c_int]),
    "pscfg_get_propagators": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp, C.POINTER(C.c_int)]),
    "pscfg_am_begin": (C.c_int, [_vp, _dp, C.POINTER(PscfgAmParam)]),
    "pscfg_am_iterate": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int)]),
    "pscfg_am_results": (C.c_int, [_vp, _dp, _dp, C.POINTER(PscfgAmResult)]),
    "pscfg_set_symmetry": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "pscfg_set_basis": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]),
    "pscfg_density_basis": (C.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "pscfg_stream": (C.c_void_p, [_vp]),
    "pscfg_set_profiling": (C.c_int, [_vp, C.c_int]),
    "pscfg_get_profile": (C.c_int, [_vp, _dp]),
    "pscfg_propagate_noalloc": (C.c_int, [C.c_int, C.POINTER(C.c_int), _vp, _vp, C.c_double, C.c_double,
                                          _vp, _vp, C.c_int, _vp]),
    "pscfg_density_adjoint": (C.c_int, [_vp, _dp, _dp, _dp]),
    "pscfg_density_adjoint_cell": (C.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "pscfg_response": (C.c_int, [_vp, C.c_int, _dp, C.c_double, C.c_int, C.POINTER(C.c_int), _dp, C.c_int,
                                 C.POINTER(C.c_int), _dp, _dp]),
    "pscfg_density_adjoint_device": (C.c_int, [_vp, _vp, _dp, _vp]),
    "pscfg_steps_per_density": (C.c_long, [_vp]),
    "pscfg_launch_count": (C.c_long, [_vp]),
    "pscfg_sweep_planes": (C.c_int, [_vp, C.c_int, C.c_int]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libpscfgpu.so and bind every declared entry point."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(
                f"engine library {path} is missing: build it with `python -m pscf_b200.build`")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def to_c(system: System) -> PscfgSystem:
    s = PscfgSystem()
    s.dim = system.dim
    for i, v in enumerate(system.n):
        s.n[i] = v
    s.n_monomer = system.n_monomer
    s.n_chain = len(system.chains)
    s.n_solvent = len(system.solvents)
    s.ensemble = system.ensemble
    for i, c in enumerate(system.chains):
        s.n_block[i] = len(c.block_length)
        for b, (m, L) in enumerate(zip(c.block_monomer, c.block_length)):
            s.block_monomer[i][b] = m
            s.block_length[i][b] = L
        s.phi_chain[i] = c.phi
        s.mu_chain[i] = c.mu
    for i, sv in enumerate(system.solvents):
        s.solvent_monomer[i] = sv.monomer
        s.solvent_size[i] = sv.size
        s.phi_solvent[i] = sv.phi
        s.mu_solvent[i] = sv.mu
    for a in range(system.n_monomer):
        s.kuhn[a] = system.kuhn[a]
        for b in range(system.n_monomer):
            s.chi[a][b] = system.chi[a, b]
    s.chain_step = system.ds
    s.crystal_system = system.crystal_code
    for k, v in enumerate(system.cell_param):
        s.cell_param[k] = v
    return s


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pscfg error {code}: {msg}")
        self.code = code


class Engine:
    """A batch of SCFT instances of one grid shape on the GPU."""

    def __init__(self, systems: Sequence[System], precision: int = FP64):
        self.lib = load_library()
        if isinstance(systems, System):
            systems = [systems]
        # private copies: cell relaxation updates these, never the caller's objects
        self.systems: List[System] = [copy.deepcopy(s) for s in systems]
        arr = (PscfgSystem * len(self.systems))(*[to_c(s) for s in self.systems])
        h = _vp()
        rc = self.lib.pscfg_create(arr, len(self.systems), precision, C.byref(h))
        if rc != OK:
            raise EngineError(rc, self.lib.pscfg_last_error(None).decode())
        self._h = h
        self.precision = precision
        s0 = self.systems[0]
        self.nr, self.nk, self.M = s0.nr, s0.nk, s0.n_monomer
        self.n_inst = len(self.systems)

    def close(self):
        if getattr(self, "_h", None):
            self.lib.pscfg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, allow=()):
        if rc != OK and rc not in allow:
            raise EngineError(rc, self.lib.pscfg_last_error(self._h).decode())
        return rc

    # -- geometry --------------------------------------------------------
    def set_cell_param(self, inst: int, cell_param: Sequence[float]):
        cp = np.zeros(MAX_CELL_PARAM)
        cp[: len(cell_param)] = cell_param
        self._check(self.lib.pscfg_set_cell_param(self._h, inst, _ptr(cp)))
        self.systems[inst].cell_param = list(cell_param)

    def ksq(self, inst: int = 0) -> np.ndarray:
        out = np.zeros(self.nk)
        self._check(self.lib.pscfg_get_ksq(self._h, inst, _ptr(out)))
        return out

    # -- hot path --------------------------------------------------------
    def density(self, omega: np.ndarray):
        """omega [n_inst][M][nr] -> (rho [n_inst][M][nr], q [n_inst][MAXC])."""
        w = np.ascontiguousarray(omega, dtype=np.float64).reshape(self.n_inst, self.M, self.nr)
        rho = np.zeros_like(w)
        q = np.zeros((self.n_inst, MAX_CHAIN))
        qs = np.zeros((self.n_inst, MAX_SOLVENT))
        self._check(self.lib.pscfg_density(self._h, _ptr(w), _ptr(rho), _ptr(q), _ptr(qs)))
        self.q_solvent = qs
        return rho, q

    def density_device(self, omega_dev_ptr: int, rho_dev_ptr: int):
        q = np.zeros((self.n_inst, MAX_CHAIN))
        self._check(self.lib.pscfg_density_device(self._h, _vp(omega_dev_ptr), _vp(rho_dev_ptr), _ptr(q), None))
        return q

    def density_adjoint(self, grad_rho, grad_lnq=None, want_cell=False):
        """dL/domega for upstream dL/drho [n_inst][M][nr] and dL/dlnQ
        [n_inst][n_chain]; with want_cell also dL/dcell_param
        [n_inst][n_cell_param] (returns the pair)."""
        G = np.ascontiguousarray(grad_rho, dtype=np.float64).reshape(self.n_inst, self.M, self.nr)
        gq = None
        if grad_lnq is not None:
            gq = np.zeros((self.n_inst, MAX_CHAIN))
            a = np.asarray(grad_lnq, dtype=np.float64).reshape(self.n_inst, -1)
            gq[:, : a.shape[1]] = a
        out = np.zeros_like(G)
        if not want_cell:
            self._check(self.lib.pscfg_density_adjoint(self._h, _ptr(G), None if gq is None else _ptr(gq), _ptr(out)))
            return out
        gc = np.zeros((self.n_inst, MAX_CELL_PARAM))
        self._check(self.lib.pscfg_density_adjoint_cell(self._h, _ptr(G), None if gq is None else _ptr(gq), _ptr(out),
                                                        _ptr(gc)))
        ncp = len(self.systems[0].cell_param)
        return out, gc[:, :ncp].copy()

    def response_raw(self, inst: int, kvec, ktrans_sq: float, pert_monomer, pert_field, read_index, read_coef):
        """pscfg_response: density response of instance `inst` to the Bloch
        perturbations exp(ik.r) pert_field[p] of monomer pert_monomer[p],
        read at the waves read_index (complex coefficients read_coef).
        Returns out [n_pert][n_monomer][n_read]."""
        pm = np.ascontiguousarray(pert_monomer, dtype=np.int32)
        P = len(pm)
        W = np.ascontiguousarray(np.asarray(pert_field, dtype=np.complex128).reshape(P, self.nr))
        ri = np.ascontiguousarray(read_index, dtype=np.int32)
        rc = np.ascontiguousarray(np.asarray(read_coef, dtype=np.complex128).reshape(len(ri)))
        k = np.zeros(3)
        kv = np.asarray(kvec, dtype=np.float64).ravel()
        k[: min(3, kv.size)] = kv[:3]
        out = np.zeros((P, self.M, len(ri)))
        ip = C.POINTER(C.c_int)
        self._check(self.lib.pscfg_response(self._h, inst, _ptr(k), float(ktrans_sq), P, pm.ctypes.data_as(ip),
                                            W.view(np.float64).ctypes.data_as(_dp), len(ri),
                                            ri.ctypes.data_as(ip), rc.view(np.float64).ctypes.data_as(_dp),
                                            _ptr(out)))
        return out

    def scf_stress(self) -> np.ndarray:
        out = np.zeros((self.n_inst, MAX_CELL_PARAM))
        self._check(self.lib.pscfg_stress(self._h, _ptr(out)))
        return out

    def free_energy(self):
        out = np.zeros((self.n_inst, 2))
        mu = np.zeros((self.n_inst, MAX_CHAIN))
        self._check(self.lib.pscfg_free_energy(self._h, _ptr(out), _ptr(mu)))
        return out[:, 0].copy(), out[:, 1].copy(), mu

    def propagate(self, inst: int, omega_m, b: float, ds: float, q_in, nsteps: int = 1) -> np.ndarray:
        w = np.ascontiguousarray(omega_m, dtype=np.float64).ravel()
        q = np.ascontiguousarray(q_in, dtype=np.float64).ravel()
        out = np.zeros(self.nr)
        self._check(self.lib.pscfg_propagate(self._h, inst, _ptr(w), b, ds, _ptr(q), _ptr(out), nsteps))
        return out

    def propagators(self, inst: int = 0, chain: int = 0):
        ns = C.c_int(0)
        self._check(self.lib.pscfg_get_propagators(self._h, inst, chain, None, None, C.byref(ns)))
        qf = np.zeros((ns.value, self.nr))
        qr = np.zeros((ns.value, self.nr))
        self._check(self.lib.pscfg_get_propagators(self._h, inst, chain, _ptr(qf), _ptr(qr), None))
        return qf, qr

    def iterate_am(self, omega: np.ndarray, error_max=1e-10, max_itr=1000, n_hist=20, domain=False,
                   switch_error=0.0, mix_max=0.0, restart=0.0, graph_check=0):
        """Anderson-mixing solve of every instance; returns (omega, rho, results).
        graph_check > 0: whole iterations replay from a captured CUDA graph
        with the Anderson step on the device, the host checking the
        instances every graph_check iterations."""
        w = np.ascontiguousarray(omega, dtype=np.float64).reshape(self.n_inst, self.M, self.nr).copy()
        rho = np.zeros_like(w)
        prm = PscfgAmParam(max_itr, n_hist, 1 if domain else 0, error_max, switch_error, mix_max, restart,
                           graph_check)
        res = (PscfgAmResult * self.n_inst)()
        self._check(self.lib.pscfg_iterate_am(self._h, _ptr(w), C.byref(prm), _ptr(rho), res), allow=(ENOTCONV,))
        return w, rho, self._results(res, domain)

    def set_symmetry(self, inst: int, group_name: str):
        """Impose a space group (pscf_b200.groups) on instance `inst`."""
        from .groups import grid_ops
        s = self.systems[inst]
        M, t = grid_ops(group_name, list(s.ngrid))
        ops = np.zeros((len(M), 12), dtype=np.int32)
        ops[:, :9] = M.reshape(len(M), 9)
        ops[:, 9:] = t
        self._check(self.lib.pscfg_set_symmetry(self._h, inst, len(M), ops.ctypes.data_as(C.POINTER(C.c_int))))

    def set_basis(self, inst: int, basis):
        """Star basis (pscf_b200.basis.StarBasis) of instance `inst` for
        density_basis: the waves of its basis functions that lie in the r2c
        half grid, with their coefficients, as device tables."""
        k, star, coef = basis.half_grid_tables()
        ck = np.ascontiguousarray(k, dtype=np.int32)
        cs = np.ascontiguousarray(star, dtype=np.int32)
        cc = np.ascontiguousarray(np.stack([coef.real, coef.imag], axis=1), dtype=np.float64).ravel()
        self._check(self.lib.pscfg_set_basis(self._h, inst, basis.n_star, len(ck),
                                             ck.ctypes.data_as(C.POINTER(C.c_int)),
                                             cs.ctypes.data_as(C.POINTER(C.c_int)), _ptr(cc)))
        if not hasattr(self, "_n_star"):
            self._n_star = [0] * self.n_inst
        self._n_star[inst] = basis.n_star

    def density_basis(self, omega_basis):
        """density() in star coefficients: omega_basis is a list (or array)
        of [n_monomer, n_star_i] per instance; returns (rho_basis list, q)."""
        ws = [np.ascontiguousarray(w, dtype=np.float64).reshape(self.M, self._n_star[i])
              for i, w in enumerate(omega_basis)]
        flat = np.concatenate([w.ravel() for w in ws])
        rho = np.zeros_like(flat)
        q = np.zeros((self.n_inst, MAX_CHAIN))
        self._check(self.lib.pscfg_density_basis(self._h, _ptr(flat), _ptr(rho), _ptr(q), None))
        out, o = [], 0
        for w in ws:
            out.append(rho[o:o + w.size].reshape(w.shape))
            o += w.size
        return out, q

    def clear_symmetry(self, inst: int):
        self._check(self.lib.pscfg_set_symmetry(self._h, inst, 0, None))

    def _results(self, res, domain):
        out = []
        for i, r in enumerate(res):
            ncp = len(self.systems[i].cell_param)
            nch = len(self.systems[i].chains)
            out.append(dict(itr=r.itr, itr_fp32=r.itr_fp32, converged=bool(r.converged), error=r.error,
                            status=AM_STATUS.get(r.status, str(r.status)),
                            f_helmholtz=r.f_helmholtz, pressure=r.pressure,
                            stress=list(r.stress)[:ncp], cell_param=list(r.cell_param)[:ncp],
                            q=list(r.q)[:nch], mu_chain=list(r.mu_chain)[:nch]))
            if domain:
                self.systems[i].cell_param = list(r.cell_param)[:ncp]
        return out

    def am_begin(self, omega, error_max=1e-10, max_itr=1000, n_hist=20, domain=False, switch_error=0.0,
                 mix_max=0.0, restart=0.0, graph_check=0):
        w = None if omega is None else np.ascontiguousarray(omega, dtype=np.float64).reshape(self.n_inst, self.M, self.nr)
        self._am_domain = domain
        prm = PscfgAmParam(max_itr, n_hist, 1 if domain else 0, error_max, switch_error, mix_max, restart,
                           graph_check)
        self._check(self.lib.pscfg_am_begin(self._h, None if w is None else _ptr(w), C.byref(prm)))

    def am_iterate(self, iters: int = 1) -> int:
        rem = C.c_int(0)
        self._check(self.lib.pscfg_am_iterate(self._h, iters, C.byref(rem)))
        return rem.value

    def am_results(self, want_fields=True):
        res = (PscfgAmResult * self.n_inst)()
        w = np.zeros((self.n_inst, self.M, self.nr)) if want_fields else None
        rho = np.zeros((self.n_inst, self.M, self.nr)) if want_fields else None
        self._check(self.lib.pscfg_am_results(self._h, None if w is None else _ptr(w),
                                              None if rho is None else _ptr(rho), res))
        return w, rho, self._results(res, getattr(self, "_am_domain", False))

    def set_profiling(self, on: bool = True):
        self._check(self.lib.pscfg_set_profiling(self._h, 1 if on else 0))

    def profile(self) -> dict:
        out = np.zeros(6)
        self._check(self.lib.pscfg_get_profile(self._h, _ptr(out)))
        return dict(sweep_ms=out[0], contour_ms=out[1], stress_ms=out[2], mix_ms=out[3],
                    steps=int(out[4]), sweep_launches=int(out[5]))

    @property
    def stream(self) -> int:
        return int(self.lib.pscfg_stream(self._h) or 0)

    @property
    def steps_per_density(self) -> int:
        return int(self.lib.pscfg_steps_per_density(self._h))

    @property
    def launch_count(self) -> int:
        return int(self.lib.pscfg_launch_count(self._h))

    def sweep_planes(self, n_fields: int, fp32: bool = False) -> int:
        """Planes per CTA the measured choice gives the 3-D register sweep of
        n_fields fields (-1: the cluster sweep; 0 while undecided)."""
        return int(self.lib.pscfg_sweep_planes(self._h, n_fields, 1 if fp32 else 0))
