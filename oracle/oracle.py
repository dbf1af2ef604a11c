"""ctypes wrapper around the FP64 CPU oracle (oracle/pscf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check in
__graft_entry__.py and by bench.py's cpu_baseline / reference legs, as the
checker.  The engine (pscf_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

MAXM, MAXC, MAXB, MAXS, MAXCP = 4, 4, 8, 4, 6


class OrcSystem(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("n", C.c_int * 3),
        ("n_monomer", C.c_int),
        ("n_chain", C.c_int),
        ("n_solvent", C.c_int),
        ("ensemble", C.c_int),
        ("n_block", C.c_int * MAXC),
        ("block_monomer", (C.c_int * MAXB) * MAXC),
        ("block_length", (C.c_double * MAXB) * MAXC),
        ("kuhn", C.c_double * MAXM),
        ("chi", (C.c_double * MAXM) * MAXM),
        ("phi_chain", C.c_double * MAXC),
        ("mu_chain", C.c_double * MAXC),
        ("solvent_monomer", C.c_int * MAXS),
        ("solvent_size", C.c_double * MAXS),
        ("phi_solvent", C.c_double * MAXS),
        ("mu_solvent", C.c_double * MAXS),
        ("ds", C.c_double),
        ("G_basis", (C.c_double * 3) * 3),
        ("n_cell_param", C.c_int),
        ("dGG", ((C.c_double * 3) * 3) * MAXCP),
    ]


class OrcAmParam(C.Structure):
    _fields_ = [
        ("max_itr", C.c_int),
        ("n_hist", C.c_int),
        ("domain", C.c_int),
        ("crystal_system", C.c_int),
        ("verbose", C.c_int),
        ("error_max", C.c_double),
    ]


class OrcAmResult(C.Structure):
    _fields_ = [
        ("itr", C.c_int),
        ("converged", C.c_int),
        ("error", C.c_double),
        ("f_helmholtz", C.c_double),
        ("pressure", C.c_double),
        ("stress", C.c_double * MAXCP),
        ("cell_param", C.c_double * MAXCP),
        ("q", C.c_double * MAXC),
        ("mu_chain", C.c_double * MAXC),
    ]


_lib = None


def build():
    """Compile the oracle with gcc via oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        vp = C.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(OrcSystem)]
        L.orc_destroy.argtypes = [vp]
        L.orc_density.argtypes = [vp, dp, dp, dp, vp]
        L.orc_stress.argtypes = [vp, dp]
        L.orc_free_energy.argtypes = [vp, dp, dp, dp]
        L.orc_free_energy_FH.argtypes = [C.POINTER(OrcSystem)]
        L.orc_free_energy_FH.restype = C.c_double
        L.orc_set_cell.argtypes = [vp, dp, C.c_int, dp]
        L.orc_get_ksq.argtypes = [vp, dp]
        L.orc_chain_slices.argtypes = [vp, C.c_int]
        L.orc_chain_slices.restype = C.c_int
        L.orc_get_q.argtypes = [vp, C.c_int, dp, dp]
        L.orc_get_mu_phi.argtypes = [vp, dp, dp]
        L.orc_iterate_am.argtypes = [vp, dp, dp, C.POINTER(OrcAmParam), dp, C.POINTER(OrcAmResult)]
        L.orc_make_unit_cell.argtypes = [C.c_int, C.c_int, dp, dp, dp]
        L.orc_make_ksq.argtypes = [C.c_int, ip, dp, dp, vp]
        L.orc_G_to_bz.argtypes = [C.c_int, ip, dp, ip, ip]
        L.orc_chain_grid.argtypes = [C.c_int, dp, C.c_double, ip, dp]
        L.orc_chain_grid.restype = C.c_int
        L.orc_step.argtypes = [ip, dp, C.c_double, C.c_double, dp, dp, dp, C.c_int]
        L.orc_fft_r2c.argtypes = [ip, dp, dp]
        L.orc_fft_c2r.argtypes = [ip, dp, dp]
        L.orc_fft_c2c.argtypes = [ip, dp, C.c_int]
        L.orc_am_deviation.argtypes = [C.POINTER(OrcSystem), C.c_long, dp, dp, dp]
        L.orc_am_deviation.restype = C.c_double
        L.orc_set_symmetry.argtypes = [vp, C.c_int, ip, ip]
        L.orc_symmetrize.argtypes = [vp, dp]
        L.orc_density_batch.argtypes = [C.POINTER(OrcSystem), C.c_int, dp, vp, C.c_int]
        L.orc_set_fft_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def to_orc(system, cell_param=None) -> OrcSystem:
    """Flatten a pscf_b200.system.System into the oracle's C struct."""
    s = OrcSystem()
    s.dim = system.dim
    n = system.n
    for i in range(3):
        s.n[i] = n[i]
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
    s.ds = system.ds
    G, dGG, ncp = unit_cell(system.dim, system.crystal_code,
                            system.cell_param if cell_param is None else cell_param)
    for i in range(3):
        for j in range(3):
            s.G_basis[i][j] = G[i, j]
    s.n_cell_param = ncp
    for k in range(ncp):
        for i in range(3):
            for j in range(3):
                s.dGG[k][i][j] = dGG[k, i, j]
    return s


def unit_cell(dim, code, cell_param):
    G = np.zeros(9)
    dGG = np.zeros(MAXCP * 9)
    cp = np.zeros(MAXCP)
    cp[: len(cell_param)] = cell_param
    ncp = lib().orc_make_unit_cell(dim, code, cp, G, dGG)
    if ncp < 0:
        raise ValueError("unknown crystal system code %d" % code)
    return G.reshape(3, 3), dGG.reshape(MAXCP, 3, 3)[:ncp].copy(), ncp


def fft_r2c(field: np.ndarray) -> np.ndarray:
    """Unnormalised r2c FFT of an x-fastest field of shape (n3, n2, n1)."""
    f = np.ascontiguousarray(field, dtype=np.float64)
    n3, n2, n1 = f.shape
    out = np.zeros((n3, n2, n1 // 2 + 1, 2))
    lib().orc_fft_r2c(np.array([n1, n2, n3], np.int32), f.ravel(), out.reshape(-1))
    return out[..., 0] + 1j * out[..., 1]


def fft_c2r(spec: np.ndarray, n1: int) -> np.ndarray:
    s = np.ascontiguousarray(spec, dtype=np.complex128)
    n3, n2, _ = s.shape
    out = np.zeros((n3, n2, n1))
    inter = np.ascontiguousarray(np.stack([s.real, s.imag], axis=-1))
    lib().orc_fft_c2r(np.array([n1, n2, n3], np.int32), inter.reshape(-1), out.reshape(-1))
    return out


def set_fft_threads(n: int) -> None:
    """Threads of the oracle's 3-D transforms (1 = serial; results identical)."""
    lib().orc_set_fft_threads(int(n))


def make_ksq(dim, n, G):
    n = np.array(list(n) + [1] * (3 - len(n)), np.int32)
    nk = (n[0] // 2 + 1) * n[1] * n[2]
    ksq = np.zeros(nk)
    lib().orc_make_ksq(dim, n, np.ascontiguousarray(G, np.float64).ravel(), ksq, None)
    return ksq


def step(system, ksq, b, ds, omega, qin, nsteps=1):
    """nsteps applications of step_exp with block parameters (b, ds)."""
    n = np.array(system.n, np.int32)
    out = np.zeros(system.nr)
    lib().orc_step(n, np.ascontiguousarray(ksq, np.float64), b, ds,
                   np.ascontiguousarray(omega, np.float64).ravel(),
                   np.ascontiguousarray(qin, np.float64).ravel(), out, nsteps)
    return out


class Oracle:
    """One system on the CPU: density / stress / free energy / Anderson."""

    def __init__(self, system, cell_param=None):
        self.system = system
        self.cell_param = list(system.cell_param if cell_param is None else cell_param)
        self._s = to_orc(system, self.cell_param)
        self._c = lib().orc_create(C.byref(self._s))
        self.nr = system.nr
        self.M = system.n_monomer
        self.q = np.zeros(MAXC)

    def close(self):
        if self._c:
            lib().orc_destroy(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_symmetry(self, M, t):
        """Impose a space group: M int [nops,3,3], t int [nops,3] (grid units)."""
        M = np.ascontiguousarray(M, np.int32)
        t = np.ascontiguousarray(t, np.int32)
        lib().orc_set_symmetry(self._c, len(M), M.reshape(-1), t.reshape(-1))

    def symmetrize(self, field):
        f = np.ascontiguousarray(field, np.float64).ravel().copy()
        lib().orc_symmetrize(self._c, f)
        return f

    def set_cell(self, cell_param):
        self.cell_param = list(cell_param)
        G, dGG, ncp = unit_cell(self.system.dim, self.system.crystal_code, cell_param)
        full = np.zeros((MAXCP, 3, 3))
        full[:ncp] = dGG
        lib().orc_set_cell(self._c, np.ascontiguousarray(G).ravel(), ncp, full.ravel())

    def ksq(self):
        out = np.zeros(self.system.nk)
        lib().orc_get_ksq(self._c, out)
        return out

    def density(self, omega):
        w = np.ascontiguousarray(omega, np.float64).reshape(self.M, self.nr)
        rho = np.zeros((self.M, self.nr))
        q = np.zeros(MAXC)
        lib().orc_density(self._c, w.ravel(), rho.reshape(-1), q, None)
        self.q = q
        return rho, q[: len(self.system.chains)].copy()

    def stress(self):
        out = np.zeros(MAXCP)
        lib().orc_stress(self._c, out)
        return out[: self._s.n_cell_param].copy()

    def free_energy(self, omega, rho):
        out = np.zeros(2)
        lib().orc_free_energy(self._c, np.ascontiguousarray(omega, np.float64).ravel(),
                              np.ascontiguousarray(rho, np.float64).ravel(), out)
        return float(out[0]), float(out[1])

    def mu_phi(self):
        mu = np.zeros(MAXC)
        phi = np.zeros(MAXC)
        lib().orc_get_mu_phi(self._c, mu, phi)
        n = len(self.system.chains)
        return mu[:n], phi[:n]

    def propagators(self, chain=0):
        ns = lib().orc_chain_slices(self._c, chain)
        qf = np.zeros((ns, self.nr))
        qr = np.zeros((ns, self.nr))
        lib().orc_get_q(self._c, chain, qf.reshape(-1), qr.reshape(-1))
        return qf, qr

    def iterate_am(self, omega, error_max=1e-10, max_itr=1000, n_hist=20, domain=False, verbose=False):
        w = np.ascontiguousarray(omega, np.float64).reshape(self.M, self.nr).copy()
        cp = np.zeros(MAXCP)
        cp[: len(self.cell_param)] = self.cell_param
        prm = OrcAmParam(max_itr, n_hist, 1 if domain else 0, self.system.crystal_code,
                         1 if verbose else 0, error_max)
        res = OrcAmResult()
        rho = np.zeros((self.M, self.nr))
        lib().orc_iterate_am(self._c, w.reshape(-1), cp, C.byref(prm), rho.reshape(-1), C.byref(res))
        ncp = self._s.n_cell_param
        self.cell_param = list(cp[:ncp])
        out = dict(itr=res.itr, converged=bool(res.converged), error=res.error,
                   f_helmholtz=res.f_helmholtz, pressure=res.pressure,
                   stress=list(res.stress)[:ncp], cell_param=list(res.cell_param)[:ncp],
                   q=list(res.q)[: len(self.system.chains)],
                   mu_chain=list(res.mu_chain)[: len(self.system.chains)])
        return w, rho, out


def free_energy_fh(system):
    s = to_orc(system)
    return lib().orc_free_energy_FH(C.byref(s))


def density_batch(system, omegas: np.ndarray, nthreads: int, want_rho=False):
    """Independent density() evaluations over POSIX threads (CPU baseline)."""
    s = to_orc(system)
    w = np.ascontiguousarray(omegas, np.float64)
    n_inst = w.shape[0]
    rho = np.zeros_like(w) if want_rho else None
    lib().orc_density_batch(C.byref(s), n_inst, w.reshape(-1),
                            rho.ctypes.data if want_rho else None, nthreads)
    return rho
