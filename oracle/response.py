"""CPU restatement (numpy) of the reference's linear-response calculation
(the RESPONSE command).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the engine's
response path.  The engine (pscf_b200) never imports it.

Follows, in order:
  * calc_exp_grid          src/response_step_mod.f90:222-283 (order+2 levels
                           of exp(-omega ds/2), exp(-ds b^2 k^2/6) on the r2c
                           grid and exp(-ds b^2 |G+k|^2/6) on the full grid)
  * fft_step / fftc_step   src/response_step_mod.f90:160-219
  * ps_propagate           src/response_step_mod.f90:114-155
  * extrapolate_*          src/extrapolate_mod.f90:40-151 (order 1: (4 y2 - y1)/3)
  * calc_q0                src/response_mod.f90:697-861
  * calc_delq              src/response_mod.f90:864-1094
  * calc_delrho            src/response_mod.f90:1097-1186
  * calc_ksqgrid_new       src/response_mod.f90:1203-1238 with Greal_to_bz
                           src/grid_mod.f90:286-345
  * calc_perturb_field     src/response_mod.f90:1275-1291 (basis_to_kgrid with
                           karray_full/no_parity, src/grid_basis_mod.f90:47-128,
                           then fftc(-1))
  * drho_domega_id         src/response_mod.f90:389-468 (kgrid_to_basis with
                           no_parity, src/grid_basis_mod.f90:146-200)
  * calc_drho_domega_full  src/response_mod.f90:484-627 (dsytrf/dsytri on the
                           lower triangle, S = smm - spm^T spp^-1 spm, dsyev,
                           eval = 1/eval - chi(1,2), Shell sort ascending,
                           src/basis_mod.f90:1453-1483)
The reference calls response_startup with order = 1 (src/pscf.fp.f90:719);
only that order is restated.  FFTs are numpy's (pocketfft):
fftc(+1) = fftn / N, fftc(-1) = N ifftn, fft/ifft unnormalised r2c/c2r.
Grid arrays are flat, x fastest, reshaped to (n3, n2, n1) for the FFTs.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

from . import oracle as O


def chain_grid(block_length: Sequence[float], ds: float, order: int = 0):
    """make_chain_grid (src/chain_mod.f90:136-158), 0-based block starts."""
    bgn, bds = [0], []
    for L in block_length:
        iblk = int(L / ds / 2.0 + 0.5)
        if iblk == 0:
            iblk = 1
            d = L / 2.0
        else:
            d = L / float(iblk) / 2.0
        d /= 2.0 ** order
        iblk *= 2 ** order
        bds.append(d)
        bgn.append(bgn[-1] + 2 * iblk)
    return bgn, bds


def greal_to_bz(g: np.ndarray, dim: int, n: Sequence[int], G: np.ndarray) -> np.ndarray:
    """Minimum image of a real wave index over shifts +1, 0, -1 (in that
    order) of each grid extent, keeping the first strictly shorter one by
    more than 1e-8 (src/grid_mod.f90:286-345)."""
    best = np.zeros(3)
    gsq_min = 1.0e10
    rng = [(1, 0, -1) if a < dim else (0,) for a in range(3)]
    for i1 in rng[0]:
        for i2 in rng[1]:
            for i3 in rng[2]:
                t = np.zeros(3)
                sh = (i1, i2, i3)
                for a in range(dim):
                    t[a] = g[a] + sh[a] * n[a]
                v = t[:dim] @ G[:dim, :dim]
                gsq = float(v @ v)
                if gsq < gsq_min - 1.0e-8:
                    best = t.copy()
                    gsq_min = gsq
    return best


def ksq_grid_new(system, kvec: Sequence[float], ktrans_sq: float, G: np.ndarray) -> np.ndarray:
    """|G + k|^2 on the full grid, flat x fastest (calc_ksqgrid_new)."""
    dim, n = system.dim, system.n
    k = np.zeros(3)
    k[: len(kvec)] = kvec
    out = np.zeros(system.nr)
    for i3 in range(n[2]):
        for i2 in range(n[1]):
            for i1 in range(n[0]):
                gbz = greal_to_bz(np.array([i1, i2, i3], dtype=float) + k, dim, n, G)
                v = gbz[:dim] @ G[:dim, :dim]
                out[i1 + n[0] * (i2 + n[1] * i3)] = float(v @ v)
    return out + ktrans_sq


def transverse_ksq(dim: int, G: np.ndarray, kvec: Sequence[float]) -> float:
    """ktrans_sq as response_sweep computes it for kdim = dim + 1
    (src/response_mod.f90:347-355): the loop assigns (not accumulates)
    g_basis(1,i)**2, so the last assignment g_basis(1,dim)**2 is used."""
    if len(kvec) != dim + 1:
        return 0.0
    return float(G[0, dim - 1] ** 2) * float(kvec[dim]) ** 2


class Response:
    """Ideal-gas and incompressible response of a (converged) periodic
    state, for one grid and field omega [M][nr]."""

    def __init__(self, system, omega: np.ndarray, order: int = 1):
        if order != 1:
            raise ValueError("only the order the reference uses (1) is restated")
        self.s = system
        self.n = list(system.n)
        self.shape = (self.n[2], self.n[1], self.n[0])
        self.nr = system.nr
        self.omega = np.asarray(omega, dtype=np.float64).reshape(system.n_monomer, self.nr)
        self.order = order
        G, _, _ = O.unit_cell(system.dim, system.crystal_code, system.cell_param)
        self.G = G
        self.ksq = O.make_ksq(system.dim, self.n, G)            # r2c half grid [nk]
        self.chains = []
        for c in system.chains:
            self.chains.append({"c": c, "grid": chain_grid(c.block_length, system.ds),
                                "grids0": [chain_grid(c.block_length, system.ds, o) for o in range(order + 1)],
                                "N": float(sum(c.block_length))})
        self.calc_q0()

    # -- transforms ---------------------------------------------------
    def _rfft(self, f):
        return np.fft.rfftn(f.reshape(self.shape))

    def _irfft(self, F):
        return np.fft.irfftn(F, s=self.shape, axes=(0, 1, 2)).ravel() * self.nr

    def exp_grid(self, monomer: int, ds: float, ksq_new=None):
        """calc_exp_grid: levels i = 0 .. order+1 with ds_i = ds / 2^i."""
        b = self.s.kuhn[monomer]
        ek, eo, ekn, dsa = [], [], [], []
        d = ds
        kh = self.ksq.reshape(self.shape[0], self.shape[1], self.n[0] // 2 + 1)
        for _ in range(self.order + 2):
            dsa.append(d)
            ek.append(np.exp(-kh * d * b ** 2 / 6.0))
            eo.append(np.exp(-self.omega[monomer] * d / 2.0))
            if ksq_new is not None:
                ekn.append(np.exp(-ksq_new * d * b ** 2 / 6.0).reshape(self.shape))
            d = d / 2.0
        return {"ek": ek, "eo": eo, "ekn": ekn, "ds": dsa}

    def fft_step(self, X, level, q):
        """src/response_step_mod.f90:160-183."""
        qr = X["eo"][level] * q
        qk = self._rfft(qr) * X["ek"][level]
        return X["eo"][level] * self._irfft(qk) / self.nr

    def fftc_step(self, X, level, q):
        """src/response_step_mod.f90:199-219 (fftc(+1) divides by N)."""
        qr = (X["eo"][level] * q).reshape(self.shape)
        qk = np.fft.fftn(qr) / self.nr * X["ekn"][level]
        return (np.fft.ifftn(qk) * self.nr).ravel() * X["eo"][level]

    # -- unperturbed chains (calc_q0) -----------------------------------
    def calc_q0(self):
        order = self.order
        for ch in self.chains:
            c = ch["c"]
            bgn, bds = ch["grid"]
            ns = bgn[-1]
            qf = np.zeros((ns + 1, self.nr))
            qr = np.zeros((ns + 1, self.nr))
            qf[0] = 1.0
            qr[ns] = 1.0
            c0f = [np.zeros((ch["grids0"][o][0][-1] + 1, self.nr)) for o in range(order + 1)]
            c0r = [np.zeros((ch["grids0"][o][0][-1] + 1, self.nr)) for o in range(order + 1)]
            for o in range(order + 1):
                c0f[o][0] = 1.0
                c0r[o][-1] = 1.0
            for b in range(len(c.block_length)):
                X = self.exp_grid(c.block_monomer[b], bds[b])
                for j in range(bgn[b] + 1, bgn[b + 1] + 1):
                    for o in range(order + 1):
                        pace = 2 ** o
                        c0f[o][(j - 1) * pace + 1] = self.fft_step(X, o, qf[j - 1])
                        for i in range((j - 1) * pace + 2, j * pace + 1):
                            c0f[o][i] = self.fft_step(X, o, c0f[o][i - 1])
                    qf[j] = (4.0 * c0f[1][j * 2] - c0f[0][j]) / 3.0
            for b in range(len(c.block_length) - 1, -1, -1):
                X = self.exp_grid(c.block_monomer[b], bds[b])
                for j in range(bgn[b + 1] - 1, bgn[b] - 1, -1):
                    for o in range(order + 1):
                        pace = 2 ** o
                        c0r[o][(j + 1) * pace - 1] = self.fft_step(X, o, qr[j + 1])
                        for i in range((j + 1) * pace - 2, j * pace - 1, -1):
                            c0r[o][i] = self.fft_step(X, o, c0r[o][i + 1])
                    qr[j] = (4.0 * c0r[1][j * 2] - c0r[0][j]) / 3.0
            ch.update(qf=qf, qr=qr, c0f=c0f, c0r=c0r, bigQ=float(np.mean(qr[0])))

    # -- perturbed chains (calc_delq) -----------------------------------
    def ps_propagate(self, X, dq_in, p_mon, field, f_inhomo, monomer, o):
        """src/response_step_mod.f90:114-155."""
        dq = dq_in
        dsl = X["ds"][o]
        for i in range(2 ** o):
            dq = self.fftc_step(X, o, dq)
            if monomer == p_mon:
                fout = self.fftc_step(X, o + 1, f_inhomo[i] * field)
                dq = dq - fout * dsl
        return dq

    def calc_delq(self, p_mon, field, ksq_new):
        order = self.order
        for ch in self.chains:
            c = ch["c"]
            bgn, bds = ch["grid"]
            nblk = len(c.block_length)
            ns = bgn[-1]
            dqf = np.zeros((ns + 1, self.nr), dtype=complex)
            dqr = np.zeros((ns + 1, self.nr), dtype=complex)
            qf, qr, c0f, c0r = ch["qf"], ch["qr"], ch["c0f"], ch["c0r"]
            for b in range(nblk):
                m = c.block_monomer[b]
                if b == 0 and m != p_mon:
                    continue
                X = self.exp_grid(m, bds[b], ksq_new)
                for j in range(bgn[b] + 1, bgn[b + 1] + 1):
                    d = []
                    for o in range(order + 1):
                        pace = 2 ** o
                        nb = (j - 1) * pace
                        qi = [(c0f[o][nb + 1] + qf[j - 1]) / 2.0]
                        for jj in range(2, pace + 1):
                            qi.append((c0f[o][nb + jj] + c0f[o][nb + jj - 1]) / 2.0)
                        d.append(self.ps_propagate(X, dqf[j - 1], p_mon, field, qi, m, o))
                    dqf[j] = (4.0 * d[1] - d[0]) / 3.0
            for b in range(nblk - 1, -1, -1):
                m = c.block_monomer[b]
                if b == nblk - 1 and m != p_mon:
                    continue
                X = self.exp_grid(m, bds[b], ksq_new)
                for j in range(bgn[b + 1] - 1, bgn[b] - 1, -1):
                    d = []
                    for o in range(order + 1):
                        pace = 2 ** o
                        nb = (j + 1) * pace
                        qi = [(c0r[o][nb - 1] + qr[j + 1]) / 2.0]
                        for jj in range(2, pace + 1):
                            qi.append((c0r[o][nb - jj] + c0r[o][nb - jj + 1]) / 2.0)
                        d.append(self.ps_propagate(X, dqr[j + 1], p_mon, field, qi, m, o))
                    dqr[j] = (4.0 * d[1] - d[0]) / 3.0
            ch.update(dqf=dqf, dqr=dqr)

    def calc_delrho(self) -> np.ndarray:
        """Simpson per block of qf dqr + qr dqf, times phi/(N Q)."""
        M = self.s.n_monomer
        drho = np.zeros((M, self.nr), dtype=complex)
        for ch in self.chains:
            c = ch["c"]
            bgn, bds = ch["grid"]
            part = np.zeros((M, self.nr), dtype=complex)
            for b in range(len(c.block_length)):
                m = c.block_monomer[b]
                i0, i1 = bgn[b], bgn[b + 1]
                acc = np.zeros(self.nr, dtype=complex)
                for i in range(i0, i1 + 1):
                    w = 1.0 if i in (i0, i1) else (4.0 if (i - i0) % 2 == 1 else 2.0)
                    acc = acc + w * (ch["qf"][i] * ch["dqr"][i] + ch["qr"][i] * ch["dqf"][i])
                part[m] += acc * bds[b] / 3.0
            drho += part * c.phi / (ch["N"] * ch["bigQ"])
        return drho

    # -- response matrices ------------------------------------------------
    def perturb_field(self, idx, coef) -> np.ndarray:
        """Basis function on the grid (basis_to_kgrid full/no_parity, then
        the unnormalised backward transform)."""
        kg = np.zeros(self.nr, dtype=complex)
        kg[np.asarray(idx)] = np.asarray(coef)
        return (np.fft.ifftn(kg.reshape(self.shape)) * self.nr).ravel()

    def drho_domega_id(self, kvec, ktrans_sq, basis: List[Tuple[np.ndarray, np.ndarray]]):
        """Returns (smm packed as full lower-triangle matrix, spm, spp) after
        the sign flip of response_sweep, and the raw coefficients
        drho[p_mon][i_gp][i][k1]."""
        if self.s.n_monomer != 2:
            raise ValueError("the reference's response code handles two monomers only")
        ksq_new = ksq_grid_new(self.s, kvec, ktrans_sq, self.G)
        nb = len(basis)
        smm = np.zeros((nb, nb))
        spm = np.zeros((nb, nb))
        spp = np.zeros((nb, nb))
        raw = np.zeros((2, nb, 2, nb))
        for p in range(2):
            for g, (idx, coef) in enumerate(basis):
                field = self.perturb_field(idx, coef)
                self.calc_delq(p, field, ksq_new)
                drho = self.calc_delrho()
                for i in range(2):
                    dk = np.fft.fftn(drho[i].reshape(self.shape)).ravel() / self.nr
                    for k1, (idx1, coef1) in enumerate(basis):
                        val = float(np.real(dk[idx1[0]] / coef1[0]))
                        raw[p, g, i, k1] = val
                        sgn_mm = (-1.0) ** ((i + 1) + (p + 1))
                        sgn_pm = (-1.0) ** (1 + (p + 1))
                        if k1 >= g:
                            smm[k1, g] += sgn_mm * val
                        spm[k1, g] += sgn_pm * val
                        spp[k1, g] += val
        return -smm / 2.0, -spm / 2.0, -spp / 2.0, raw


def lower_sym(a: np.ndarray) -> np.ndarray:
    low = np.tril(a)
    return low + np.tril(a, -1).T


def shell_sort(a: np.ndarray, index: np.ndarray):
    """Shell insertion sort ascending with index (src/basis_mod.f90:1453-1483)."""
    a = a.copy()
    index = index.copy()
    n = len(a)
    inc = 1
    while True:
        inc = 3 * inc + 1
        if inc > n:
            break
    while True:
        inc //= 3
        for i in range(inc, n):
            v, k, j = a[i], index[i], i
            while a[j - inc] > v:
                a[j] = a[j - inc]
                index[j] = index[j - inc]
                j -= inc
                if j < inc:
                    break
            a[j] = v
            index[j] = k
        if inc <= 1:
            break
    return a, index


def drho_domega_full(smm, spm, spp, chi12: float, n_eigval_out: int):
    """Eigenvalues 1/eval - chi of S = smm - spm^T spp^-1 spm (lower
    triangles as the reference's LAPACK calls read them), sorted ascending,
    with the divergent k = 0 eigenvalue dropped.  Returns (eval, evec)."""
    sppi = np.linalg.inv(lower_sym(spp))
    S = lower_sym(smm) - lower_sym(spm.T @ sppi @ spm)
    ev, V = np.linalg.eigh(S)
    ev = 1.0 / ev - chi12
    ev, idx = shell_sort(ev, np.arange(len(ev)))
    if abs(ev[0]) > 1.0e5:
        n_out = min(n_eigval_out, len(ev) - 1)
        return ev[1:1 + n_out], V[:, idx[1:1 + n_out]]
    n_out = min(n_eigval_out, len(ev))
    return ev[:n_out], V[:, idx[:n_out]]
