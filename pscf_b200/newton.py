"""Newton-Raphson / Broyden iteration in the star basis (iterate_NR).

Restates the reference's iterate_NR (src/iterate_mod.fp.f90:273-656):
  * residual (make_residual :787-828): for every non-uniform star i,
    sum_a rho_a,i (incompressibility) and, for monomers a >= 2,
    omega_a,i - xi_i - sum_b chi_ba rho_b,i with the pressure field
    xi_i = omega_1,i - sum_b chi_b1 rho_b,i; plus the stress when the cell
    is relaxed;
  * Jacobian (Jacobian_response :840-967, response_pd_omega/cell
    src/response_pd_mod.f90:91-147, 276-339) by forward differences with
    increment 1e-8 -- every column of the Jacobian comes from one density
    evaluation, and all of them run as the instances of one batched engine
    call instead of one after another; the stress rows use the reference's
    symmetry d stress/d omega = d rho/d cell;
  * the Jacobian is inverted once (LU, torch.linalg on the GPU when one is
    present) and then updated by Broyden rank-1 corrections of its inverse
    (:443-458); steps use the backtracking line search of
    update_with_linesearch (:544-654);
  * convergence when max(|SCF residual|, 100 |stress residual|) < error_max
    (:380-385).

The density provider is any callable
  provider(omegas[B, M, nr], cells[B] or None) ->
      dict(rho[B, M, nr], q[B, n_chain], stress[B, ncp] or None)
so the same loop runs on the engine (pscf_b200.newton.EngineProvider) or,
in tests, on the CPU oracle.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .basis import StarBasis
from .system import System


def _inverse(J: np.ndarray) -> np.ndarray:
    try:
        import torch
        if torch.cuda.is_available():
            t = torch.from_numpy(J).to("cuda")
            return torch.linalg.inv(t).cpu().numpy()
    except Exception:
        pass
    return np.linalg.inv(J)


class EngineProvider:
    """Batched density (and stress) of many omega / cell variants of one
    system on the GPU engine; instances are reused across calls."""

    def __init__(self, system: System, group: Optional[str], max_batch: int = 256):
        from .engine import Engine, FP64
        import copy
        self.system = system
        self.max_batch = max_batch
        self.engine = Engine([copy.deepcopy(system) for _ in range(max_batch)], FP64)
        self.group = group
        if group:
            for i in range(max_batch):
                self.engine.set_symmetry(i, group)
        self.cells = [list(system.cell_param) for _ in range(max_batch)]

    def __call__(self, omegas: np.ndarray, cells=None, want_stress=False):
        B = omegas.shape[0]
        e = self.engine
        rho = np.zeros_like(omegas)
        q = np.zeros((B, len(self.system.chains)))
        stress = np.zeros((B, len(self.system.cell_param))) if want_stress else None
        for c0 in range(0, B, self.max_batch):
            c1 = min(B, c0 + self.max_batch)
            w = np.zeros((self.max_batch, e.M, e.nr))
            w[: c1 - c0] = omegas[c0:c1]
            w[c1 - c0:] = omegas[c0]
            for k in range(self.max_batch):
                cell = list(cells[c0 + k]) if (cells is not None and c0 + k < B) else list(self.system.cell_param)
                if cell != self.cells[k]:
                    e.set_cell_param(k, cell)
                    self.cells[k] = cell
            r, qq = e.density(w)
            rho[c0:c1] = r[: c1 - c0]
            q[c0:c1] = qq[: c1 - c0, : q.shape[1]]
            if want_stress:
                st = e.scf_stress()
                stress[c0:c1] = st[: c1 - c0, : stress.shape[1]]
        return dict(rho=rho, q=q, stress=stress)


def star_gsq(basis: StarBasis, system: System, cell_param=None) -> np.ndarray:
    """|G|^2 of every star (its first wave, minimum image over the shifts
    -1, 0, +1 of each index as in G_to_bz, src/grid_mod.f90:225-283), with
    the reciprocal basis of the cell (2 pi included, like ksq)."""
    Gb, _, _ = system.unit_cell(cell_param)
    dim = system.dim
    n = np.array(basis.n[:dim])
    out = np.zeros(basis.n_star)
    shifts = np.array(np.meshgrid(*[[-1, 0, 1]] * dim, indexing="ij")).reshape(dim, -1).T
    for s, idx in enumerate(basis.star_idx):
        w = int(idx[0])
        g = np.array([w % basis.n[0], (w // basis.n[0]) % basis.n[1], w // (basis.n[0] * basis.n[1])])[:dim]
        g = np.where(g > n // 2, g - n, g)
        v = (g[None, :] + shifts * n[None, :]) @ np.asarray(Gb)[:dim, :dim]
        out[s] = float(np.min((v * v).sum(axis=1)))
    return out


def debye_correlation(system: System, gsq: np.ndarray) -> np.ndarray:
    """Ideal-chain correlation functions corrlt(alpha, beta, star) of the
    homogeneous melt at q^2 = |G|^2 (make_correlation,
    src/response_pd_mod.f90:419-526): per chain, with x_i = L_i b_i^2 q^2/6
    and f_i = L_i / L, the self terms g1(x_i) f_i^2 phi L and the block-pair
    terms g2(x_i, x_j) prod_{i<k<j} exp(-x_k) f_i f_j phi L (twice on the
    diagonal), g1(x) = 2(e^-x + x - 1)/x^2, g2 = (1 - e^-x1)/x1 (1 - e^-x2)/x2."""
    eps = 1e-14

    def g1(x):
        return 2.0 * (math.exp(-x) + x - 1.0) / (x * x) if x > eps else 1.0

    def g2(x1, x2):
        a = (1.0 - math.exp(-x1)) / x1 if x1 > eps else 1.0
        b = (1.0 - math.exp(-x2)) / x2 if x2 > eps else 1.0
        return a * b

    M = system.n_monomer
    kuhn = system.kuhn
    corr = np.zeros((M, M, len(gsq)))
    for s, g in enumerate(gsq):
        q = g / 6.0
        for ch in system.chains:
            L = ch.length
            phiL = ch.phi * L
            mon = list(ch.block_monomer)
            x = [lb * kuhn[m] ** 2 * q for lb, m in zip(ch.block_length, mon)]
            f = [lb / L for lb in ch.block_length]
            nb = len(mon)
            for i in range(nb):
                corr[mon[i], mon[i], s] += g1(x[i]) * f[i] ** 2 * phiL
            for i in range(nb):
                for j in range(i + 1, nb):
                    prop = 1.0
                    for k in range(i + 1, j):
                        prop *= math.exp(-x[k])
                    t = g2(x[i], x[j]) * prop * f[i] * f[j] * phiL
                    a, b = mon[i], mon[j]
                    if a == b:
                        corr[a, a, s] += 2.0 * t
                    else:
                        corr[a, b, s] += t
                        corr[b, a, s] += t
    return corr


def iterate_nr(provider, basis: StarBasis, system: System, omega_grid: np.ndarray, error_max: float = 1e-10,
               max_itr: int = 100, domain: bool = False, crystal_update=None, n_cut: Optional[int] = None):
    """Newton/Broyden solve.  omega_grid [M, nr] (symmetric).  n_cut: the
    reference's N_cut -- finite-difference Jacobian columns for the first
    n_cut stars only, the rest from the Debye functions of the homogeneous
    melt (response_pd_omega, src/response_pd_mod.f90:91-147); None: every
    star by differences.  Returns (omega_grid, rho_grid, result dict)."""
    M = system.n_monomer
    N = basis.n_star
    ens = system.ensemble
    i0 = 1 - ens                       # first star with unknowns (0-based)
    nI = N - i0
    cell = list(system.cell_param)
    ncp = len(cell) if domain else 0
    n_res = M * nI + ncp
    chi = system.chi
    large = 100.0
    stress_rescale = 100.0
    error_index = n_res - ncp

    omega = np.stack([basis.to_basis(omega_grid[a]) for a in range(M)])      # [M, N]
    if ens == 0:
        omega[:, 0] = system.omega_uniform()                                  # set_omega_uniform

    def grid_of(om):
        return np.stack([basis.to_grid(om[a]) for a in range(M)])

    def evaluate(om, cl, want_stress):
        out = provider(grid_of(om)[None], [cl] if cl is not None else None, want_stress=want_stress)
        rho = np.stack([basis.to_basis(out["rho"][0, a]) for a in range(M)])
        st = out["stress"][0] if want_stress else None
        return rho, out["q"][0], st

    def residual(om, rho, st):
        res = np.zeros(n_res)
        xi = om[0] - chi[:, 0] @ rho                                          # [N]
        l = 0
        for i in range(i0, N):
            res[l] = rho[:, i].sum()
            l += 1
            for a in range(1, M):
                res[l] = om[a, i] - xi[i] - chi[:, a] @ rho[:, i]
                l += 1
        if ens == 1:
            res[0] -= 1.0
        if domain:
            res[l:l + ncp] = st[:ncp]
        return res

    def errors(res):
        e1 = np.max(np.abs(res[:error_index])) if error_index > 0 else 0.0
        e2 = np.max(np.abs(res[error_index - 1:])) if n_res > 0 else 0.0
        return max(e1, e2 * stress_rescale) if domain else e1

    cut = N if n_cut is None else max(0, min(int(n_cut), N))

    def jacobian(om, cl, rho0):
        # forward differences of rho in the unknowns of the first `cut`
        # stars, one batched call (response_pd_omega)
        inc = 1e-8
        nfd = cut if cut > 1 else i0
        cols = [(b, j) for j in range(i0, nfd) for b in range(M)]
        oms = np.empty((len(cols), M, basis.nr))
        g0 = grid_of(om)
        for c, (b, j) in enumerate(cols):
            w = om.copy()
            w[b, j] += inc
            oms[c] = g0
            oms[c, b] = basis.to_grid(w[b])
        cells = [cl] * len(cols) if domain else None
        out = provider(oms, cells, want_stress=False)
        drho = np.zeros((M, N, M, N))
        for c, (b, j) in enumerate(cols):
            p = np.stack([basis.to_basis(out["rho"][c, a]) for a in range(M)])
            drho[:, i0:, b, j] = (p[:, i0:] - rho0[:, i0:]) / inc
        if nfd < N:
            # rows of the differenced stars by symmetry, then the diagonal
            # Debye response beyond them (debye_rsp, :160-180)
            for j in range(nfd, N):
                drho[:, i0:nfd, :, j] = np.transpose(drho[:, j, :, i0:nfd], (1, 2, 0))
            corr = debye_correlation(system, star_gsq(basis, system, cl))
            for j in range(nfd, N):
                drho[:, j, :, j] = -corr[:, :, j]
        dxi = np.zeros((N, M, N))                                             # dxi(i, beta, j)
        for j in range(N):
            for b in range(M):
                dxi[:, b, j] = -(chi[:, 0] @ drho[:, :, b, j])
        for i in range(N):
            dxi[i, 0, i] += 1.0
        J = np.zeros((n_res, n_res))
        for j in range(i0, N):
            for b in range(M):
                col = b + M * (j - i0)
                for i in range(i0, N):
                    J[M * (i - i0), col] = drho[:, i, b, j].sum()
                    for a in range(1, M):
                        J[a + M * (i - i0), col] = -(chi[:, a] @ drho[:, i, b, j]) - dxi[i, b, j]
                if b > 0:
                    J[col, col] += 1.0
        if domain:
            # response_pd_cell: d rho / d cell and d stress / d cell
            _, _, st0 = evaluate(om, cl, True)
            cells = []
            for k in range(ncp):
                c2 = list(cl)
                c2[k] += inc
                cells.append(c2)
            out = provider(np.repeat(g0[None], ncp, axis=0), cells, want_stress=True)
            for k in range(ncp):
                p = np.stack([basis.to_basis(out["rho"][k, a]) for a in range(M)])
                drc = np.zeros((M, N))
                drc[:, i0:] = (p[:, i0:] - rho0[:, i0:]) / inc
                dst = (out["stress"][k][:ncp] - st0[:ncp]) / inc
                dxic = -(chi[:, 0] @ drc)
                row = M * nI + k
                for j in range(i0, N):
                    for a in range(M):
                        J[row, a + M * (j - i0)] = drc[a, j]
                colk = M * nI + k
                for i in range(i0, N):
                    J[M * (i - i0), colk] = drc[:, i].sum()
                    for a in range(1, M):
                        J[a + M * (i - i0), colk] = -(chi[:, a] @ drc[:, i]) - dxic[i]
                J[M * nI:M * nI + ncp, colk] = dst
        return J

    def apply_step(om, cl, delta):
        w = om.copy()
        k = 0
        for i in range(i0, N):
            for a in range(M):
                w[a, i] += delta[k]
                k += 1
        c2 = list(cl)
        if domain:
            for b in range(ncp):
                c2[b] = cl[b] + delta[M * nI + b]
        return w, c2

    rho, q, st = evaluate(omega, cell, domain)
    vsum = float(sum(np.dot(omega[a, i0:], omega[a, i0:]) for a in range(M)))
    if domain:
        vsum += float(np.dot(cell[:ncp], cell[:ncp]))
    stpmax = 100.0 * max(math.sqrt(vsum), float(n_res))
    res = residual(omega, rho, st)
    error = errors(res)
    Jinv = None
    r_old = None
    delta = None
    lam = 1.0
    itr = 0
    converged = False
    while True:
        if error < error_max:
            converged = True
            break
        if itr > max_itr or not (error <= 100.0 * large):
            break
        if Jinv is None:
            J = jacobian(omega, cell, rho)
            Jinv = _inverse(J)
        if itr > 0:
            # Broyden update of the inverse Jacobian (:443-458)
            dn = float(np.dot(delta, delta))
            dlt = delta / dn
            r_o = res - (1.0 - lam) * r_old
            u = Jinv @ r_o
            v = Jinv.T @ dlt
            uv = 1.0 + float(np.dot(v, r_o))
            u = u / uv
            Jinv = Jinv - np.outer(u, v)
        r_old = res.copy()
        p = -Jinv @ res
        fold = 0.5 * float(np.dot(res, res))
        slope = -2.0 * fold
        # update_with_linesearch (:544-654)
        vs = math.sqrt(float(np.dot(p, p)))
        if vs > stpmax:
            p = p * stpmax / vs
            slope = slope * stpmax / vs
        test = 0.0
        k = 0
        for i in range(i0, N):
            for a in range(M):
                test = max(test, abs(p[k]) / max(abs(omega[a, i]), 1.0))
                k += 1
        for b in range(ncp):
            test = max(test, abs(p[k + b]) / max(abs(cell[b]), 1.0))
        lamin = 1e-7 / test if test > 0 else 0.0
        lam = 1.0
        ow, ocell = omega.copy(), list(cell)
        lam2 = f2 = 0.0
        while True:
            delta = lam * p
            omega, cell = apply_step(ow, ocell, delta)
            if domain and crystal_update is not None:
                crystal_update(cell)
            rho, q, st = evaluate(omega, cell, domain)
            res = residual(omega, rho, st)
            error = errors(res)
            fnew = 0.5 * float(np.dot(res, res))
            if lam < lamin or fnew < fold + 1e-4 * lam * slope:
                break
            if lam == 1.0:
                tmplam = -slope / (2.0 * (fnew - fold - slope))
            else:
                rhs1 = fnew - fold - lam * slope
                rhs2 = f2 - fold - lam2 * slope
                a_ = (rhs1 / lam ** 2 - rhs2 / lam2 ** 2) / (lam - lam2)
                b_ = (-lam2 * rhs1 / lam ** 2 + lam * rhs2 / lam2 ** 2) / (lam - lam2)
                if a_ == 0.0:
                    tmplam = -slope / (2.0 * b_)
                else:
                    disc = b_ * b_ - 3.0 * a_ * slope
                    if disc < 0.0:
                        tmplam = 0.5 * lam
                    elif b_ < 0.0:
                        tmplam = (-b_ + math.sqrt(disc)) / (3.0 * a_)
                    else:
                        tmplam = -slope / (b_ + math.sqrt(disc))
                tmplam = min(tmplam, 0.5 * lam)
            lam2, f2 = lam, fnew
            lam = max(tmplam, 0.1 * lam)
        itr += 1
    om_grid = grid_of(omega)
    rho_grid = np.stack([basis.to_grid(rho[a]) for a in range(M)])
    return om_grid, rho_grid, dict(itr=itr, converged=converged, error=error, cell_param=list(cell),
                                   q=list(q), omega_basis=omega, rho_basis=rho)
