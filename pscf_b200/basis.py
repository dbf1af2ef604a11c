"""Symmetry-adapted (star) basis on the FFT grid.

The reference represents omega and rho by coefficients of real basis
functions, one per star of waves related by the space group
(make_waves / make_stars, src/basis_mod.f90:453-1227; basis_to_kgrid /
kgrid_to_basis, src/grid_basis_mod.f90:47-200).  Here a star is the orbit
of a wave index G under the point operations G -> M^T G (mod n) of the
group's action on the grid, and its basis function is the projection of the
plane wave e^{iG.r} onto the group-invariant fields,

    P e_G = (1/|g|) sum_g exp(2 pi i G.t_g / n) e_{M_g^T G},

made real (centrosymmetric groups give a real function up to a phase) and
normalised to a grid average of 1 for its square.  Stars whose projection
vanishes are the reference's cancelled stars and are dropped.  Stars are
ordered by |G|^2 of their minimum-image wave, like the reference.

Coefficients are taken by FFT: a_s = <f, f_s> = sum_G conj(c_s(G)) F[f](G)/N.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np

from .groups import grid_ops


class StarBasis:
    def __init__(self, group_name: str, ngrid: Sequence[int], G_basis: np.ndarray = None):
        self.ngrid = list(ngrid)
        dim = len(ngrid)
        n = self.ngrid + [1] * (3 - dim)
        self.n = n
        self.nr = n[0] * n[1] * n[2]
        M, t = grid_ops(group_name, ngrid)
        nops = len(M)
        # all waves of the full grid (x fastest flat index)
        I3, I2, I1 = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
        G = np.stack([I1.ravel(), I2.ravel(), I3.ravel()], axis=1)          # [nr, 3]
        # minimum-image squared length for ordering (metric G_basis or identity)
        Gb = np.eye(3) if G_basis is None else np.asarray(G_basis)
        Gf = G.copy()
        for a in range(3):
            Gf[:, a] = np.where(Gf[:, a] > n[a] // 2, Gf[:, a] - n[a], Gf[:, a])
        v = Gf[:, :dim] @ Gb[:dim, :dim]
        gsq = (v * v).sum(axis=1)
        order = np.lexsort((np.arange(self.nr), np.round(gsq, 10)))
        nvec = np.array(n)
        visited = np.zeros(self.nr, dtype=bool)
        flat = lambda g: g[..., 0] + n[0] * (g[..., 1] + n[1] * g[..., 2])
        self.star_idx: List[np.ndarray] = []
        self.star_coef: List[np.ndarray] = []
        self.star_gsq: List[float] = []
        for w in order:
            if visited[w]:
                continue
            g0 = G[w]
            imgs = np.einsum("kji,j->ki", M, g0) % nvec                   # M^T g0
            ph = np.exp(2j * np.pi * (t * g0[None, :] / nvec[None, :]).sum(axis=1))
            keys = flat(imgs)
            uniq, inv = np.unique(keys, return_inverse=True)
            coef = np.zeros(len(uniq), dtype=complex)
            np.add.at(coef, inv, ph)
            coef /= nops
            visited[uniq] = True
            # real part or imaginary part, whichever survives (with the
            # conjugate partner -G inside the orbit for centrosymmetric groups)
            neg = flat((-G[uniq]) % nvec)
            pos = {int(k): i for i, k in enumerate(uniq)}
            partner = np.array([pos.get(int(k), -1) for k in neg])
            if np.any(partner < 0):
                cre, cim = coef, np.zeros_like(coef)
            else:
                cre = 0.5 * (coef + np.conj(coef[partner]))
                cim = 0.5 * (coef - np.conj(coef[partner])) / 1j
            best = cre if np.sum(np.abs(cre) ** 2) >= np.sum(np.abs(cim) ** 2) else cim
            nrm = np.sum(np.abs(best) ** 2)
            if nrm < 1e-20:
                continue                                                     # cancelled star
            self.star_idx.append(uniq)
            self.star_coef.append(best / np.sqrt(nrm))
            self.star_gsq.append(float(gsq[w]))
        self.n_star = len(self.star_idx)

    def half_grid_tables(self):
        """The waves of every star that lie in the r2c half grid
        (0 <= kx <= n1/2): their flat half-grid index kx + (n1/2+1)(ky + n2 kz),
        star index and coefficient -- the device tables of
        pscfg_set_basis.  The partner -G of every wave must belong to the
        same star with the conjugate coefficient (centrosymmetric groups)."""
        n = self.n
        n1h = n[0] // 2 + 1
        flat = lambda g: g[..., 0] + n[0] * (g[..., 1] + n[1] * g[..., 2])
        ks, ss, cs = [], [], []
        for s, (idx, c) in enumerate(zip(self.star_idx, self.star_coef)):
            x = idx % n[0]
            rest = idx // n[0]
            g = np.stack([x, rest % n[1], rest // n[1]], axis=1)
            neg = flat((-g) % np.array(n))
            pos = {int(k): i for i, k in enumerate(idx)}
            for i, kneg in enumerate(neg):
                j = pos.get(int(kneg), -1)
                if j < 0 or abs(c[j] - np.conj(c[i])) > 1e-12:
                    raise NotImplementedError("star basis tables need each wave's partner -G in its star "
                                              "(centrosymmetric groups)")
            keep = x <= n[0] // 2
            ks.append(x[keep] + n1h * rest[keep])
            ss.append(np.full(int(keep.sum()), s))
            cs.append(c[keep])
        return np.concatenate(ks), np.concatenate(ss), np.concatenate(cs)

    def _fft(self, f):
        n = self.n
        return np.fft.fftn(np.asarray(f, dtype=np.float64).reshape(n[2], n[1], n[0])).ravel(order="C")

    def _flat_fft_index(self, idx):
        # engine layout flat index x + n1 (y + n2 z) -> numpy fftn C-order index (z, y, x)
        n = self.n
        x = idx % n[0]
        y = (idx // n[0]) % n[1]
        z = idx // (n[0] * n[1])
        return (z * n[1] + y) * n[0] + x

    def to_basis(self, field) -> np.ndarray:
        """Coefficients a_s = <f, f_s> (grid average) of a grid field."""
        F = self._fft(field) / self.nr
        out = np.zeros(self.n_star)
        for s, (idx, c) in enumerate(zip(self.star_idx, self.star_coef)):
            out[s] = np.real(np.sum(np.conj(c) * F[self._flat_fft_index(idx)]))
        return out

    def to_grid(self, coeffs) -> np.ndarray:
        """Grid field sum_s a_s f_s (x fastest, flat)."""
        n = self.n
        F = np.zeros(self.nr, dtype=complex)
        for a, idx, c in zip(coeffs, self.star_idx, self.star_coef):
            F[self._flat_fft_index(idx)] += a * c
        f = np.fft.ifftn(F.reshape(n[2], n[1], n[0])).real * self.nr
        return f.ravel()
