"""Symmetry-adapted (star) basis on the FFT grid.

The reference represents omega and rho by coefficients of real basis
functions, one per star of waves related by the space group
(make_waves / make_stars, src/basis_mod.f90:453-1227; basis_to_kgrid /
kgrid_to_basis, src/grid_basis_mod.f90:47-200).  Here a star is the orbit
of a wave index G under the point operations G -> M^T G (mod n) of the
group's action on the grid, and its star function is the projection of the
plane wave e^{iG.r} onto the group-invariant fields,

    phi = P e_G = (1/|g|) sum_g exp(2 pi i G.t_g / n) e_{M_g^T G},

normalised to a grid average of 1 for |phi|^2.  Stars whose projection
vanishes are the reference's cancelled stars and are dropped.  Stars are
ordered by |G|^2 of their minimum-image wave, like the reference.

A star closed under inversion (-G in the star for every G; every star of a
centrosymmetric group) gives one real basis function: phi itself, or -i phi
when phi is odd under inversion (the reference's sine-like closed stars,
basis_sign = -1).  In a group without inversion, stars also come in pairs
related by inversion (star_invert = +1 / -1, src/basis_mod.f90:206-310):
the second star's function is conj(phi), and the pair gives the two real
functions (phi + conj phi)/sqrt(2) and (phi - conj phi)/(i sqrt(2)), listed
one after the other (cosine-like first).  Every basis function is thus
real, with coefficients c(-G) = conj c(G) over a wave set closed under
inversion, and the functions are orthonormal.

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
        flat = lambda g: g[..., 0] + n[0] * (g[..., 1] + n[1] * g[..., 2])
        # orbits of the point operations g -> M^T g (mod n), each led by its
        # member that comes first in `order` (a walk through `order` that
        # skips waves already seen meets the same leaders in the same order)
        rank = np.empty(self.nr, dtype=np.int64)
        rank[order] = np.arange(self.nr)
        lead_rank = np.empty(self.nr, dtype=np.int64)
        # images M^T g of a block of waves as one exact small-integer product
        Mt = np.asarray(M, dtype=np.float64).transpose(1, 0, 2).reshape(3, nops * 3)     # [j, (k, i)]

        nvec32 = nvec.astype(np.int32)

        def images(g):
            return np.rint(g.astype(np.float64) @ Mt).astype(np.int32).reshape(len(g), nops, 3) % nvec32
        chunk = max(1, (1 << 22) // nops)
        for c0 in range(0, self.nr, chunk):
            keys = flat(images(G[c0:c0 + chunk]))                                      # [waves, ops]
            lead_rank[c0:c0 + chunk] = rank[keys].min(axis=1)
        lead_ranks, orbit_id = np.unique(lead_rank, return_inverse=True)
        leads = order[lead_ranks]
        # projection coefficients phi(M^T g0) += exp(2 pi i g0.t / n) / |g|,
        # summed over the operations in their order
        coef_all = np.zeros(self.nr, dtype=complex)
        for c0 in range(0, len(leads), chunk):
            g0 = G[leads[c0:c0 + chunk]]                                              # [leaders, 3]
            keys = flat(images(g0))
            ph = np.exp(2j * np.pi * (t[None, :, :] * g0[:, None, :] / nvec[None, None, :]).sum(axis=2))
            np.add.at(coef_all, keys.ravel(), ph.ravel())
        coef_all /= nops
        # stars: wave indices (ascending), normalised coefficients, |G|^2 of
        # the leader; stars whose projection vanishes are dropped
        by_orbit = np.lexsort((np.arange(self.nr), orbit_id))
        starts = np.searchsorted(orbit_id[by_orbit], np.arange(len(leads) + 1))
        orb_idx, orb_coef, orb_gsq = [], [], []
        orbit_of = np.full(self.nr, -1, dtype=np.int64)
        pos_in_orbit = np.empty(self.nr, dtype=np.int64)
        pos_in_orbit[by_orbit] = np.arange(self.nr) - starts[orbit_id[by_orbit]]
        neg_of = flat((-G) % nvec)                                           # flat index of -G
        # a sequential sum of the non-negative |c|^2 is within 1e-12 (relative)
        # of the pairwise np.sum below, so it settles every orbit away from
        # the cancellation threshold; the others get the exact test
        seq = np.add.reduceat(np.abs(coef_all[by_orbit]) ** 2, starts[:-1])
        for o in np.nonzero(seq >= 1e-20 * (1.0 - 1e-12))[0]:
            uniq = by_orbit[starts[o]:starts[o + 1]]
            coef = coef_all[uniq]
            nrm = np.sum(np.abs(coef) ** 2)
            if nrm < 1e-20:
                continue                                                     # cancelled star
            orbit_of[uniq] = len(orb_idx)
            orb_idx.append(uniq)
            orb_coef.append(coef / np.sqrt(nrm))
            orb_gsq.append(float(gsq[leads[o]]))
        # inverse partner of every star (itself when closed under inversion)
        partner = [int(x) for x in orbit_of[neg_of[np.array([idx[0] for idx in orb_idx], dtype=np.int64)]]] \
            if orb_idx else []
        self.orbit_idx, self.orbit_coef, self.orbit_partner = orb_idx, orb_coef, partner
        # real basis functions
        self.star_idx: List[np.ndarray] = []
        self.star_coef: List[np.ndarray] = []
        self.star_gsq: List[float] = []
        self.star_invert: List[int] = []
        self.star_orbit: List[int] = []
        for o, (idx, c) in enumerate(zip(orb_idx, orb_coef)):
            p = partner[o]
            if p == o:
                # phi(-G) = +- conj phi(G): real (cosine-like) or i x real
                j = pos_in_orbit[neg_of[idx]]
                odd = np.sum(np.abs(c + np.conj(c[j])) ** 2) < np.sum(np.abs(c - np.conj(c[j])) ** 2)
                self.star_idx.append(idx)
                self.star_coef.append(-1j * c if odd else c)
                self.star_gsq.append(orb_gsq[o])
                self.star_invert.append(0)
                self.star_orbit.append(o)
            elif p > o:
                # the pair (o, p): conj phi on the inverse waves of p
                both = np.concatenate([idx, neg_of[idx]])
                r2 = np.sqrt(2.0)
                self.star_idx += [both, both]
                self.star_coef += [np.concatenate([c, np.conj(c)]) / r2,
                                   np.concatenate([c, -np.conj(c)]) / (1j * r2)]
                self.star_gsq += [orb_gsq[o], orb_gsq[o]]
                self.star_invert += [1, -1]
                self.star_orbit += [o, p]
        self.n_star = len(self.star_idx)

    def half_grid_tables(self):
        """The waves of every basis function that lie in the r2c half grid
        (0 <= kx <= n1/2): their flat half-grid index kx + (n1/2+1)(ky + n2 kz),
        basis-function index and coefficient -- the device tables of
        pscfg_set_basis.  Every function is real (the partner -G of each of
        its waves is in its wave set with the conjugate coefficient); a wave
        belongs to two functions for the pairs of stars related by
        inversion."""
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
                    raise ValueError(f"basis function {s} is not real")
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
