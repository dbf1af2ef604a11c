"""Field files in the reference's formats (src/field_io_mod.f90).

Basis format (input_field / output_field, :55-135): a header
  format 1 0 / dim / crystal_system / N_cell_param / cell_param /
  group_name / N_monomer / N_star
then one line per star: the N_monomer coefficients (ES20.12), the star's
first wave G (I4 each, in first-Brillouin-zone form) and the number of
waves in the star (I6).  A reader finds the star by its wave, so the line
order does not matter (input_field :71-79).  The reference's star function
is sum_G c_G exp(iG.r) with the coefficient of the star's wave real and
positive, 1/sqrt(N) with sqrt taken in single precision
(src/basis_mod.f90:916-936); the waves of a star are ordered by G_lt
(components compared in turn, :1576-1620) and the star's wave is the first
(largest) one.  A star closed under inversion is one real basis function,
its coefficients multiplied by -i when the function is odd (sine-like,
:1160-1192).  In a group without inversion two stars related by inversion
form a pair (star_invert = +1, -1): the +1 star is the one holding the
larger wave, the -1 star's wave is its last one (the inverse of the +1
star's wave) and its coefficients are real and positive there; their
coefficients a, b weigh the waves as (a -+ i b) c_G / sqrt(2)
(basis_to_kgrid / kgrid_to_basis, src/grid_basis_mod.f90:47-200).

Grid format (output_field_grid :151-200, read back by RGRID_TO_FIELD,
src/pscf.fp.f90:890-980): the same header up to N_monomer, then ngrid and
the values at every grid point, x fastest, N_monomer values (F18.9) per
line.

Fields are handled here as grid arrays [n_monomer][nr] (x fastest), the
engine's representation; the star coefficients are computed from them by
FFT.
"""
from __future__ import annotations

import threading
from collections import OrderedDict
from typing import Dict, List, Sequence, Tuple

import numpy as np

from .basis import StarBasis
from .system import make_unit_cell


def _fl32_sqrt(n: int) -> float:
    return float(np.sqrt(np.float32(n)))


def _label(name: str) -> str:
    return f"{name:<20}"


def _header(cell: Dict, group_name: str, n_monomer: int) -> List[str]:
    cp = list(cell["cell_param"])
    return [" format  1  0",
            _label("dim"), f"{cell['dim']:>20d}",
            _label("crystal_system"), f"{chr(39) + cell['crystal_system'] + chr(39):>20}",
            _label("N_cell_param"), f"{len(cp):>20d}",
            _label("cell_param"), "".join(f"{v:20.10E}" for v in cp),
            _label("group_name"), f"{chr(39) + group_name + chr(39):>20}",
            _label("N_monomer"), f"{n_monomer:>20d}"]


def _read_header(lines: List[str]) -> Tuple[Dict, int]:
    """Parse 'name / value' pairs after the version line; returns the
    header and the index of the first unread line."""
    h: Dict = {}
    i = 1
    keys = ("dim", "crystal_system", "N_cell_param", "cell_param", "group_name", "N_monomer")
    for k in keys:
        assert lines[i].split()[0] == k, f"expected {k!r} in field file header, got {lines[i]!r}"
        val = lines[i + 1].split()
        i += 2
        if k in ("dim", "N_cell_param", "N_monomer"):
            h[k] = int(val[0])
        elif k == "cell_param":
            h[k] = [float(v.replace("D", "E")) for v in val]
        else:
            h[k] = " ".join(val).strip("'\"")
    return h, i


def _g_to_bz(G: np.ndarray, n: Sequence[int], Gb: np.ndarray, dim: int) -> np.ndarray:
    """Minimum image of integer waves, images +1, 0, -1 per dimension in
    that order, a later one winning only if shorter by more than 1e-8
    (G_to_bz, src/grid_mod.f90:225-283).  G: [k, 3]."""
    best = np.zeros_like(G)
    gmin = np.full(len(G), 1.0e10)
    rng = [(1, 0, -1) if a < dim else (0,) for a in range(3)]
    for s1 in rng[0]:
        for s2 in rng[1]:
            for s3 in rng[2]:
                t = G + np.array([s1 * n[0], s2 * n[1], s3 * n[2]])
                v = t[:, :dim] @ Gb[:dim, :dim]
                q = (v * v).sum(axis=1)
                win = q < gmin - 1.0e-8
                best[win] = t[win]
                gmin[win] = q[win]
    return best


def _grid_waves(idx: np.ndarray, n: Sequence[int]) -> np.ndarray:
    return np.stack([idx % n[0], (idx // n[0]) % n[1], idx // (n[0] * n[1])], axis=1)


def _spectrum(field: np.ndarray, n: Sequence[int]) -> np.ndarray:
    """F(G) = (1/N) sum_r f(r) exp(-iG.r), flat x fastest."""
    nr = int(np.prod(n))
    return (np.fft.fftn(field.reshape(n[2], n[1], n[0])) / nr).ravel()


_STAR_BASES: "OrderedDict[Tuple, StarBasis]" = OrderedDict()
_FIELD_BASES: "OrderedDict[Tuple, FieldBasis]" = OrderedDict()


_CACHE_LOCK = threading.Lock()


def _cached(cache: OrderedDict, key: Tuple, make, keep: int):
    """cache[key], made by make() when missing; the least recently used
    entries beyond `keep` are dropped.  Safe across host threads (the
    bases are read-only once made)."""
    with _CACHE_LOCK:
        obj = cache.pop(key, None)
        if obj is not None:
            cache[key] = obj
            return obj
    obj = make()
    with _CACHE_LOCK:
        obj = cache.pop(key, obj)          # another thread may have made it meanwhile
        cache[key] = obj
        while len(cache) > keep:
            cache.popitem(last=False)
    return obj


def star_basis(group_name: str, ngrid: Sequence[int]) -> StarBasis:
    """StarBasis(group_name, ngrid) for the file conventions, kept for the
    last few (group, grid) pairs: it does not depend on the cell, so the
    points of a sweep share it."""
    key = (group_name, tuple(int(x) for x in ngrid))
    return _cached(_STAR_BASES, key, lambda: StarBasis(group_name, ngrid), 4)


def field_basis(group_name: str, system) -> "FieldBasis":
    """FieldBasis(group_name, system), kept for the last two (group, grid,
    cell) triples (a field file's omega and rho are written with the same
    one)."""
    key = (group_name, system.dim, tuple(int(x) for x in system.ngrid), system.crystal_system,
           tuple(float(c) for c in system.cell_param))
    return _cached(_FIELD_BASES, key, lambda: FieldBasis(group_name, system), 2)


class FieldBasis:
    """Star basis of a group on a grid with the reference's file
    conventions (star waves, coefficient phases and normalisation, the
    +1 / -1 pairs of a group without inversion), in the line order of
    StarBasis.  stars[k]: dict(idx = flat waves, cref = their coefficients,
    kind = 0 (closed), 1 or -1, wave = flat index of the star's wave,
    wave_bz = its first-zone form, count)."""

    def __init__(self, group_name: str, system):
        self.group = group_name
        self.dim = system.dim
        self.n = list(system.n)
        self.nr = system.nr
        self.basis = star_basis(group_name, system.ngrid)
        self.Gb = make_unit_cell(system.dim, system.crystal_system, system.cell_param)[0]
        b = self.basis
        # first-zone forms of every orbit's waves, in one pass over all of them
        self._bz_off = np.concatenate([[0], np.cumsum([len(i) for i in b.orbit_idx])])
        all_idx = np.concatenate([np.asarray(i) for i in b.orbit_idx])
        self._bz_all = _g_to_bz(_grid_waves(all_idx, self.n), self.n, self.Gb, self.dim)
        self.stars: List[Dict] = []
        done = set()
        for s in range(b.n_star):
            o = b.star_orbit[s]
            if o in done:
                continue
            p = b.orbit_partner[o]
            if p == o:
                self.stars.append(self._closed(o))
                done.add(o)
            else:
                self.stars += self._pair(o, p)
                done |= {o, p}
        self.star_of = {}
        for k, st in enumerate(self.stars):
            for i in st["idx"]:
                self.star_of[int(i)] = k
        # first-zone waves and counts of the file lines
        self.first = [st["wave"] for st in self.stars]
        self.first_bz = [st["wave_bz"] for st in self.stars]
        self.count = [st["count"] for st in self.stars]

    def _sorted(self, o):
        """Waves of star o in G_lt order (largest first), their first-zone forms."""
        idx = np.asarray(self.basis.orbit_idx[o])
        bz = self._bz_all[self._bz_off[o]:self._bz_off[o + 1]]
        order = sorted(range(len(idx)), key=lambda j: tuple(bz[j][:self.dim]), reverse=True)
        return idx, bz, order

    def _flat(self, g):
        n = self.n
        g = np.asarray(g) % np.array(n)
        return int(g[0] + n[0] * (g[1] + n[1] * g[2]))

    def _closed(self, o):
        idx, bz, order = self._sorted(o)
        c = np.asarray(self.basis.orbit_coef[o])
        j0 = order[0]
        g0 = _grid_waves(idx[j0:j0 + 1], self.n)[0]
        jm = int(np.nonzero(idx == self._flat(-g0))[0][0])
        ratio = c[jm] / c[j0]
        if abs(ratio - 1) < 1e-8:
            phase = 1.0
        elif abs(ratio + 1) < 1e-8:
            phase = -1j                                    # sine-like closed star
        else:
            raise ValueError(f"closed star {o} is neither cosine- nor sine-like")
        cref = c / c[j0] / _fl32_sqrt(len(idx)) * phase
        return dict(idx=idx, cref=cref, kind=0, wave=int(idx[j0]), wave_pos=j0,
                    wave_bz=bz[j0][:self.dim].astype(int), count=len(idx))

    def _pair(self, o, p):
        so, sp = self._sorted(o), self._sorted(p)
        first = lambda srt: tuple(srt[1][srt[2][0]][:self.dim])
        (ip, bzp, ordp), (im, bzm, ordm) = (so, sp) if first(so) > first(sp) else (sp, so)
        op, om = (o, p) if first(so) > first(sp) else (p, o)
        j0 = ordp[0]
        jl = ordm[-1]
        g0 = _grid_waves(ip[j0:j0 + 1], self.n)[0]
        if int(im[jl]) != self._flat(-g0):
            raise ValueError(f"stars {op}, {om}: the last wave of the -1 star is not the inverse of the +1 star's wave")
        cp = np.asarray(self.basis.orbit_coef[op])
        cm = np.asarray(self.basis.orbit_coef[om])
        plus = dict(idx=ip, cref=cp / cp[j0] / _fl32_sqrt(len(ip)), kind=1, wave=int(ip[j0]), wave_pos=j0,
                    wave_bz=bzp[j0][:self.dim].astype(int), count=len(ip))
        minus = dict(idx=im, cref=cm / cm[jl] / _fl32_sqrt(len(im)), kind=-1, wave=int(im[jl]), wave_pos=jl,
                     wave_bz=bzm[jl][:self.dim].astype(int), count=len(im))
        return [plus, minus]

    def to_coeffs(self, field: np.ndarray) -> np.ndarray:
        """Reference basis coefficients [n_star] of a grid field
        (kgrid_to_basis)."""
        return self.spectrum_to_coeffs(_spectrum(np.asarray(field, dtype=np.float64), self.n))

    def spectrum_to_coeffs(self, F: np.ndarray) -> np.ndarray:
        """Reference basis coefficients [n_star] of Fourier components F(G)
        over the full grid (flat, x fastest): each star's coefficient is
        read from its own wave alone (kgrid_to_basis,
        src/grid_basis_mod.f90:146-200)."""
        out = np.zeros(len(self.stars))
        r2 = np.sqrt(2.0)
        for k, st in enumerate(self.stars):
            z = F[st["wave"]] / st["cref"][st["wave_pos"]]
            out[k] = z.real if st["kind"] == 0 else (r2 * z.real if st["kind"] == 1 else r2 * z.imag)
        return out

    def to_grid(self, coeffs: Sequence[float]) -> np.ndarray:
        """Grid field of the reference's basis coefficients (basis_to_kgrid)."""
        F = np.zeros(self.nr, dtype=complex)
        r2 = np.sqrt(2.0)
        for k, st in enumerate(self.stars):
            if st["kind"] == 0:
                z = coeffs[k]
            elif st["kind"] == 1:
                z = complex(coeffs[k], -coeffs[k + 1]) / r2
            else:
                z = complex(coeffs[k - 1], coeffs[k]) / r2
            F[st["idx"]] += z * st["cref"]
        n = self.n
        f = np.fft.ifftn(F.reshape(n[2], n[1], n[0])) * self.nr
        return np.real(f).ravel()


def write_field(path: str, fields: np.ndarray, system, group_name: str) -> None:
    """Basis-format file of grid fields [n_monomer][nr] (output_field)."""
    fb = field_basis(group_name, system)
    fields = np.asarray(fields, dtype=np.float64).reshape(-1, system.nr)
    write_coeffs(path, np.stack([fb.to_coeffs(f) for f in fields]), system, group_name, fb)


def write_coeffs(path: str, coeffs: np.ndarray, system, group_name: str, fb: "FieldBasis" = None) -> None:
    """Basis-format file of coefficients [n_monomer][n] of the first n stars
    of the group's basis (output_field with N_basis_out = n,
    src/field_io_mod.f90:101-135)."""
    fb = fb or field_basis(group_name, system)
    coeffs = np.atleast_2d(np.asarray(coeffs, dtype=np.float64))
    if coeffs.shape[1] > len(fb.stars):
        raise ValueError(f"{coeffs.shape[1]} coefficients for a basis of {len(fb.stars)} stars")
    cell = {"dim": system.dim, "crystal_system": system.crystal_system, "cell_param": system.cell_param}
    out = _header(cell, group_name, len(coeffs))
    out += [_label("N_star"), f"{coeffs.shape[1]:>20d}"]
    for s in range(coeffs.shape[1]):
        line = "".join(f"{a:20.12E}" for a in coeffs[:, s]) + "    "
        line += "".join(f"{g:4d}" for g in fb.first_bz[s]) + f"{fb.count[s]:6d}"
        out.append(line)
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def read_field(path: str, system, group_name: str = None) -> Tuple[Dict, np.ndarray]:
    """(header, grid fields [n_monomer][nr]) of a basis-format file
    (input_field).  `system` gives the grid; the group is the file's unless
    given.  A star count in the file that differs from the basis rescales
    its coefficient by sqrt(N_file / N_basis), as input_field does."""
    lines = open(path).read().splitlines()
    h, i = _read_header(lines)
    assert lines[i].split()[0] == "N_star"
    nstar = int(lines[i + 1].split()[0])
    M = h["N_monomer"]
    fb = field_basis(group_name or h["group_name"], system)
    coeffs = np.zeros((M, len(fb.stars)))
    n = np.array(system.n)
    for line in lines[i + 2:i + 2 + nstar]:
        v = line.split()
        a = np.array([float(x.replace("D", "E")) for x in v[:M]])
        g = np.zeros(3, dtype=int)
        g[:system.dim] = [int(x) for x in v[M:M + system.dim]]
        n_arm = int(v[M + system.dim])
        gi = g % n
        flat = int(gi[0] + n[0] * (gi[1] + n[1] * gi[2]))
        s = fb.star_of.get(flat)
        if s is None:
            continue                      # a wave with no star on this grid (valid_wave false)
        coeffs[:, s] = a * np.sqrt(n_arm / fb.count[s])
    fields = np.stack([fb.to_grid(coeffs[m]) for m in range(M)])
    return h, fields


def write_rgrid(path: str, fields: np.ndarray, system, group_name: str) -> None:
    """Grid-format file (output_field_grid)."""
    fields = np.asarray(fields, dtype=np.float64).reshape(-1, system.nr)
    cell = {"dim": system.dim, "crystal_system": system.crystal_system, "cell_param": system.cell_param}
    out = _header(cell, group_name, len(fields))
    out += [_label("ngrid"), "".join(f"{g:20d}" for g in system.ngrid)]
    for r in range(system.nr):
        out.append("".join(f"{fields[m, r]:18.9f}" for m in range(len(fields))) + "    ")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def write_kgrid(path: str, fields: np.ndarray, system, group_name: str) -> None:
    """Wave-grid file of grid fields [n_monomer][nr]: the grid-format header,
    then the Fourier components F(G) = (1/N) sum_r f(r) exp(-iG.r) on the
    half grid 0 <= G1 <= n1/2, G3 fastest and G1 slowest, one line of
    n_monomer complex values '(re,im)' per wave -- the file that
    KGRID_TO_RGRID reads (src/pscf.fp.f90:813-888)."""
    fields = np.asarray(fields, dtype=np.float64).reshape(-1, system.nr)
    n = list(system.n)
    spec = [_spectrum(f, n).reshape(n[2], n[1], n[0]) for f in fields]
    cell = {"dim": system.dim, "crystal_system": system.crystal_system, "cell_param": system.cell_param}
    out = _header(cell, group_name, len(fields))
    out += [_label("ngrid"), "".join(f"{g:20d}" for g in system.ngrid)]
    for i1 in range(n[0] // 2 + 1):
        for i2 in range(n[1]):
            for i3 in range(n[2]):
                out.append("  ".join(f"({z[i3, i2, i1].real:.16E},{z[i3, i2, i1].imag:.16E})" for z in spec))
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def read_kgrid(path: str, system) -> Tuple[Dict, np.ndarray]:
    """(header, Fourier components [n_monomer][nr] over the full grid, flat
    x fastest) of a wave-grid file (KGRID_TO_RGRID,
    src/pscf.fp.f90:813-888).  The file holds the half grid
    0 <= G1 <= n1/2 with G3 fastest, n_monomer complex values per wave in
    list-directed form ('(re,im)', or two plain numbers); the other half
    is F(-G) = conj F(G).  A grid that differs from the system's raises
    ValueError, as the reference stops there."""
    import re
    lines = open(path).read().splitlines()
    h, i = _read_header(lines)
    if lines[i].split()[0] != "ngrid":
        raise ValueError(f"{path}: expected 'ngrid', got {lines[i]!r}")
    g = [int(x) for x in lines[i + 1].split()]
    if g[:system.dim] != list(system.ngrid)[:system.dim]:
        raise ValueError(f"{path}: inconsistent grid {g} in the wave-grid file (system grid {list(system.ngrid)})")
    M = h["N_monomer"]
    n = list(system.n)
    n1h = n[0] // 2 + 1
    text = "\n".join(lines[i + 2:]).replace("D", "E").replace("d", "e")
    pairs = re.findall(r"\(\s*([^,()\s]+)\s*,\s*([^,()\s]+)\s*\)", text)
    if pairs:
        vals = np.array([complex(float(a), float(b)) for a, b in pairs])
    else:
        v = np.array([float(x) for x in text.split()])
        vals = v[0::2] + 1j * v[1::2]
    need = n1h * n[1] * n[2] * M
    if len(vals) < need:
        raise ValueError(f"{path}: {len(vals)} values, {need} expected")
    half = vals[:need].reshape(n1h, n[1], n[2], M)                     # [G1][G2][G3][monomer]
    out = np.zeros((M, n[2], n[1], n[0]), dtype=complex)
    out[:, :, :, :n1h] = half.transpose(3, 2, 1, 0)
    for x in range(n1h, n[0]):
        # F(x, y, z) = conj F(-x, -y, -z), with -x in the half grid
        src = out[:, :, :, (-x) % n[0]]
        out[:, :, :, x] = np.conj(src[:, (-np.arange(n[2])) % n[2]][:, :, (-np.arange(n[1])) % n[1]])
    return h, out.reshape(M, -1)


def read_rgrid(path: str) -> Tuple[Dict, List[int], np.ndarray]:
    """(header, ngrid, grid fields [n_monomer][nr]) of a grid-format file."""
    lines = open(path).read().splitlines()
    h, i = _read_header(lines)
    assert lines[i].split()[0] == "ngrid"
    ngrid = [int(x) for x in lines[i + 1].split()]
    nr = int(np.prod(ngrid))
    vals = np.array([[float(x) for x in ln.split()] for ln in lines[i + 2:i + 2 + nr]])
    return h, ngrid, vals.T.copy()
