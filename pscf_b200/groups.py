"""Space groups used by the symmetric (star-basis) fields of the reference.

The reference restricts omega and rho to a symmetry-adapted basis of a
space group (src/basis_mod.f90, src/grid_basis_mod.f90:47-200), reading the
group elements from tables (src/space_groups_mod.f90).  The engine keeps
fields on the FFT grid instead and imposes the same symmetry by projecting
a field onto the group-invariant subspace (the average over the orbit
x -> m x + v of every grid point), which spans the same fields as the
star basis.

Each group here is built as the closure of International Tables generators,
in the settings the reference uses (x' = m x + v in fractional
coordinates, src/group_mod.f90:69-80, mat_dot_vec :718-730).
"""
from __future__ import annotations

import itertools
from fractions import Fraction as Fr
from typing import Dict, List, Sequence, Tuple

import numpy as np

Op = Tuple[Tuple[Tuple[int, ...], ...], Tuple[Fr, ...]]


def _op(m, v) -> Op:
    return (tuple(tuple(int(x) for x in row) for row in m), tuple(Fr(x) % 1 for x in v))


def _mul(a: Op, b: Op) -> Op:
    """a after b: x -> ma (mb x + vb) + va."""
    ma, va = a
    mb, vb = b
    d = len(ma)
    m = tuple(tuple(sum(ma[i][k] * mb[k][j] for k in range(d)) for j in range(d)) for i in range(d))
    v = tuple((sum(ma[i][k] * vb[k] for k in range(d)) + va[i]) % 1 for i in range(d))
    return (m, v)


def closure(gens: Sequence[Op]) -> List[Op]:
    d = len(gens[0][0])
    ident = _op(np.eye(d, dtype=int), [0] * d)
    elems = {ident}
    frontier = [ident]
    while frontier:
        new = []
        for x in frontier:
            for g in gens:
                y = _mul(g, x)
                if y not in elems:
                    elems.add(y)
                    new.append(y)
        frontier = new
        if len(elems) > 1000:
            raise RuntimeError("group closure did not terminate")
    return sorted(elems)


def _parse(expr: str, d: int) -> Op:
    """'-x+1/2,-y,z+1/2' -> (m, v)."""
    names = "xyz"[:d]
    m = np.zeros((d, d), dtype=int)
    v = [Fr(0)] * d
    for i, comp in enumerate(expr.replace(" ", "").split(",")):
        tok = ""
        terms = []
        for ch in comp:
            if ch in "+-" and tok:
                terms.append(tok)
                tok = ch
            else:
                tok += ch
        terms.append(tok)
        for t in terms:
            sign = -1 if t.startswith("-") else 1
            body = t.lstrip("+-")
            if body in names:
                m[i, names.index(body)] += sign
            else:
                v[i] += sign * Fr(body)
    return _op(m, v)


def _from_positions(d: int, gens: Sequence[str]) -> List[Op]:
    return closure([_parse(g, d) for g in gens])


def _signed_permutations() -> List[str]:
    out = []
    for p in itertools.permutations("xyz"):
        for s in itertools.product("+-", repeat=3):
            out.append(",".join(("-" if si == "-" else "") + pi for si, pi in zip(s, p)))
    return out


# Generators (International Tables for Crystallography, Vol. A).
_GENERATORS: Dict[str, Tuple[int, List[str]]] = {
    "1": (1, ["x"]),
    "-1": (1, ["-x"]),
    "p 1": (2, ["x,y"]),
    "p 2": (2, ["-x,-y"]),
    "P 1": (3, ["x,y,z"]),
    "P -1": (3, ["-x,-y,-z"]),
    "p 6 m m": (2, ["x-y,x", "-y,-x"]),
    "I m -3 m": (3, _signed_permutations() + ["x+1/2,y+1/2,z+1/2"]),
    "I a -3 d": (3, ["-x+1/2,-y,z+1/2", "-x,y+1/2,-z+1/2", "z,x,y", "y+3/4,x+1/4,-z+1/4",
                     "-x,-y,-z", "x+1/2,y+1/2,z+1/2"]),
    "F d d d : 2": (3, ["-x+3/4,-y+3/4,z", "-x+3/4,y,-z+3/4", "-x,-y,-z",
                        "x,y+1/2,z+1/2", "x+1/2,y,z+1/2", "x+1/2,y+1/2,z"]),
    # no inversion: the alternating gyroid of ABC triblocks (stars in pairs
    # related by inversion, star_invert = +-1)
    "I 41 3 2": (3, ["-x+1/2,-y,z+1/2", "-x,y+1/2,-z+1/2", "z,x,y", "y+3/4,x+1/4,-z+1/4",
                     "x+1/2,y+1/2,z+1/2"]),
}

ALIASES = {"P 6 m m": "p 6 m m", "229": "I m -3 m", "230": "I a -3 d", "70": "F d d d : 2", "17": "p 6 m m",
           "214": "I 41 3 2", "I 4_1 3 2": "I 41 3 2"}
# 1-D names as the reference spells them in 3-D notation (response_startup
# maps 'P 1' to '1' for dim = 1, src/response_mod.f90:227)
ALIASES_1D = {"P 1": "1", "P -1": "-1", "p -1": "-1"}


def resolve(name: str, dim: int = None) -> str:
    if dim == 1 and name in ALIASES_1D:
        return ALIASES_1D[name]
    return ALIASES.get(name, name)


def group(name: str, dim: int = None) -> List[Op]:
    name = resolve(name, dim)
    if name not in _GENERATORS:
        raise KeyError(f"space group {name!r} is not tabulated here")
    d, gens = _GENERATORS[name]
    return _from_positions(d, gens)


def group_names() -> List[str]:
    return list(_GENERATORS)


def grid_ops(name: str, ngrid: Sequence[int]):
    """Integer action of every element on grid indices.

    Returns (M, t): M int32 [nops, 3, 3], t int32 [nops, 3] with
    i' = M i + t (mod n) for grid index vectors i (unused dimensions 0).
    Raises ValueError if the grid is not mapped onto itself (a translation
    not a multiple of 1/n, or a rotation mixing axes of different extent).
    """
    ops = group(name, len(ngrid))
    d = len(ops[0][0])
    if d != len(ngrid):
        raise ValueError(f"group {name!r} is {d}-dimensional, grid is {len(ngrid)}-dimensional")
    n = list(ngrid)
    M = np.zeros((len(ops), 3, 3), dtype=np.int32)
    t = np.zeros((len(ops), 3), dtype=np.int32)
    for k, (m, v) in enumerate(ops):
        for i in range(d):
            for j in range(d):
                if m[i][j] != 0 and n[i] != n[j]:
                    raise ValueError("rotation mixes axes of different grid extent")
                M[k, i, j] = m[i][j]
            tv = v[i] * n[i]
            if tv.denominator != 1:
                raise ValueError(f"translation {v[i]} is not a multiple of 1/{n[i]}")
            t[k, i] = int(tv) % n[i]
    return M, t


def symmetrize(field: np.ndarray, name: str, ngrid: Sequence[int]) -> np.ndarray:
    """Average of f(g x) over the group (numpy; host-side helper)."""
    M, t = grid_ops(name, ngrid)
    n = list(ngrid) + [1] * (3 - len(ngrid))
    f = np.asarray(field, dtype=np.float64).reshape(n[2], n[1], n[0])
    I3, I2, I1 = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
    idx = np.stack([I1, I2, I3])  # [3, n3, n2, n1]
    acc = np.zeros_like(f)
    for k in range(len(M)):
        j = np.einsum("ij,j...->i...", M[k], idx) + t[k][:, None, None, None]
        j = [j[d] % n[d] for d in range(3)]
        acc += f[j[2], j[1], j[0]]
    return (acc / len(M)).ravel()
