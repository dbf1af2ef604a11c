"""Host-side description of one SCFT system (the reference's module globals).

The reference keeps the physical system in module globals read by the hot
path: monomers and chains (src/chemistry_mod.f90:41-46), the grid
(src/grid_mod.f90:43-46) and the unit cell (src/unit_cell_mod.f90).  Here it
is one plain object, converted to the flat C struct ``pscfg_system`` that the
C-ABI takes (include/pscf_gpu.h).

Conventions kept from the reference:
  * grid fields are stored x fastest (Fortran column-major): a numpy array of
    shape (n3, n2, n1) in C order, or flat length n1*n2*n3;
  * unused dimensions have extent 1 (src/grid_mod.f90:84-93);
  * monomer indices are 0-based here (1-based in the Fortran input files).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

MAX_MONOMER = 4
MAX_CHAIN = 4
MAX_BLOCK = 8
MAX_SOLVENT = 4
MAX_CELL_PARAM = 6

# Crystal systems (src/unit_cell_mod.f90:309-664) and their integer codes in
# the C-ABI.
CRYSTAL_CODES = {
    (1, "lamellar"): 0,
    (2, "square"): 10,
    (2, "rectangular"): 11,
    (2, "hexagonal"): 12,
    (2, "oblique"): 13,
    (3, "cubic"): 20,
    (3, "tetragonal"): 21,
    (3, "orthorhombic"): 22,
    (3, "hexagonal"): 23,
    (3, "monoclinic"): 24,
}


def chain_grid(block_length: Sequence[float], ds: float):
    """Contour discretisation of one chain (src/chain_mod.f90:136-158).

    Each block gets an even number of steps 2*int(L/ds/2+0.5) (at least 2)
    so that Simpson's rule applies per block.  Returns (block_bgn, block_ds)
    with block_bgn 0-based slice indices of length nblk+1: block i spans
    slices block_bgn[i] .. block_bgn[i+1] inclusive.
    """
    bgn = [0]
    bds = []
    for L in block_length:
        iblk = int(L / ds / 2.0 + 0.5)
        if iblk == 0:
            iblk = 1
            bds.append(L / 2.0)
        else:
            bds.append(L / float(iblk) / 2.0)
        bgn.append(bgn[-1] + 2 * iblk)
    return bgn, bds


def make_unit_cell(dim: int, crystal_system: str, cell_param: Sequence[float]):
    """Reciprocal basis and its cell-parameter derivatives.

    Follows make_unit_cell / make_G_basis (src/unit_cell_mod.f90:309-664,
    723-757): G_basis = 2 pi inverse(R_basis)^T (row i is reciprocal vector
    b_i), dG_basis(i,j,k) = -sum_lm G(i,l) dR(m,l,k) G(m,j) / 2 pi and
    dGG(k,i,j) = d(b_i . b_j)/d(cell_param k).

    Returns (G_basis[3,3], dGG[ncp,3,3], ncp); unused rows/cols are zero.
    """
    key = (dim, crystal_system)
    if key not in CRYSTAL_CODES:
        raise ValueError(f"unknown crystal system {crystal_system!r} for dim={dim}")
    cp = [float(c) for c in cell_param]
    R = np.zeros((3, 3))
    dR = np.zeros((3, 3, MAX_CELL_PARAM))
    s75 = math.sqrt(0.75)
    if crystal_system == "lamellar":
        ncp = 1
        R[0, 0] = cp[0]
        dR[0, 0, 0] = 1.0
    elif crystal_system == "square":
        ncp = 1
        R[0, 0] = R[1, 1] = cp[0]
        dR[0, 0, 0] = dR[1, 1, 0] = 1.0
    elif crystal_system == "rectangular":
        ncp = 2
        R[0, 0], R[1, 1] = cp[0], cp[1]
        dR[0, 0, 0] = dR[1, 1, 1] = 1.0
    elif crystal_system == "hexagonal" and dim == 2:
        ncp = 1
        R[0, 0] = cp[0]
        R[1, 0] = -0.5 * cp[0]
        R[1, 1] = cp[0] * s75
        dR[0, 0, 0], dR[1, 0, 0], dR[1, 1, 0] = 1.0, -0.5, s75
    elif crystal_system == "oblique":
        # dR(1,1,1) = a exactly as written in src/unit_cell_mod.f90:630
        ncp = 3
        a, b, g = cp[0], cp[1], cp[2]
        R[0, 0] = a
        R[1, 0], R[1, 1] = b * math.cos(g), b * math.sin(g)
        dR[0, 0, 0] = a
        dR[1, 0, 1], dR[1, 1, 1] = math.cos(g), math.sin(g)
        dR[1, 0, 2], dR[1, 1, 2] = -b * math.sin(g), b * math.cos(g)
    elif crystal_system == "cubic":
        ncp = 1
        R[0, 0] = R[1, 1] = R[2, 2] = cp[0]
        dR[0, 0, 0] = dR[1, 1, 0] = dR[2, 2, 0] = 1.0
    elif crystal_system == "tetragonal":
        ncp = 2
        R[0, 0] = R[1, 1] = cp[0]
        R[2, 2] = cp[1]
        dR[0, 0, 0] = dR[1, 1, 0] = 1.0
        dR[2, 2, 1] = 1.0
    elif crystal_system == "orthorhombic":
        ncp = 3
        R[0, 0], R[1, 1], R[2, 2] = cp[0], cp[1], cp[2]
        dR[0, 0, 0] = dR[1, 1, 1] = dR[2, 2, 2] = 1.0
    elif crystal_system == "hexagonal" and dim == 3:
        ncp = 2
        R[0, 0] = cp[0]
        R[1, 0] = -0.5 * cp[0]
        R[1, 1] = cp[0] * s75
        R[2, 2] = cp[1]
        dR[0, 0, 0], dR[1, 0, 0], dR[1, 1, 0] = 1.0, -0.5, s75
        dR[2, 2, 1] = 1.0
    elif crystal_system == "monoclinic":
        ncp = 4
        a, b, c, beta = cp[:4]
        R[0, 0], R[1, 1] = a, b
        R[2, 0], R[2, 2] = c * math.cos(beta), c * math.sin(beta)
        dR[0, 0, 0] = dR[1, 1, 1] = 1.0
        dR[2, 0, 2], dR[2, 2, 2] = math.cos(beta), math.sin(beta)
        dR[2, 0, 3], dR[2, 2, 3] = -c * math.sin(beta), c * math.cos(beta)
    else:  # pragma: no cover - guarded by CRYSTAL_CODES
        raise ValueError(crystal_system)
    twopi = 4.0 * math.acos(0.0)
    Rl = np.eye(3)
    Rl[:dim, :dim] = R[:dim, :dim]
    G = np.zeros((3, 3))
    G[:dim, :dim] = (twopi * np.linalg.inv(Rl).T)[:dim, :dim]
    dG = np.zeros((3, 3, MAX_CELL_PARAM))
    for k in range(ncp):
        dG[:dim, :dim, k] = -(G[:dim, :dim] @ dR[:dim, :dim, k].T @ G[:dim, :dim]) / twopi
    dGG = np.zeros((ncp, 3, 3))
    for k in range(ncp):
        M = G[:dim, :dim] @ dG[:dim, :dim, k].T
        dGG[k, :dim, :dim] = M + M.T
    return G, dGG, ncp


@dataclasses.dataclass
class Chain:
    block_monomer: List[int]          # 0-based monomer index per block
    block_length: List[float]
    phi: float = 1.0
    mu: float = 0.0

    @property
    def length(self) -> float:
        return float(sum(self.block_length))


@dataclasses.dataclass
class Solvent:
    monomer: int
    size: float
    phi: float = 0.0
    mu: float = 0.0


@dataclasses.dataclass
class System:
    """One SCFT system: chemistry, grid, discretisation and unit cell."""
    dim: int
    ngrid: Sequence[int]
    crystal_system: str
    cell_param: List[float]
    kuhn: List[float]
    chi: np.ndarray
    chains: List[Chain]
    ds: float
    solvents: List[Solvent] = dataclasses.field(default_factory=list)
    ensemble: int = 0
    # interaction_type 'chi_T' (src/chemistry_mod.f90): chi = chi_A / T + chi_B,
    # with chi computed from these when temperature is set
    chi_A: Optional[np.ndarray] = None
    chi_B: Optional[np.ndarray] = None
    temperature: Optional[float] = None

    def __post_init__(self):
        if self.temperature is not None:
            self.chi_A = np.asarray(self.chi_A, dtype=np.float64)
            self.chi_B = np.asarray(self.chi_B, dtype=np.float64)
            self.chi = self.chi_A / float(self.temperature) + self.chi_B
        self.chi = np.asarray(self.chi, dtype=np.float64)
        self.cell_param = [float(c) for c in self.cell_param]
        if not (1 <= self.dim <= 3):
            raise ValueError("dim must be 1, 2 or 3")
        if len(self.ngrid) != self.dim:
            raise ValueError("ngrid must have dim entries")
        if len(self.kuhn) > MAX_MONOMER or len(self.chains) > MAX_CHAIN:
            raise ValueError("too many monomers or chains")
        if any(len(c.block_length) > MAX_BLOCK for c in self.chains):
            raise ValueError("too many blocks")
        if self.chi.shape != (len(self.kuhn), len(self.kuhn)):
            raise ValueError("chi must be n_monomer x n_monomer")

    @property
    def n_monomer(self) -> int:
        return len(self.kuhn)

    @property
    def n(self):
        n = list(self.ngrid) + [1] * (3 - self.dim)
        return tuple(int(v) for v in n)

    @property
    def nr(self) -> int:
        n = self.n
        return n[0] * n[1] * n[2]

    @property
    def nk(self) -> int:
        n = self.n
        return (n[0] // 2 + 1) * n[1] * n[2]

    def unit_cell(self, cell_param: Optional[Sequence[float]] = None):
        return make_unit_cell(self.dim, self.crystal_system,
                              self.cell_param if cell_param is None else cell_param)

    @property
    def crystal_code(self) -> int:
        return CRYSTAL_CODES[(self.dim, self.crystal_system)]

    def phi_monomer(self) -> np.ndarray:
        """Average volume fraction of each monomer type
        (src/scf_mod.fp.f90:732-745)."""
        phi = np.zeros(self.n_monomer)
        for c in self.chains:
            for m, L in zip(c.block_monomer, c.block_length):
                phi[m] += c.phi * L / c.length
        for s in self.solvents:
            phi[s.monomer] += s.phi
        return phi

    def omega_uniform(self) -> np.ndarray:
        """k=0 component of omega (set_omega_uniform, src/scf_mod.fp.f90:724-750)."""
        return self.chi @ self.phi_monomer()

    def contour_steps(self) -> int:
        """Total MDE steps of one sweep summed over chains (one direction)."""
        return sum(chain_grid(c.block_length, self.ds)[0][-1] for c in self.chains)
