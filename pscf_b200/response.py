"""Linear response of a periodic SCFT state (the RESPONSE command).

Mirrors response_mod (src/response_mod.f90):
  * response_sweep (:309-378)       -> response_sweep()
  * drho_domega_id (:389-468)       -> drho_domega_id(): the ideal-gas
    response matrices smm, spm, spp of the two-monomer system in a basis of
    Bloch perturbations exp(ik.r) f_j(r); the per-perturbation propagation
    (calc_q0, calc_delq, calc_delrho) runs on the engine (pscfg_response),
    all perturbations of a k point in one batched call;
  * calc_drho_domega_full (:484-627) -> drho_domega_full(): the response of
    the incompressible melt S = smm - spm^T spp^-1 spm, its eigenvalues
    1/lambda - chi_12 sorted ascending (Shell sort, src/basis_mod.f90:
    1453-1483), the divergent k = 0 eigenvalue dropped.  The dense
    symmetric algebra (LAPACK dsytrf/dsytri/dsyev in the reference) runs on
    the host, as in the reference.
The basis functions are the stars of a subgroup k_group of the little group
of k (pscf_b200.basis.StarBasis): star j is f_j(r) = sum_G c_G e^{iG.r},
perturbation field N * IFFT of those coefficients (calc_perturb_field
:1275-1291), readout Re(drho(G_0)/c_0) at the star's first wave
(kgrid_to_basis with no_parity, src/grid_basis_mod.f90:146-200).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

from .basis import StarBasis
from .engine import Engine

Basis = List[Tuple[np.ndarray, np.ndarray]]


def perturbation_basis(k_group: str, ngrid: Sequence[int]) -> Basis:
    """(grid indices, coefficients) of every star of k_group on the grid."""
    b = StarBasis(k_group, ngrid)
    return [(np.asarray(i), np.asarray(c, dtype=complex)) for i, c in zip(b.star_idx, b.star_coef)]


def transverse_ksq(dim: int, G: np.ndarray, kvec: Sequence[float]) -> float:
    """ktrans_sq of response_sweep for kdim = dim + 1 (src/response_mod.f90:
    347-355): the loop there assigns g_basis(1,i)**2 for i = 1..dim, so the
    value of the last iteration, g_basis(1,dim)**2, times kvec(dim+1)**2
    is what the reference adds."""
    if len(kvec) != dim + 1:
        return 0.0
    return float(G[0, dim - 1] ** 2) * float(kvec[dim]) ** 2


def _fields(basis: Basis, n: Sequence[int]) -> np.ndarray:
    nr = int(np.prod(n))
    shape = (n[2], n[1], n[0])
    out = np.zeros((len(basis), nr), dtype=complex)
    for j, (idx, coef) in enumerate(basis):
        kg = np.zeros(nr, dtype=complex)
        kg[idx] = coef
        out[j] = (np.fft.ifftn(kg.reshape(shape)) * nr).ravel()
    return out


def drho_domega_id(engine: Engine, inst: int, kvec: Sequence[float], basis: Basis, ktrans_sq: float = 0.0):
    """(smm, spm, spp) after the sign flip of response_sweep (:362-364);
    smm holds the lower triangle (k1 >= j) the reference stores packed.
    Requires a preceding engine.density call (the state to perturb)."""
    if engine.M != 2:
        raise ValueError("the reference's response code handles two monomer types only")
    n = list(engine.systems[inst].n)
    nb = len(basis)
    W = _fields(basis, n)
    pm = np.repeat(np.arange(2, dtype=np.int32), nb)
    fields = np.concatenate([W, W])
    ri = np.array([int(idx[0]) for idx, _ in basis], dtype=np.int32)
    rc = np.array([complex(c[0]) for _, c in basis])
    out = engine.response_raw(inst, list(kvec), ktrans_sq, pm, fields, ri, rc)
    raw = out.reshape(2, nb, 2, nb)              # [p_mon][j][i][k1]
    smm = np.zeros((nb, nb))
    spm = np.zeros((nb, nb))
    spp = np.zeros((nb, nb))
    low = np.tril(np.ones((nb, nb), dtype=bool))
    for p in range(2):
        for i in range(2):
            v = raw[p, :, i, :].T                    # [k1][j]
            smm += np.where(low, (-1.0) ** ((i + 1) + (p + 1)) * v, 0.0)
            spm += (-1.0) ** (1 + (p + 1)) * v
            spp += v
    return -smm / 2.0, -spm / 2.0, -spp / 2.0


def _lower_sym(a: np.ndarray) -> np.ndarray:
    return np.tril(a) + np.tril(a, -1).T


def _shell_sort(a: np.ndarray, index: np.ndarray):
    a, index = a.copy(), index.copy()
    n, inc = len(a), 1
    while True:
        inc = 3 * inc + 1
        if inc > n:
            break
    while True:
        inc //= 3
        for i in range(inc, n):
            v, k, j = a[i], index[i], i
            while a[j - inc] > v:
                a[j], index[j] = a[j - inc], index[j - inc]
                j -= inc
                if j < inc:
                    break
            a[j], index[j] = v, k
        if inc <= 1:
            break
    return a, index


def drho_domega_full(smm, spm, spp, chi12: float, n_eigval_out: int):
    """Eigenvalues (ascending) and eigenvectors of the incompressible
    response, as calc_drho_domega_full computes them."""
    sppi = np.linalg.inv(_lower_sym(spp))
    S = _lower_sym(smm) - _lower_sym(spm.T @ sppi @ spm)
    ev, V = np.linalg.eigh(S)
    ev = 1.0 / ev - chi12
    ev, idx = _shell_sort(ev, np.arange(len(ev)))
    if abs(ev[0]) > 1.0e5:
        n_out = min(n_eigval_out, len(ev) - 1)
        return ev[1:1 + n_out], V[:, idx[1:1 + n_out]]
    n_out = min(n_eigval_out, len(ev))
    return ev[:n_out], V[:, idx[:n_out]]


def response_sweep(engine: Engine, inst: int, kvec0: Sequence[float], dkvec: Sequence[float], nkstep: int,
                   k_group: str, n_eigval_out: int) -> List[dict]:
    """k = kvec0 + j dkvec, j = 0..nkstep: eigenvalues/eigenvectors of the
    incompressible response at each k (kdim = len(kvec0): dim, or dim + 1
    with a transverse component).  The engine must hold the converged state
    of instance `inst` (a preceding density call)."""
    s = engine.systems[inst]
    G = s.unit_cell()[0]
    basis = perturbation_basis(k_group, s.ngrid)
    chi12 = float(s.chi[0, 1])
    out = []
    k = np.array(kvec0, dtype=float)
    for _ in range(nkstep + 1):
        kt = transverse_ksq(s.dim, G, k)
        smm, spm, spp = drho_domega_id(engine, inst, k[: s.dim], basis, kt)
        ev, V = drho_domega_full(smm, spm, spp, chi12, n_eigval_out)
        out.append({"kvec": k.copy(), "eval": ev, "evec": V, "n_basis": len(basis)})
        k = k + np.asarray(dkvec, dtype=float)
    return out
