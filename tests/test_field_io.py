"""Field files in the reference's basis and grid formats, pinned to the
reference's own field file fixture (tests/golden/fieldfile_rho.txt, copied
from tools/python/tests/fieldfile/rho by make_fieldfile_fixture.py)."""
import os

import numpy as np
import pytest

from pscf_b200 import field_io as F
from pscf_b200 import groups as G
from tests.cases import diblock, omega_guess

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "fieldfile_rho.txt")


def _lines(path):
    return open(path).read().splitlines()


def test_reference_rho_round_trip(tmp_path):
    """Reading the reference's file and writing it back reproduces every
    coefficient to the 12 printed digits, every first wave and star count,
    and the header."""
    h = F._read_header(_lines(FIX))[0]
    assert h["group_name"] == "-1" and h["dim"] == 1 and h["N_monomer"] == 2
    # 21 stars of group -1 on a 40-point grid: waves 0..20
    s = diblock(1, [40], "lamellar", h["cell_param"])
    hdr, rho = F.read_field(FIX, s)
    assert abs(rho.mean(axis=1) - [0.56, 0.44]).max() < 1e-12       # star 0 is the mean
    out = tmp_path / "rho_out"
    F.write_field(str(out), rho, s, "-1")
    a, b = _lines(FIX), _lines(str(out))
    assert len(a) == len(b)
    assert [x.split() for x in a[:14]] == [x.split() for x in b[:14]]
    for la, lb in zip(a[15:], b[15:]):
        va, vb = la.split(), lb.split()
        assert va[2:] == vb[2:]                                      # first wave, star count
        for x, y in zip(va[:2], vb[:2]):
            assert abs(float(x) - float(y)) <= 1e-12 * max(1e-3, abs(float(x)))


@pytest.mark.parametrize("group,dim,ngrid,crystal,cell", [
    ("I m -3 m", 3, [16, 16, 16], "cubic", [1.95]),
    ("p 6 m m", 2, [24, 24], "hexagonal", [1.9]),
    ("I a -3 d", 3, [16, 16, 16], "cubic", [3.7]),
])
def test_basis_file_round_trip_and_first_waves(tmp_path, group, dim, ngrid, crystal, cell):
    """A symmetric field written in the basis format and read back is the
    same grid field; every line's wave is the largest of its star in the
    reference's G ordering and its star count matches the basis."""
    s = diblock(dim, ngrid, crystal, cell)
    w = omega_guess(s, 5, 2.0)
    w = np.stack([G.symmetrize(w[m], group, ngrid) for m in range(2)])
    p = tmp_path / "w"
    F.write_field(str(p), w, s, group)
    _, back = F.read_field(str(p), s)
    assert np.max(np.abs(back - w)) < 1e-10 * max(1.0, np.max(np.abs(w)))
    fb = F.FieldBasis(group, s)
    lines = _lines(str(p))
    nstar = int(lines[14].split()[0])
    assert nstar == fb.basis.n_star
    for ln, bz, cnt in zip(lines[15:], fb.first_bz, fb.count):
        v = ln.split()
        assert [int(x) for x in v[2:2 + dim]] == list(bz) and int(v[2 + dim]) == cnt


def test_rgrid_round_trip(tmp_path):
    s = diblock(2, [12, 18], "rectangular", [1.5, 2.2])
    w = omega_guess(s, 3, 2.0)
    p = tmp_path / "r"
    F.write_rgrid(str(p), w, s, "p 1")
    h, ngrid, back = F.read_rgrid(str(p))
    assert ngrid == [12, 18] and h["crystal_system"] == "rectangular" and h["cell_param"] == [1.5, 2.2]
    assert np.max(np.abs(back - w)) < 1e-9 * 5            # F18.9 printing
    # the grid reader of the reference skips 14 header lines before ngrid
    assert _lines(str(p))[14].split()[0] == "12"


@pytest.mark.parametrize("group,dim,ngrid,crystal,cell", [
    ("1", 1, [16], "lamellar", [1.5]),
    ("P 1", 3, [4, 6, 8], "orthorhombic", [1.0, 1.5, 2.0]),
    ("I 41 3 2", 3, [16, 16, 16], "cubic", [3.7]),
])
def test_basis_file_without_inversion(tmp_path, group, dim, ngrid, crystal, cell):
    """Groups without inversion: stars related by inversion are written as
    +1 / -1 pairs (the -1 line carries the inverse of the +1 line's wave),
    and a symmetric field survives the round trip."""
    s = diblock(dim, ngrid, crystal, cell)
    w = omega_guess(s, 5, 2.0)
    w = np.stack([G.symmetrize(w[m], group, ngrid) for m in range(2)])
    p = tmp_path / "w"
    F.write_field(str(p), w, s, group)
    _, back = F.read_field(str(p), s)
    assert np.max(np.abs(back - w)) < 1e-10 * max(1.0, np.max(np.abs(w)))
    fb = F.FieldBasis(group, s)
    kinds = [st["kind"] for st in fb.stars]
    assert len(fb.stars) == fb.basis.n_star and kinds.count(1) == kinds.count(-1) > 0
    for k, st in enumerate(fb.stars):
        if st["kind"] == 1:
            assert fb.stars[k + 1]["kind"] == -1
            g = np.array(st["wave_bz"])
            gm = np.array(fb.stars[k + 1]["wave_bz"])
            assert np.all((g + gm) % np.array(ngrid) == 0)
    # coefficients of one basis function come back as a unit vector
    for k in range(min(len(fb.stars), 12)):
        a = np.zeros(len(fb.stars))
        a[k] = 1.0
        np.testing.assert_allclose(fb.to_coeffs(fb.to_grid(a)), a, atol=1e-12)


@pytest.mark.parametrize("group,dim,ngrid,crystal,cell", [
    ("P 1", 3, [6, 5, 4], "orthorhombic", [1.0, 1.5, 2.0]),
    ("I 41 3 2", 3, [8, 8, 8], "cubic", [3.7]),
    ("p 6 m m", 2, [9, 9], "hexagonal", [1.9]),
])
def test_wave_grid_file(tmp_path, group, dim, ngrid, crystal, cell):
    """Wave-grid files (read by KGRID_TO_RGRID, src/pscf.fp.f90:813-888):
    the half grid G1 <= n1/2 with G3 fastest; the reader fills the other
    half from F(-G) = conj F(G), so a general real field's full spectrum
    comes back; a group's field read through its basis is unchanged."""
    s = diblock(dim, ngrid, crystal, cell)
    w = omega_guess(s, 7, 2.0)
    p = tmp_path / "k"
    F.write_kgrid(str(p), w, s, group)
    n = list(s.n)
    lines = _lines(str(p))
    assert lines[13].split()[0] == "ngrid" and len(lines) == 15 + (n[0] // 2 + 1) * n[1] * n[2]
    _, spec = F.read_kgrid(str(p), s)
    for m in range(2):
        full = np.fft.fftn(w[m].reshape(n[2], n[1], n[0])).ravel() / s.nr
        np.testing.assert_allclose(spec[m], full, rtol=0, atol=1e-15 * max(1.0, np.max(np.abs(full))))
    ws = np.stack([G.symmetrize(w[m], group, ngrid) for m in range(2)])
    F.write_kgrid(str(p), ws, s, group)
    _, spec = F.read_kgrid(str(p), s)
    fb = F.FieldBasis(group, s)
    back = np.stack([fb.to_grid(fb.spectrum_to_coeffs(z)) for z in spec])
    assert np.max(np.abs(back - ws)) < 1e-12 * max(1.0, np.max(np.abs(ws)))
