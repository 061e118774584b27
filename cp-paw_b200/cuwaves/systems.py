"""Seeded synthetic inputs for the WAVES hot path.

The reference gets its inputs from objects that are outside this engine:
- the cell and atoms come from CELL and ATOMLIST;
- the G-set and its ordering come from PLANEWAVE$INITIALIZE (src/paw_fft.f90:872-1327);
- the projector tables, Y_lm, DO and the wave-function mass come from SETUP and
  WAVES_UPDATEGSET (src/paw_waves1.f90:6237-6353);
- V_loc comes from POTENTIAL$VOFRHO, and DH from AUGMENTATION$SPHERE.

This module builds the same arrays, in the same layouts, for model systems:
- Si8: cubic diamond, a=10.26 bohr;
- Si64: the 2x2x2 supercell of Si8;
- H2O32: 32 water molecules in an 18.64-bohr box;
- small Si and molecular cells of uneven size.

The setups are synthetic, because the reference's setup generator is out of
scope:
- radial projectors are Fourier transforms of normalised r^l exp(-r^2/2a^2);
- DO and DH follow the l-block structure of the reference (src/paw_waves2.f90:521-541);
- V_loc is a sum of Gaussian wells.

The G-set ordering, MINUSG and the wave-function mass are restatements of the
reference's integer and index rules, and must match them bit for bit.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional, Sequence

import numpy as np

PI = math.pi
AMU = 1822.888486  # electron masses per atomic mass unit

# ----------------------------------------------------------------------------
# lattice helpers
# ----------------------------------------------------------------------------


def gbass(rbas: np.ndarray):
    """GBASS (src/paw_generalpurpose.f90:72-107): reciprocal vectors and volume.

    rbas[:, i] is the i-th lattice vector (Fortran RBAS(:,I)); returns gbas with
    gbas[:, i] the i-th reciprocal vector, and |det|.
    """
    r = np.asarray(rbas, dtype=np.float64)
    g = np.empty((3, 3))
    g[0, 0] = r[1, 1] * r[2, 2] - r[2, 1] * r[1, 2]
    g[1, 0] = r[2, 1] * r[0, 2] - r[0, 1] * r[2, 2]
    g[2, 0] = r[0, 1] * r[1, 2] - r[1, 1] * r[0, 2]
    g[0, 1] = r[1, 2] * r[2, 0] - r[2, 2] * r[1, 0]
    g[1, 1] = r[2, 2] * r[0, 0] - r[0, 2] * r[2, 0]
    g[2, 1] = r[0, 2] * r[1, 0] - r[1, 2] * r[0, 0]
    g[0, 2] = r[1, 0] * r[2, 1] - r[2, 0] * r[1, 1]
    g[1, 2] = r[2, 0] * r[0, 1] - r[0, 0] * r[2, 1]
    g[2, 2] = r[0, 0] * r[1, 1] - r[1, 0] * r[0, 1]
    det = r[0, 0] * g[0, 0] + r[1, 0] * g[1, 0] + r[2, 0] * g[2, 0]
    if det == 0.0:
        raise ValueError("LATTICE VECTORS LINEAR DEPENDEND")
    g *= 2.0 * PI / det
    return g, abs(det)


def boxsph(basis: np.ndarray, rmax: float):
    """BOXSPH at the origin (src/paw_generalpurpose.f90:115-180)."""
    t1, t2, t3 = basis[:, 0], basis[:, 1], basis[:, 2]
    g1 = np.array([t2[1] * t3[2] - t2[2] * t3[1], t2[2] * t3[0] - t2[0] * t3[2], t2[0] * t3[1] - t2[1] * t3[0]])
    g2 = np.array([t3[1] * t1[2] - t3[2] * t1[1], t3[2] * t1[0] - t3[0] * t1[2], t3[0] * t1[1] - t3[1] * t1[0]])
    g3 = np.array([t1[1] * t2[2] - t1[2] * t2[1], t1[2] * t2[0] - t1[0] * t2[2], t1[0] * t2[1] - t1[1] * t2[0]])
    det = t1[0] * g1[0] + t1[1] * g1[1] + t1[2] * g1[2]
    g1, g2, g3 = g1 / det, g2 / det, g3 / det
    ibig = 1000000
    out = []
    for gv in (g1, g2, g3):
        xn = math.sqrt(gv[0] ** 2 + gv[1] ** 2 + gv[2] ** 2) * rmax
        out.append((int(0.0 - xn + 1.0 + ibig) - ibig, int(0.0 + xn + ibig) - ibig))
    return out


def fft_adjust_grid(nr: int) -> int:
    """LIB$FFTADJUSTGRD (src/paw_library.f90:2336-2393)."""
    ifr: List[int] = []
    done = False
    for h in range(1, 26):
        for i in range(3):
            for j in range(2):
                for k in range(2):
                    for m in range(2):
                        if len(ifr) >= 300:
                            done = True
                            break
                        s = 2.0 ** h * 3.0 ** i * 5.0 ** j * 7.0 ** k * 11.0 ** m
                        if s > 37748736.0:
                            continue
                        ifr.append(int(round(s)))
                    if done:
                        break
                if done:
                    break
            if done:
                break
        if done:
            break
    ifr.sort()
    for v in ifr[1:]:
        if v >= nr:
            return v
    raise ValueError("REQUESTED GRIDPOINT OUT OF RANGE")


def reference_grid(rbas: np.ndarray, epw_rho: float):
    """PLANEWAVE$DIVIDERGRIDONTASKS grid for one task (src/paw_fft.f90:823-869)."""
    gbas, _ = gbass(rbas)
    rad = math.sqrt(2.0 * epw_rho) + 1e-6
    (mn1, mx1), (mn2, mx2), (mn3, mx3) = boxsph(gbas, rad)
    return tuple(fft_adjust_grid(n) for n in (mx1 - mn1 + 1, mx2 - mn2 + 1, mx3 - mn3 + 1))


def get_ig(gbas: np.ndarray, epw: float) -> np.ndarray:
    """PLANEWAVE_GETIG at Gamma (src/paw_fft.f90:1211-1327).

    Returns igvec (NG,3) int32 ordered by increasing |G|^2 with ties (|dG^2| <
    1e-5 relative to the first of a shell) ordered lexicographically in
    (i1,i2,i3), including the reference's handling of the last element.
    """
    rad = math.sqrt(2.0 * epw) + 1e-6
    (mn1, mx1), (mn2, mx2), (mn3, mx3) = boxsph(gbas, rad)
    i, j, k = np.meshgrid(np.arange(mn1, mx1 + 1), np.arange(mn2, mx2 + 1), np.arange(mn3, mx3 + 1), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    a, b, c = i.astype(np.float64), j.astype(np.float64), k.astype(np.float64)
    x = gbas[0, 0] * a + gbas[0, 1] * b + gbas[0, 2] * c
    y = gbas[1, 0] * a + gbas[1, 1] * b + gbas[1, 2] * c
    z = gbas[2, 0] * a + gbas[2, 1] * b + gbas[2, 2] * c
    gs = x * x + y * y + z * z
    keep = ~(0.5 * gs > epw)
    iv = np.stack([i[keep], j[keep], k[keep]], axis=1).astype(np.int64)
    g2 = gs[keep]
    order = np.argsort(g2, kind="stable")
    iv, g2 = iv[order], g2[order]
    n = len(g2)
    out = iv.copy()
    istart = 0
    svar = g2[0]
    ig = 1
    while ig < n:
        last = ig == n - 1
        if abs(g2[ig] - svar) < 1e-5 and not last:
            ig += 1
            continue
        istop = n - 1 if last else ig - 1
        blk = out[istart:istop + 1]
        idx = np.lexsort((blk[:, 2], blk[:, 1], blk[:, 0]))
        out[istart:istop + 1] = blk[idx]
        if istop == n - 1:
            break
        istart = istop + 1
        svar = g2[istart]
        ig = istart + 1
    return out.astype(np.int32)


def minus_g(igvec: np.ndarray) -> np.ndarray:
    """PLANEWAVE$MINUSG at Gamma (src/paw_fft.f90:1157-1208); 1-based result."""
    key = {tuple(v): n for n, v in enumerate(igvec.tolist())}
    out = np.zeros(len(igvec), dtype=np.int32)
    for n, v in enumerate(igvec.tolist()):
        m = key.get((-v[0], -v[1], -v[2]))
        if m is None:
            raise ValueError("INVERSION SYMMETRIC PARTNER NOT FOUND")
        out[n] = m + 1
    return out


def gvectors(gbas: np.ndarray, igvec: np.ndarray) -> np.ndarray:
    """PLANEWAVE_GVECTORS at Gamma (src/paw_fft.f90:1475-1508); returns (NGL,3)."""
    t = igvec.astype(np.float64)
    g = np.empty((len(igvec), 3))
    for r in range(3):
        g[:, r] = gbas[r, 0] * t[:, 0] + gbas[r, 1] * t[:, 1] + gbas[r, 2] * t[:, 2]
    return g


def real_ylm(gvec: np.ndarray, lmx: int) -> np.ndarray:
    """Real spherical harmonics in the order LM = 1 + L**2 + L - M.

    The functions for L <= 2 are the ones listed in the header of SPHERICAL$YLM
    (src/paw_spherical.f90:66-92): 1; x, z, y; x^2-y^2, xz, 3z^2-r^2, yz, xy.
    At G=0 only the L=0 function is nonzero (:130-135).  Returns (NGL,LMX).
    """
    if lmx > 9:
        raise ValueError("real_ylm implements L<=2")
    n = len(gvec)
    out = np.zeros((n, lmx))
    x, y, z = gvec[:, 0], gvec[:, 1], gvec[:, 2]
    r = np.sqrt(x * x + y * y + z * z)
    zero = r < 1e-12
    rs = np.where(zero, 1.0, r)
    x, y, z = x / rs, y / rs, z / rs
    fpi = 4.0 * PI
    cols = [
        np.full(n, 1.0 / math.sqrt(fpi)),
        math.sqrt(3.0 / fpi) * x,
        math.sqrt(3.0 / fpi) * z,
        math.sqrt(3.0 / fpi) * y,
        math.sqrt(15.0 / (4.0 * fpi)) * (x * x - y * y),
        math.sqrt(60.0 / (4.0 * fpi)) * x * z,
        math.sqrt(5.0 / (4.0 * fpi)) * (3.0 * z * z - 1.0),
        math.sqrt(60.0 / (4.0 * fpi)) * y * z,
        math.sqrt(60.0 / (4.0 * fpi)) * x * y,
    ]
    for lm in range(lmx):
        out[:, lm] = cols[lm]
        if lm > 0:
            out[zero, lm] = 0.0
    return out


# ----------------------------------------------------------------------------
# synthetic species ("setups")
# ----------------------------------------------------------------------------


@dataclasses.dataclass
class Species:
    name: str
    lox: List[int]            # angular momentum of each radial projector
    width: List[float]        # Gaussian width a of each radial projector (bohr)
    do_s: np.ndarray          # DO block for the s channel (pairs of ln)
    do_p: Optional[np.ndarray]
    dh_s: np.ndarray          # DH block (l-diagonal part)
    dh_p: Optional[np.ndarray]
    v0: float                 # depth of the local Gaussian well (Ha)
    sigma: float              # width of the local Gaussian well (bohr)
    mass_amu: float

    @property
    def lnx(self) -> int:
        return len(self.lox)

    @property
    def lmnx(self) -> int:
        return sum(2 * l + 1 for l in self.lox)


SI = Species("Si", [0, 0, 1, 1], [0.95, 1.45, 1.05, 1.55],
             np.array([[0.35, -0.10], [-0.10, 0.20]]), np.array([[0.25, -0.08], [-0.08, 0.15]]),
             np.array([[-0.55, 0.12], [0.12, -0.25]]), np.array([[-0.20, 0.08], [0.08, -0.10]]),
             1.6, 1.25, 28.0855)
O_ = Species("O", [0, 0, 1, 1], [0.60, 0.95, 0.65, 1.00],
             np.array([[0.30, -0.08], [-0.08, 0.18]]), np.array([[0.22, -0.06], [-0.06, 0.12]]),
             np.array([[-0.80, 0.15], [0.15, -0.35]]), np.array([[-0.30, 0.10], [0.10, -0.15]]),
             2.5, 0.85, 15.999)
H_ = Species("H", [0, 0], [0.45, 0.75],
             np.array([[0.20, -0.05], [-0.05, 0.10]]), None,
             np.array([[-0.40, 0.08], [0.08, -0.15]]), None,
             1.0, 0.65, 1.008)

SPECIES = {"Si": SI, "O": O_, "H": H_}


def radial_projector(sp: Species, ln: int, g: np.ndarray, omega: float) -> np.ndarray:
    """Bessel transform (4 pi/Omega) int r^2 j_l(Gr) p(r) dr of the normalised
    p(r) = c r^l exp(-r^2/2a^2), which is (4 pi/Omega) c sqrt(pi/2) a^(2l+3) G^l exp(-G^2 a^2/2)."""
    l, a = sp.lox[ln], sp.width[ln]
    c = math.sqrt(2.0 / (math.gamma(l + 1.5) * a ** (2 * l + 3)))
    return (4.0 * PI / omega) * c * math.sqrt(PI / 2.0) * a ** (2 * l + 3) * g ** l * np.exp(-0.5 * (g * a) ** 2)


def do_matrix(sp: Species) -> np.ndarray:
    """DO(LNX,LNX): nonzero only between radial projectors of equal l."""
    n = sp.lnx
    d = np.zeros((n, n))
    for l, blk in ((0, sp.do_s), (1, sp.do_p)):
        idx = [i for i in range(n) if sp.lox[i] == l]
        if blk is not None and idx:
            d[np.ix_(idx, idx)] = blk
    return d


def dh_matrix(sp: Species, rng: np.random.Generator, coupling: float = 0.02) -> np.ndarray:
    """DH(LMNX,LMNX) real symmetric: l-block/m-diagonal part plus a small full
    symmetric coupling, stored complex like the reference's DH argument."""
    n = sp.lmnx
    d = np.zeros((n, n))
    # lmn index of (ln, m)
    lmn0, off = [], 0
    for l in sp.lox:
        lmn0.append(off)
        off += 2 * l + 1
    for ln1, l1 in enumerate(sp.lox):
        for ln2, l2 in enumerate(sp.lox):
            if l1 != l2:
                continue
            blk = sp.dh_s if l1 == 0 else sp.dh_p
            i1 = [i for i in range(sp.lnx) if sp.lox[i] == l1].index(ln1)
            i2 = [i for i in range(sp.lnx) if sp.lox[i] == l2].index(ln2)
            for m in range(2 * l1 + 1):
                d[lmn0[ln1] + m, lmn0[ln2] + m] = blk[i1, i2]
    p = rng.uniform(-coupling, coupling, size=(n, n))
    d += 0.5 * (p + p.T)
    return d.astype(np.complex128)


# ----------------------------------------------------------------------------
# systems
# ----------------------------------------------------------------------------

DIAMOND = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                    [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])


@dataclasses.dataclass
class System:
    name: str
    rbas: np.ndarray                 # (3,3), columns are lattice vectors
    pos: np.ndarray                  # (NAT,3) cartesian bohr
    species: List[Species]           # distinct species, in ISP order
    isp: np.ndarray                  # (NAT,) 1-based
    nb: int
    epw_psi: float                   # Hartree
    grid: tuple
    delt: float = 10.0
    emass: float = 1000.0
    emasscg2: Optional[float] = None
    annee: float = 0.0
    seed: int = 0

    @property
    def nat(self) -> int:
        return len(self.pos)


def si_cell(ncell: int = 1, a: float = 10.26, disp: float = 0.0, seed: int = 1, nb: Optional[int] = None,
            epw_psi_ry: float = 30.0, grid=None, name: Optional[str] = None) -> System:
    """Cubic diamond Si (8 atoms per cubic cell), ncell^3 cubic cells; the cell
    edge is ncell*a.  Displacements are uniform in [-disp, disp] bohr (seeded)."""
    rng = np.random.default_rng(seed)
    frac = []
    for i in range(ncell):
        for j in range(ncell):
            for k in range(ncell):
                for f in DIAMOND:
                    frac.append((f + np.array([i, j, k])) / ncell)
    L = ncell * a
    pos = np.array(frac) * L
    if disp:
        pos = pos + rng.uniform(-disp, disp, size=pos.shape)
    nat = len(pos)
    if nb is None:
        nb = 2 * nat  # 4 valence electrons per Si, doubly occupied
    return System(name or f"Si{nat}", np.eye(3) * L, pos, [SI], np.ones(nat, dtype=np.int32), nb,
                  0.5 * epw_psi_ry, grid or (0, 0, 0), seed=seed)


def si_small(nat: int, seed: int = 3, epw_psi_ry: float = 30.0, grid=None) -> System:
    """Si2..Si16 cells cut from the diamond lattice: an orthorhombic box with
    the first nat atoms of the cubic cell (nat <= 8) or of a 1x1x2 stack."""
    a = 10.26
    base = DIAMOND if nat <= 8 else np.concatenate([DIAMOND * [1, 1, 0.5], DIAMOND * [1, 1, 0.5] + [0, 0, 0.5]])
    cz = a if nat <= 8 else 2 * a
    rng = np.random.default_rng(seed)
    pos = base[:nat] * np.array([a, a, cz]) + rng.uniform(-0.05, 0.05, size=(nat, 3))
    return System(f"Si{nat}", np.diag([a, a, cz]), pos, [SI], np.ones(nat, dtype=np.int32), 2 * nat,
                  0.5 * epw_psi_ry, grid or (0, 0, 0), seed=seed)


def water_box(nmol: int = 32, box: float = 18.64, lattice=(4, 4, 2), seed: int = 2,
              epw_psi_ry: float = 40.0, grid=None) -> System:
    """nmol water molecules on a lattice with seeded random orientations,
    O-H 1.81 bohr, H-O-H 104.5 degrees; molecules ordered O,H,H."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = lattice
    ang = math.radians(104.5)
    oh = 1.81
    hloc = np.array([[oh * math.sin(ang / 2), 0.0, oh * math.cos(ang / 2)],
                     [-oh * math.sin(ang / 2), 0.0, oh * math.cos(ang / 2)]])
    o_list, h_list = [], []
    cnt = 0
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                if cnt >= nmol:
                    break
                o = np.array([(i + 0.5) * box / nx, (j + 0.5) * box / ny, (k + 0.5) * box / nz])
                q = rng.normal(size=4)
                q /= np.linalg.norm(q)
                w, x, y, z = q
                rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                                [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                                [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
                o_list.append(o)
                h_list.append(o + hloc @ rot.T)
                cnt += 1
    pos = np.concatenate([np.stack(o_list)] + [np.stack(h_list).reshape(-1, 3)])
    isp = np.array([1] * len(o_list) + [2] * (2 * len(o_list)), dtype=np.int32)
    nb = 4 * nmol  # 8 valence electrons per molecule
    return System(f"H2O{nmol}", np.eye(3) * box, pos, [O_, H_], isp, nb, 0.5 * epw_psi_ry,
                  grid or (0, 0, 0), seed=seed)


def molecule_box(kind: str, box: float = 20.0, seed: int = 3, epw_psi_ry: float = 30.0, grid=None) -> System:
    """Isolated H2O or Si2 molecule in a cubic box."""
    if kind == "H2O":
        s = water_box(1, box, (1, 1, 1), seed=seed, epw_psi_ry=epw_psi_ry, grid=grid)
        s.name = "H2O-mol"
        return s
    if kind == "Si2":
        pos = np.array([[box / 2 - 2.1, box / 2, box / 2], [box / 2 + 2.1, box / 2, box / 2]])
        return System("Si2-mol", np.eye(3) * box, pos, [SI], np.ones(2, dtype=np.int32), 4,
                      0.5 * epw_psi_ry, grid or (0, 0, 0), seed=seed)
    raise ValueError(kind)


def si_supercell(n1: int, n2: int, n3: int, a: float = 10.26, disp: float = 0.05, seed: int = 1,
                 epw_psi_ry: float = 30.0, grid=None) -> System:
    """n1 x n2 x n3 cubic cells of diamond Si (8 n1 n2 n3 atoms) with seeded
    uniform [-disp, disp] bohr displacements; doubly occupied valence bands."""
    rng = np.random.default_rng(seed)
    frac = []
    for i in range(n1):
        for j in range(n2):
            for k in range(n3):
                for f in DIAMOND:
                    frac.append(f + np.array([i, j, k]))
    pos = np.array(frac, dtype=np.float64) * a
    pos = pos + rng.uniform(-disp, disp, size=pos.shape)
    nat = len(pos)
    return System(f"Si{nat}", np.diag([n1 * a, n2 * a, n3 * a]), pos, [SI], np.ones(nat, dtype=np.int32), 2 * nat,
                  0.5 * epw_psi_ry, grid or (0, 0, 0), seed=seed)


def water_cluster(nmol: int, seed: int = 5, epw_psi_ry: float = 40.0, spacing: float = 5.6,
                  vacuum: float = 8.0) -> System:
    """A cluster of nmol water molecules (seeded orientations, on a cubic
    lattice of the given spacing) centred in a cubic box with `vacuum` bohr of
    space on every side."""
    side = int(math.ceil(nmol ** (1.0 / 3.0) - 1e-9))
    box = side * spacing + 2.0 * vacuum
    s = water_box(nmol, box=side * spacing, lattice=(side, side, side), seed=seed, epw_psi_ry=epw_psi_ry)
    s.pos = s.pos + vacuum
    s.rbas = np.eye(3) * box
    s.name = f"(H2O){nmol}"
    return s


# Batched workload: 64 independent small systems of uneven size (bulk Si2-Si16
# cells and isolated molecules in 20-bohr boxes, 4-32 bands, 30 Ry).
def batched_mix(count: int = 64, seed: int = 11) -> List[System]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        k = int(rng.integers(0, 10))
        if k < 8:
            out.append(si_small(int(2 * (k + 1)), seed=100 + i))  # Si2..Si16
        else:
            out.append(molecule_box("Si2" if k == 8 else "H2O", box=20.0, seed=100 + i))
    return out


# Batched workload of the benchmark configuration: 64 systems of uneven size,
# bulk Si2..Si16 cells and Si2 / H2O molecules in 20-bohr boxes, 4-32 bands,
# 30/60 Ry, each on the smallest FFT grid (16 to 40 points per axis) that
# holds its wave-function sphere without aliasing.
FFT_LENGTHS = (16, 18, 20, 24, 28, 30, 32, 36, 40)


def psi_grid(sys: System):
    gbas, _ = gbass(sys.rbas)
    ig = get_ig(gbas, sys.epw_psi)
    out = []
    for d in range(3):
        m = int(np.abs(ig[:, d]).max())
        out.append(next(n for n in FFT_LENGTHS if 2 * m < n))
    return tuple(out)


def config_batch_mix(count: int = 64, seed: int = 11) -> List[System]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        k = int(rng.integers(0, 10))
        if k < 8:
            sy = si_small(int(2 * (k + 1)), seed=100 + i)  # Si2..Si16: 4..32 bands
        else:
            sy = molecule_box("Si2" if k == 8 else "H2O", box=20.0, seed=100 + i)
        sy.grid = psi_grid(sy)
        out.append(sy)
    return out


# Serving workload: perturbed bulk Si_n (n in 8..128) and water clusters of
# 1-16 molecules, 30-40 Ry.
SERVING_SI = {8: (1, 1, 1), 16: (1, 1, 2), 32: (1, 2, 2), 64: (2, 2, 2), 128: (2, 2, 4)}
SERVING_WATER = (1, 2, 4, 8, 16)


def serving_system(kind: str, n: int, seed: int) -> System:
    if kind == "Si":
        return si_supercell(*SERVING_SI[n], disp=0.05, seed=seed, epw_psi_ry=30.0)
    return water_cluster(n, seed=seed, epw_psi_ry=40.0)


# ----------------------------------------------------------------------------
# arrays for the engine
# ----------------------------------------------------------------------------


def build_inputs(sys: System, grid=None, seed: Optional[int] = None, psi_init: str = "gauss") -> Dict[str, np.ndarray]:
    """All arrays the engine needs, in the reference's layouts (numpy arrays in
    Fortran order are returned as C-contiguous arrays of the transposed shape,
    i.e. psi has shape (NBH, NGL) and is exactly PSI(NGL,1,NBH) in memory)."""
    seed = sys.seed if seed is None else seed
    rng = np.random.default_rng(1000 + seed)
    gbas, omega = gbass(sys.rbas)
    if grid is None:
        grid = sys.grid if sys.grid and sys.grid[0] else reference_grid(sys.rbas, 2.0 * sys.epw_psi)
    nr1, nr2, nr3 = grid
    igvec = get_ig(gbas, sys.epw_psi)
    ngl = len(igvec)
    # the FFT grid must hold the sphere without aliasing of +G/-G
    for d, n in enumerate(grid):
        if 2 * np.abs(igvec[:, d]).max() >= n:
            raise ValueError(f"grid {grid} too small for the G sphere")
    minusg = minus_g(igvec)
    gvec = gvectors(gbas, igvec)
    g2 = gvec[:, 0] ** 2 + gvec[:, 1] ** 2 + gvec[:, 2] ** 2
    gabs = np.sqrt(g2)
    lmax = max(max(sp.lox) for sp in sys.species)
    lmx = (lmax + 1) ** 2
    ylm = real_ylm(gvec, lmx)
    pro_cols = []
    for sp in sys.species:
        for ln in range(sp.lnx):
            pro_cols.append(radial_projector(sp, ln, gabs, omega))
    pro = np.stack(pro_cols)  # (NBAREPRO, NGL) == PRO(NGL,NBAREPRO)
    emass = sys.emass
    emasscg2 = sys.emasscg2
    if emasscg2 is None:  # src/paw_ioroutines.f90:1406-1414
        emasscg2 = 0.5 * (10.0 / (2.0 * PI)) ** 2 * sys.delt ** 2 / emass
    mpsi = emass * (1.0 + emasscg2 * g2)  # WAVES_PSIMASS (src/paw_waves1.f90:6595-6673)
    # local potential: Gaussian wells, built in G space so that it is periodic
    f1 = np.fft.fftfreq(nr1, 1.0 / nr1)
    f2 = np.fft.fftfreq(nr2, 1.0 / nr2)
    f3 = np.fft.fftfreq(nr3, 1.0 / nr3)
    I1, I2, I3 = np.meshgrid(f1, f2, f3, indexing="ij")
    GX = gbas[0, 0] * I1 + gbas[0, 1] * I2 + gbas[0, 2] * I3
    GY = gbas[1, 0] * I1 + gbas[1, 1] * I2 + gbas[1, 2] * I3
    GZ = gbas[2, 0] * I1 + gbas[2, 1] * I2 + gbas[2, 2] * I3
    GG = GX * GX + GY * GY + GZ * GZ
    vg = np.zeros((nr1, nr2, nr3), dtype=np.complex128)
    isp0 = np.asarray(sys.isp) - 1
    for s, sp in enumerate(sys.species):
        amp = -sp.v0 * (2.0 * PI * sp.sigma ** 2) ** 1.5 / omega
        form = amp * np.exp(-0.5 * GG * sp.sigma ** 2)
        sf = np.zeros_like(vg)
        for a in np.nonzero(isp0 == s)[0]:
            R = sys.pos[a]
            sf += np.exp(-1j * (GX * R[0] + GY * R[1] + GZ * R[2]))
        vg += form * sf
    vr = np.fft.ifftn(vg).real * (nr1 * nr2 * nr3)  # V(r)=sum_G V(G) exp(iGr)
    v = np.ascontiguousarray(vr.transpose(2, 1, 0))  # x fastest: V(NR1,NR2,NR3)
    # one-centre matrices
    lmnxx = max(sp.lmnx for sp in sys.species)
    lnxx = max(sp.lnx for sp in sys.species)
    dh = np.zeros((sys.nat, lmnxx, lmnxx), dtype=np.complex128)  # DH(LMNXX,LMNXX,NAT)^T per atom
    dhrng = np.random.default_rng(2000 + seed)
    for a in range(sys.nat):
        sp = sys.species[isp0[a]]
        m = dh_matrix(sp, dhrng)
        dh[a, :sp.lmnx, :sp.lmnx] = m.T  # stored transposed: memory == DH(:,:,a) column-major
    dover = np.zeros((len(sys.species), lnxx, lnxx))
    for s, sp in enumerate(sys.species):
        dover[s, :sp.lnx, :sp.lnx] = do_matrix(sp).T
    # occupations: doubly occupied
    occ = np.full(sys.nb, 2.0)
    nbh = (sys.nb + 1) // 2
    # initial coefficients: seeded complex Gaussians damped by exp(-|G|^2/8)
    if psi_init == "gauss":
        psi = (rng.normal(size=(nbh, ngl)) + 1j * rng.normal(size=(nbh, ngl))) * np.exp(-g2 / 8.0)[None, :]
    else:
        psi = np.zeros((nbh, ngl), dtype=np.complex128)
    masses = np.array([sys.species[i].mass_amu * AMU for i in isp0])
    return dict(
        name=sys.name, ngl=ngl, nb=sys.nb, nbh=nbh, nat=sys.nat, nsp=len(sys.species),
        grid=tuple(grid), lmx=lmx, lmnxx=lmnxx, lnxx=lnxx,
        lnx=[sp.lnx for sp in sys.species], lox=[sp.lox for sp in sys.species],
        isp=np.asarray(sys.isp, dtype=np.int32),
        rbas=sys.rbas, gbas=gbas, omega=omega,
        igvec=np.ascontiguousarray(igvec), minusg=minusg, gvec=np.ascontiguousarray(gvec), g2=g2,
        pro=np.ascontiguousarray(pro), ylm=np.ascontiguousarray(ylm.T), mpsi=mpsi,
        v=v, dh=dh, dover=dover, occ=occ,
        psi=np.ascontiguousarray(psi), r0=np.ascontiguousarray(sys.pos), masses=masses,
        delt=sys.delt, annee=sys.annee, emass=emass, emasscg2=emasscg2,
        rhoset=rhoset_inputs(sys, gbas, omega, grid, seed),
    )


# Synthetic tables of the potential (the SETUP quantities that POTENTIAL_UPDATE
# transforms to G space, src/paw_potential.f90:300-309), per species:
# compensation Gaussian radius rcsm, the wider Gaussian rcbg of V0, pseudo-core
# charge and radius, VADD well depth and width, valence charge.
RHO_SETUP = {"Si": (0.55, 1.10, 0.30, 0.80, 0.50, 1.00, 4.0),
             "O": (0.40, 0.80, 0.40, 0.55, 0.80, 0.70, 6.0),
             "H": (0.30, 0.60, 0.00, 0.40, 0.30, 0.50, 1.0)}


def rhoset_inputs(sys: System, gbas: np.ndarray, omega: float, grid, seed: int):
    """The density G set of the potential and its tables (see
    cuwaves_set_rhoset): the sphere 0.5|G|^2 <= 2 EPWPSI in PLANEWAVE_GETIG
    order, reduced to one G of each +-G pair as PLANEWAVE$SUPFFT does
    (MINUSG(IG) >= IG); YLMOFG = Y_lm(G)|G|^l for l <= 2; G0 and V0 of Gaussian
    compensation charges, a Gaussian pseudo core and a Gaussian VADD well per
    species, each normalised so that a factor Y0 recovers the charge per cell
    volume at G = 0; QLM: minus the valence charge on the monopole plus small
    seeded higher moments.  None when the grid cannot hold the sphere."""
    full = get_ig(gbas, 2.0 * sys.epw_psi)
    for d, n in enumerate(grid):
        if 2 * np.abs(full[:, d]).max() >= n:
            return None
    mg = minus_g(full) - 1  # 0-based partner of each G
    keep = mg >= np.arange(len(full))
    igvec = np.ascontiguousarray(full[keep])
    gvec = gvectors(gbas, igvec)
    g2 = gvec[:, 0] ** 2 + gvec[:, 1] ** 2 + gvec[:, 2] ** 2
    glen = np.sqrt(g2)
    lmrxx = 9
    ylm = real_ylm(gvec, lmrxx)
    for lm in range(1, 4):
        ylm[:, lm] *= glen
    for lm in range(4, 9):
        ylm[:, lm] *= g2
    y0 = 1.0 / math.sqrt(4.0 * PI)
    nsp = len(sys.species)
    g0 = np.zeros((nsp, len(g2)))
    v0 = np.zeros_like(g0)
    pscore = np.zeros_like(g0)
    vbar = np.zeros_like(g0)
    gs = np.where(g2 > 1e-12, g2, 1.0)
    for k, sp in enumerate(sys.species):
        rcsm, rcbg, qcore, rcore, vb, sb, _ = RHO_SETUP[sp.name]
        a = np.exp(-0.25 * g2 * rcsm ** 2)
        b = np.exp(-0.25 * g2 * rcbg ** 2)
        g0[k] = a / (omega * y0)
        v0[k] = np.where(g2 > 1e-12, 4.0 * PI * (a - b) / gs, PI * (rcbg ** 2 - rcsm ** 2)) / (omega * y0)
        pscore[k] = qcore * np.exp(-0.25 * g2 * rcore ** 2) / (omega * y0)
        vbar[k] = -vb * (2.0 * PI * sb ** 2) ** 1.5 * np.exp(-0.5 * g2 * sb ** 2) / (omega * y0)
    rng = np.random.default_rng(3000 + seed)
    isp0 = np.asarray(sys.isp) - 1
    qlm = np.zeros((sys.nat, lmrxx))
    for a in range(sys.nat):
        sp = sys.species[isp0[a]]
        qlm[a, 0] = -(RHO_SETUP[sp.name][6] + RHO_SETUP[sp.name][2])
        qlm[a, 1:] = 0.05 * rng.uniform(-1.0, 1.0, lmrxx - 1)
    return dict(igvec=igvec, gvec=np.ascontiguousarray(gvec), g2=g2, lmrxx=lmrxx,
                lmrx=np.full(nsp, lmrxx, dtype=np.int32), ylm=np.ascontiguousarray(ylm),
                g0=g0, v0=v0, pscore=pscore, vbar=vbar, qlm=qlm)


def named_system(name: str) -> System:
    """The workloads of the benchmark configurations."""
    if name == "Si8":
        return si_cell(1, grid=(32, 32, 32), name="Si8")
    if name == "Si8-ref":
        return si_cell(1, name="Si8")
    if name == "Si64":
        return si_cell(2, a=10.26, disp=0.05, seed=1, grid=(64, 64, 64), name="Si64")
    if name == "Si64-ref":
        return si_cell(2, a=10.26, disp=0.05, seed=1, name="Si64")
    if name == "H2O32":
        return water_box(32, grid=(72, 72, 72))
    if name == "Si128":  # the largest system of the serving mix (256 bands)
        return serving_system("Si", 128, 1)
    if name.startswith("Si") and name[2:].isdigit():
        return si_small(int(name[2:]))
    raise ValueError(name)
