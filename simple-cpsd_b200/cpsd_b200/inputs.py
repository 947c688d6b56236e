"""Seeded synthetic inputs for the steepest-descent path, in the reference's layouts.

Everything ``cpsd()`` takes is built here, exactly as the reference's driver
builds it (``ccpsdv3/main.c``), with the analytic pseudopotential family and
seeded orbitals the workloads use in place of the reference's tabulated
``.vpp`` files and ``cmakepsi`` plane waves:

* lattice and reciprocal vectors -- ``ccpsdv3/get_cube.c:29-85``
* G-vector table in half-box order -- ``ccpsdv3/get_g.c:12-35``
* cutoff mask -- ``ccpsdv3/get_masker.c:12-37`` (``ggcut`` in bohr^-2 equals
  the cutoff in Rydberg)
* tg = G^2/2, vc = 4 pi/G^2, vg = vc exp(-G^2 rcut^2/4), all masked, and the
  mask duplicated per re/im -- ``ccpsdv3/main.c:169-198``
* Ewald constant and the 27-cell image lattice -- ``ccpsdv3/main.c:286-313``
* ``.vpp`` arrays vl, vnl, vnlnrm -- layout of ``ckbppv3/kbppv3.c:138-150``
  (read at ``ccpsdv3/main.c:264-284``), values from Gaussian model potentials
* orbitals: complex normal coefficients on the half sphere with the kx=0
  plane Hermitian (``cmakepsi/makepsi.c:121-128`` layout), Gram-Schmidt
  orthonormalised with the Gamma-point metric of ``ccpsdv3/gcdotc.c``; or,
  when a cell lists ``start_waves``, the reference's plane-wave start
  (``cmakepsi/dmakepsi.c:93-140``).

Complex arrays are float64 views of the half box: per band
``n2ft3d = (nfft+2)*nfft*nfft`` doubles, index ``2*(i + j*nh + k*nh*nfft)``
with ``nh = nfft//2+1`` (``kx`` fastest).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Sequence, Tuple

import numpy as np

# Madelung constants by lattice type, ccpsdv3/main.c:149-152
_MADELUNG = {1: 1.76011888, 2: 1.791753, 3: 1.791860}


@dataclasses.dataclass
class Species:
    """One ion kind: valence charge, mass (amu) and Gaussian model psp."""

    symbol: str
    zv: float
    amass: float
    lmax: int  # reference convention: lmmax = lmax*lmax projectors (1 = s, 2 = s+p)
    rc_loc: float  # width of the erf-screened local potential
    rc_kb: float  # width of the Gaussian KB projectors
    ekb: Tuple[float, ...]  # KB strength per l (Ha)


@dataclasses.dataclass
class CellSpec:
    """A steepest-descent problem: cell, grid, cutoff, ions, bands, seed."""

    name: str
    unit: float  # lattice constant (bohr)
    nfft: int
    ecut_ry: float  # |G|^2 < ecut_ry (bohr^-2) defines the mask
    species: List[Species]
    katm: List[int]  # 0-based species index per ion
    positions: np.ndarray  # (nion, 3) bohr
    ne: Tuple[int, int]
    ispin: int = 1
    icube: int = 1
    seed: int = 0
    dt: float = 5.8
    fmass: float = 400000.0
    move: int = 0
    # PSI0.DAT rows (i, j, k, l) of a plane-wave start in place of the seeded
    # orbitals; spin 1 reuses the first ne[1] rows, as dmakepsi does
    start_waves: Tuple[Tuple[int, int, int, int], ...] = ()


# ----------------------------------------------------------------- tables

def get_cube(icube: int, unit: float):
    """Primitive vectors, reciprocal vectors and volume: get_cube.c:29-85."""
    if icube == 1:
        a = np.eye(3)
    elif icube == 2:
        a = np.array([[0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    elif icube == 3:
        a = np.array([[0.5, 0.5, 0.5], [-0.5, 0.5, 0.5], [0.5, 0.5, -0.5]])
    else:
        raise ValueError("get_cube: unknown lattice itype %d" % icube)
    unita = (a * unit).reshape(9)  # unita[3*d + c] = component c of vector d
    A = unita.reshape(3, 3)
    g = np.empty((3, 3))
    g[0] = np.cross(A[1], A[2])
    g[1] = np.cross(A[2], A[0])
    g[2] = np.cross(A[0], A[1])
    v = float(A[0] @ g[0])
    unitg = (g * (2.0 * math.pi / v)).reshape(9)
    return abs(v), unita, unitg


def _half_box_k(nfft: int):
    """Signed (k1,k2,k3) of every half-box index, each of shape (nfft3d,)."""
    nh = nfft // 2 + 1
    k1 = np.arange(nh)
    k2 = np.arange(nfft)
    k2 = np.where(k2 > nfft // 2, k2 - nfft, k2)
    kk3, kk2, kk1 = np.meshgrid(k2, k2, k1, indexing="ij")
    return kk1.reshape(-1), kk2.reshape(-1), kk3.reshape(-1)


def get_g(nfft: int, unitg: np.ndarray) -> np.ndarray:
    """G[3*nfft3d]: get_g.c:12-35 (k in (-n/2, n/2], wrapped to [0, n))."""
    k1, k2, k3 = _half_box_k(nfft)
    U = unitg.reshape(3, 3)
    G = np.empty((3, k1.size))
    for c in range(3):
        G[c] = k1 * U[0, c] + k2 * U[1, c] + k3 * U[2, c]
    return G.reshape(-1)


def get_masker(nfft: int, ggcut: float, unitg: np.ndarray) -> np.ndarray:
    """masker1[nfft3d]: 1 where |G|^2 < ggcut over the open box, get_masker.c:12-37."""
    k1, k2, k3 = _half_box_k(nfft)
    nh = nfft // 2
    inside = (k1 < nh) & (np.abs(k2) < nh) & (np.abs(k3) < nh) & (k2 > -nh) & (k3 > -nh)
    U = unitg.reshape(3, 3)
    gg = np.zeros(k1.size)
    for c in range(3):
        gc = k1 * U[0, c] + k2 * U[1, c] + k3 * U[2, c]
        gg += gc * gc
    return ((gg < ggcut) & inside).astype(np.int32)


def gssum_np(nfft: int, x: np.ndarray) -> float:
    """gssum.c:30-41: 2*sum(all) - sum(kx=0 plane)."""
    nh = nfft // 2 + 1
    return 2.0 * float(np.sum(x)) - float(np.sum(x[::nh]))


# ----------------------------------------------------------------- psp

def analytic_psp(sp: Species, G: np.ndarray, nfft3d: int):
    """vl[nfft3d], vnl[9*nfft3d], vnlnrm[9] for a Gaussian model psp.

    Local: V(r) = -Z erf(r/rc)/r, so vl(G) = -4 pi Z exp(-G^2 rc^2/4)/G^2 and
    vl(0) = pi Z rc^2 (the Coulomb divergence dropped, as the reference does).
    KB: normalised Gaussian projectors p_s ~ exp(-r^2/2rc^2) and
    p_x,y,z ~ r_{x,y,z} exp(-r^2/2rc^2); vnl holds |FT| (the reference
    multiplies the p channels by i itself, ccpsdv3/cpsd.c:277-286) and
    vnlnrm = 1/E_KB, so -<chi|c> chi/(Omega vnlnrm) is E_KB |p><p|.
    """
    Gx, Gy, Gz = G[:nfft3d], G[nfft3d:2 * nfft3d], G[2 * nfft3d:]
    gg = Gx * Gx + Gy * Gy + Gz * Gz
    Z, rl, rk = sp.zv, sp.rc_loc, sp.rc_kb
    vl = np.empty(nfft3d)
    with np.errstate(divide="ignore", invalid="ignore"):
        vl[:] = -4.0 * math.pi * Z * np.exp(-gg * rl * rl / 4.0) / gg
    vl[gg == 0.0] = math.pi * Z * rl * rl
    vnl = np.zeros(9 * nfft3d)
    vnlnrm = np.zeros(9)
    lmmax = sp.lmax * sp.lmax
    gauss = np.exp(-gg * rk * rk / 2.0)
    ns = (math.pi * rk * rk) ** -0.75
    ft = (2.0 * math.pi * rk * rk) ** 1.5
    if lmmax >= 1:
        vnl[:nfft3d] = ns * ft * gauss
        vnlnrm[0] = 1.0 / sp.ekb[0]
    if lmmax >= 4:
        npn = ((rk * rk / 2.0) * (math.pi * rk * rk) ** 1.5) ** -0.5
        for l, comp in enumerate((Gx, Gy, Gz), start=1):
            vnl[l * nfft3d:(l + 1) * nfft3d] = npn * rk * rk * ft * comp * gauss
            vnlnrm[l] = 1.0 / sp.ekb[1]
    return vl, vnl, vnlnrm


# ----------------------------------------------------------------- orbitals

def plane_wave_orbitals(nfft: int, ispin: int, ne, rows) -> np.ndarray:
    """The plane-wave start of cmakepsi/dmakepsi.c:93-140: band n of spin
    ms is the wave of row n (coefficient 1 for l = 0, 1/sqrt(2) for l > 0,
    i/sqrt(2) for l < 0), with its Hermitian partner on the kx = 0 plane."""
    nh = nfft // 2 + 1
    n2 = (nfft + 2) * nfft * nfft
    s = 1.0 / math.sqrt(2.0)
    out = np.zeros((int(ne[0]) + (int(ne[1]) if ispin == 2 else 0)) * n2)
    b = 0
    for ms in range(ispin):
        for n in range(int(ne[ms])):
            i, j, k, l = (int(v) for v in rows[n])
            re, im = (0.0, s) if l < 0 else ((1.0, 0.0) if l == 0 else (s, 0.0))
            k2, k3 = (j + nfft) % nfft, (k + nfft) % nfft
            idx = b * n2 + 2 * (i + k2 * nh + k3 * nh * nfft)
            out[idx], out[idx + 1] = re, im
            if i == 0:
                idx = b * n2 + 2 * (((nfft - k2) % nfft) * nh + ((nfft - k3) % nfft) * nh * nfft)
                out[idx], out[idx + 1] = re, -im
            b += 1
    return out


def gamma_weights(nfft: int) -> np.ndarray:
    """Per half-box point weight of the Gamma-point dot: 1 on kx=0, else 2."""
    nh = nfft // 2 + 1
    w = np.full(nh * nfft * nfft, 2.0)
    w[::nh] = 1.0
    return w


def hermitian_partner(nfft: int) -> np.ndarray:
    """Index of (0,-ky,-kz) for every half-box index (only meaningful at kx=0)."""
    nh = nfft // 2 + 1
    idx = np.arange(nh * nfft * nfft)
    i = idx % nh
    j = (idx // nh) % nfft
    k = idx // (nh * nfft)
    return i + ((nfft - j) % nfft) * nh + ((nfft - k) % nfft) * nh * nfft


def random_orbitals(nfft: int, masker1: np.ndarray, nbands: int, seed: int) -> np.ndarray:
    """(nbands, n2ft3d) float64: seeded, Hermitian on kx=0, orthonormal."""
    nh = nfft // 2 + 1
    nfft3d = nh * nfft * nfft
    pts = np.flatnonzero(masker1)
    rng = np.random.default_rng(seed)
    partner = hermitian_partner(nfft)
    on_plane = (pts % nh) == 0
    w = gamma_weights(nfft)[pts]
    C = np.zeros((nbands, pts.size), dtype=np.complex128)
    # position of each point's partner inside pts (for kx=0 points)
    pos = np.full(nfft3d, -1, dtype=np.int64)
    pos[pts] = np.arange(pts.size)
    ppos = pos[partner[pts]]
    follower = on_plane & (partner[pts] < pts)  # take conj of an earlier partner
    self_conj = on_plane & (partner[pts] == pts)  # G = 0
    for b in range(nbands):
        c = rng.standard_normal(pts.size) + 1j * rng.standard_normal(pts.size)
        c[follower] = np.conj(c[ppos[follower]])
        c[self_conj] = c[self_conj].real
        C[b] = c
    # modified Gram-Schmidt, two passes, metric <a|b> = sum w Re(conj(a) b)
    for _ in range(2):
        for b in range(nbands):
            v = C[b]
            for a in range(b):
                v = v - np.sum(w * (C[a].conj() * v).real) * C[a]
            v = v / math.sqrt(np.sum(w * (v.conj() * v).real))
            C[b] = v
    out = np.zeros((nbands, nfft3d), dtype=np.complex128)
    out[:, pts] = C
    return np.ascontiguousarray(out).view(np.float64).reshape(nbands, 2 * nfft3d)


# ----------------------------------------------------------------- assembly

@dataclasses.dataclass
class CpsdInputs:
    """All arguments of cpsd() (ccpsdv3/cpsd.c:33-71) as host arrays."""

    spec: CellSpec
    nfft: int
    nfft3d: int
    n2ft3d: int
    ispin: int
    ne: np.ndarray  # int32[2]
    nion: int
    unita: np.ndarray
    unitg: np.ndarray
    omega: float
    dt: float
    fmass: float
    katm: np.ndarray  # int32[nion]
    amass: np.ndarray  # [nkatm], already x1822.89 (main.c:272)
    zv: np.ndarray
    nsh: int
    rcell: np.ndarray  # [3*nsh]
    cewald: float
    rcut: float
    masker1: np.ndarray  # int32[nfft3d]
    masker: np.ndarray  # int32[n2ft3d]
    G: np.ndarray
    tg: np.ndarray
    vc: np.ndarray
    vg: np.ndarray
    lmmax: np.ndarray  # int32[nkatm]
    vnlnrm: np.ndarray  # [9*nkatm]
    vl: np.ndarray  # [nkatm*nfft3d]
    vnl: np.ndarray  # [9*nkatm*nfft3d]
    r2: np.ndarray  # [3*nion]
    c2: np.ndarray  # [(ne0+ne1)*n2ft3d]

    @property
    def nbands(self) -> int:
        return int(self.ne[0] + self.ne[1])

    @property
    def npw(self) -> int:
        return int(self.masker1.sum())


def build_inputs(spec: CellSpec) -> CpsdInputs:
    nfft = spec.nfft
    nh = nfft // 2 + 1
    nfft3d = nh * nfft * nfft
    n2ft3d = 2 * nfft3d
    omega, unita, unitg = get_cube(spec.icube, spec.unit)
    G = get_g(nfft, unitg)
    masker1 = get_masker(nfft, spec.ecut_ry, unitg)
    rcut = spec.unit / math.pi  # main.c:153
    gg = G[:nfft3d] ** 2 + G[nfft3d:2 * nfft3d] ** 2 + G[2 * nfft3d:] ** 2
    tg = np.zeros(nfft3d)
    vc = np.zeros(nfft3d)
    vg = np.zeros(nfft3d)
    w = 0.25 * rcut * rcut
    tg[1:] = 0.5 * gg[1:]
    vc[1:] = 4.0 * math.pi / gg[1:]
    vg[1:] = vc[1:] * np.exp(-w * gg[1:])
    tg *= masker1
    vc *= masker1
    vg *= masker1
    masker = np.repeat(masker1, 2).astype(np.int32)

    nkatm = len(spec.species)
    katm = np.asarray(spec.katm, dtype=np.int32)
    nion = katm.size
    zv = np.array([s.zv for s in spec.species], dtype=np.float64)
    amass = np.array([s.amass * 1822.89 for s in spec.species], dtype=np.float64)
    lmmax = np.array([s.lmax * s.lmax for s in spec.species], dtype=np.int32)
    vl = np.zeros(nkatm * nfft3d)
    vnl = np.zeros(9 * nkatm * nfft3d)
    vnlnrm = np.zeros(9 * nkatm)
    for ia, sp in enumerate(spec.species):
        a, b, c = analytic_psp(sp, G, nfft3d)
        vl[ia * nfft3d:(ia + 1) * nfft3d] = a
        vnl[ia * 9 * nfft3d:(ia + 1) * 9 * nfft3d] = b
        vnlnrm[ia * 9:(ia + 1) * 9] = c

    # Ewald, main.c:286-313
    alpha = _MADELUNG.get(spec.icube, 0.0)
    rs = (3.0 * omega / (4.0 * math.pi)) ** (1.0 / 3.0)
    q = zv[katm]
    zz = float(np.sum(q * q))
    z = float(np.sum(q))
    cewald = (-0.5 * zz * (alpha / rs + gssum_np(nfft, vg) / omega)
              - 0.5 * (z * z - zz) * rcut * rcut * math.pi / omega)
    ncut = 1
    cells = [(i1, i2, i3) for i3 in range(-ncut, ncut + 1)
             for i2 in range(-ncut, ncut + 1) for i1 in range(-ncut, ncut + 1)]
    nsh = len(cells)
    U = unita.reshape(3, 3)
    rcell = np.zeros(3 * nsh)
    for l, (i1, i2, i3) in enumerate(cells):
        v = i1 * U[0] + i2 * U[1] + i3 * U[2]
        rcell[l], rcell[l + nsh], rcell[l + 2 * nsh] = v

    ne = np.array(spec.ne, dtype=np.int32)
    if spec.start_waves:
        c2 = plane_wave_orbitals(nfft, spec.ispin, ne, spec.start_waves)
    else:
        c2 = random_orbitals(nfft, masker1, int(ne.sum()), spec.seed).reshape(-1)
    r2 = np.asarray(spec.positions, dtype=np.float64).reshape(-1).copy()
    return CpsdInputs(spec=spec, nfft=nfft, nfft3d=nfft3d, n2ft3d=n2ft3d, ispin=spec.ispin,
                      ne=ne, nion=nion, unita=unita, unitg=unitg, omega=omega, dt=spec.dt,
                      fmass=spec.fmass, katm=katm, amass=amass, zv=zv, nsh=nsh, rcell=rcell,
                      cewald=cewald, rcut=rcut, masker1=masker1, masker=masker, G=G, tg=tg,
                      vc=vc, vg=vg, lmmax=lmmax, vnlnrm=vnlnrm, vl=vl, vnl=vnl, r2=r2, c2=c2)
