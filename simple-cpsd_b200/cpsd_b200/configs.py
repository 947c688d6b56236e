"""Named workloads: seeded synthetic cells with the analytic psp family.

* ``h2_dimer_32``      -- SC a=20, 32^3 grid, 30 Ry, two Z=1 ions at (+-0.7,0,0),
  s projector r_c=0.6 / E_KB=0.5, one doubly occupied band (CPU-runnable,
  200 SD steps of inner=1).
* ``diamond8_64``      -- SC a=10.26, 64^3, 40 Ry, 8 Z=4 ions on diamond sites
  with seeded +-0.05 bohr jitter, s+p projectors, 16 bands.
* ``diamond64_128``    -- SC a=20.5, 128^3, 40 Ry, 2x2x2 diamond supercell
  (64 Z=4 ions, +-0.1 bohr jitter), s+p, 128 bands.
* ``batched_cells``    -- 48 cells drawn from one seed: grid 32/48/64, a=0.5 n
  bohr, 2-16 ions with Z in {1,4} at least 1.5 bohr apart, nb = ceil(sum Z/2)
  rounded up into [4, 32], 30 Ry.
* ``small_*``          -- reduced cells for fast parity tests.

Positions live in the box centred on the origin, [-a/2, a/2)^3: the
reference's phase factors carry a +pi shift that puts the real-space grid
origin at the box corner -a/2 (``ccpsdv3/strfac.c:22-24``).
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

from .inputs import CellSpec, Species

H_S = Species("H", zv=1.0, amass=1.008, lmax=1, rc_loc=0.5, rc_kb=0.6, ekb=(0.5,))
C_SP = Species("C", zv=4.0, amass=12.011, lmax=2, rc_loc=0.9, rc_kb=1.0, ekb=(1.0, 0.3))

_DIAMOND_FRAC = np.array([
    [0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0],
    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25],
])


def _wrap(pos: np.ndarray, a: float) -> np.ndarray:
    return (pos + 0.5 * a) % a - 0.5 * a


def h2_dimer_32(seed: int = 0) -> CellSpec:
    pos = np.array([[-0.7, 0.0, 0.0], [0.7, 0.0, 0.0]])
    return CellSpec(name="h2_dimer_32", unit=20.0, nfft=32, ecut_ry=30.0, species=[H_S],
                    katm=[0, 0], positions=pos, ne=(1, 0), seed=seed)


def diamond_positions(a: float, reps: int, jitter: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed + 7919)
    frac = []
    for i in range(reps):
        for j in range(reps):
            for k in range(reps):
                frac.append((_DIAMOND_FRAC + np.array([i, j, k])) / reps)
    frac = np.concatenate(frac)
    pos = a * frac - 0.5 * a + rng.uniform(-jitter, jitter, size=frac.shape)
    return _wrap(pos, a)


def diamond8_64(seed: int = 0) -> CellSpec:
    a = 10.26
    pos = diamond_positions(a, 1, 0.05, seed)
    return CellSpec(name="diamond8_64", unit=a, nfft=64, ecut_ry=40.0, species=[C_SP],
                    katm=[0] * 8, positions=pos, ne=(16, 0), seed=seed)


def diamond64_128(seed: int = 0, nbands: int = 128) -> CellSpec:
    a = 20.5
    pos = diamond_positions(a, 2, 0.1, seed)
    name = "diamond64_128" if nbands == 128 else "diamond64_128_b%d" % nbands
    return CellSpec(name=name, unit=a, nfft=128, ecut_ry=40.0, species=[C_SP],
                    katm=[0] * 64, positions=pos, ne=(nbands, 0), seed=seed)


def batched_cells(seed: int = 0, count: int = 48) -> List[CellSpec]:
    rng = np.random.default_rng(seed + 104729)
    cells = []
    for c in range(count):
        n = int(rng.choice([32, 48, 64]))
        a = 0.5 * n
        nion = int(rng.integers(2, 17))
        kinds = rng.integers(0, 2, size=nion)  # 0 -> H (Z=1), 1 -> C (Z=4)
        pos: List[np.ndarray] = []
        tries = 0
        while len(pos) < nion and tries < 100000:
            tries += 1
            p = rng.uniform(-0.5 * a, 0.5 * a, size=3)
            ok = True
            for q in pos:
                d = p - q
                d -= a * np.round(d / a)
                if np.sqrt(d @ d) < 1.5:
                    ok = False
                    break
            if ok:
                pos.append(p)
        zsum = float(sum(4.0 if k else 1.0 for k in kinds))
        nb = int(min(32, max(4, math.ceil(zsum / 2.0))))
        species = [H_S, C_SP]
        cells.append(CellSpec(name="batched_%02d" % c, unit=a, nfft=n, ecut_ry=30.0,
                              species=species, katm=[int(k) for k in kinds],
                              positions=np.array(pos), ne=(nb, 0), seed=seed * 1000 + c))
    return cells


def h2_molecules(seed: int = 0, count: int = 4, a: float = 16.0, nfft: int = 32) -> CellSpec:
    """`count` H2 molecules (bond 1.4 bohr, seeded centres at least 5 bohr
    apart and seeded orientations) in an SC box: one doubly occupied band per
    molecule, a large gap between the bonding and antibonding levels, so the
    fixed-occupation SD minimum is unique (a control for path-dependent ends)."""
    rng = np.random.default_rng(seed + 4241)
    centres: List[np.ndarray] = []
    while len(centres) < count:
        p = rng.uniform(-0.5 * a, 0.5 * a, size=3)
        ok = True
        for q in centres:
            d = p - q
            d -= a * np.round(d / a)
            if np.sqrt(d @ d) < 5.0:
                ok = False
                break
        if ok:
            centres.append(p)
    pos = []
    for c in centres:
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        pos += [c + 0.7 * u, c - 0.7 * u]
    return CellSpec(name="h2_molecules_%d" % count, unit=a, nfft=nfft, ecut_ry=30.0, species=[H_S],
                    katm=[0] * (2 * count), positions=_wrap(np.array(pos), a), ne=(count, 0), seed=seed)


def small_diamond(nfft: int = 24, nb: int = 4, ecut: float = 20.0, seed: int = 3,
                  ispin: int = 1) -> CellSpec:
    """8-atom diamond cell on a small grid: s+p projectors, few bands."""
    a = 10.26
    pos = diamond_positions(a, 1, 0.05, seed)
    ne = (nb, 0) if ispin == 1 else (nb, max(nb - 1, 1))
    return CellSpec(name="small_diamond_%d" % nfft, unit=a, nfft=nfft, ecut_ry=ecut,
                    species=[C_SP], katm=[0] * 8, positions=pos, ne=ne, ispin=ispin, seed=seed)


def spin_h2(nfft: int = 16, ne=(2, 1)) -> CellSpec:
    """Spin-polarised H2 from the reference's plane-wave start.  The
    reference's Dirac exchange takes xi from the first two density values
    (dirac_exchange.c:101) and returns NaN wherever |xi| > 1; near-uniform
    plane-wave densities keep |xi| small for the first steps."""
    spec = small_h2(nfft)
    spec.name = "spin_h2_%d" % nfft
    spec.ispin = 2
    spec.ne = tuple(ne)
    spec.start_waves = ((0, 0, 0, 0), (1, 0, 0, 1), (1, 0, 0, -1), (0, 1, 0, 1))[:max(ne)]
    return spec


def spin_diamond(nfft: int = 24, ne=(3, 2), ecut: float = 20.0) -> CellSpec:
    """Spin-polarised 8-atom diamond from the plane-wave start (see spin_h2)."""
    spec = small_diamond(nfft, ne[0], ecut=ecut)
    spec.name = "spin_diamond_%d" % nfft
    spec.ispin = 2
    spec.ne = tuple(ne)
    spec.start_waves = ((0, 0, 0, 0), (1, 0, 0, 1), (1, 0, 0, -1), (0, 1, 0, 1), (0, 1, 0, -1))[:max(ne)]
    return spec


def small_h2(nfft: int = 16, nb: int = 1, seed: int = 1) -> CellSpec:
    pos = np.array([[-0.7, 0.0, 0.0], [0.7, 0.0, 0.0]])
    return CellSpec(name="small_h2_%d" % nfft, unit=10.0, nfft=nfft, ecut_ry=12.0, species=[H_S],
                    katm=[0, 0], positions=pos, ne=(nb, 0), seed=seed)


NAMED = {
    "h2_dimer_32": h2_dimer_32,
    "diamond8_64": diamond8_64,
    "diamond64_128": diamond64_128,
    # the 128^3 cell with 16 bands: small enough for a full ncu capture
    "diamond64_128_b16": lambda seed=0: diamond64_128(seed, nbands=16),
    "h2_molecules": h2_molecules,
}
