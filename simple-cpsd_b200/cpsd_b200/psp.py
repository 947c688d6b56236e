"""Tabulated pseudopotentials: the input of the reference's psp formatter
(ckbppv3/dkbppv3.c) and its GPU replacement.

``radial_table`` makes a seeded synthetic table in the shape the formatter
reads (dkbppv3.c main(): atom, zv, amass, lmax, rc[0..lmax], nrho, drho,
then nrho rows "rho vp_0 .. vp_lmax" and nrho rows "rho wp_0 .. wp_lmax"):
a uniform radial grid of step drho whose first point is drho/48 instead of
0, a local channel -zv erf(r/rc)/r (exactly -zv/r in the tail, as the
formatter's long-range term assumes), nonlocal channels that differ from it
inside rc by a Gaussian well, and node-less pseudo-wavefunctions
wp_l = r^(l+1) exp(-r^2/(2 s_l^2)).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class RadialTable:
    atom: str
    zv: float
    amass: float
    lmax: int
    rc: np.ndarray      # [lmax+1]
    drho: float
    rho: np.ndarray     # [nrho]
    vp: np.ndarray      # [(lmax+1) * nrho], channel lmax local
    wp: np.ndarray      # [(lmax+1) * nrho]

    @property
    def nrho(self) -> int:
        return len(self.rho)


def radial_table(lmax: int, seed: int = 0, nrho: int = 501, drho: float = 0.02, zv: float = 4.0,
                 atom: str = "C", amass: float = 12.0) -> RadialTable:
    rng = np.random.default_rng(seed)
    rho = drho * np.arange(nrho, dtype=np.float64)
    rho[0] = drho / 48.0
    rc = 0.8 + 0.4 * rng.random(lmax + 1)
    erf = np.vectorize(math.erf)
    vloc = -zv * erf(rho / rc[lmax]) / rho
    vp = np.zeros((lmax + 1, nrho))
    wp = np.zeros((lmax + 1, nrho))
    for l in range(lmax + 1):
        depth = 1.0 + 4.0 * rng.random()
        vp[l] = vloc if l == lmax else vloc - depth * np.exp(-(rho / rc[l]) ** 2)
        s = 0.6 + 0.5 * rng.random()
        wp[l] = rho ** (l + 1) * np.exp(-rho ** 2 / (2.0 * s * s))
    return RadialTable(atom=atom, zv=zv, amass=amass, lmax=lmax, rc=rc, drho=drho, rho=rho,
                       vp=vp.ravel(), wp=wp.ravel())


def write_table(path: str, t: RadialTable) -> None:
    """The text file dkbppv3.c main() reads (17 significant digits)."""
    n = t.nrho
    vp = t.vp.reshape(t.lmax + 1, n)
    wp = t.wp.reshape(t.lmax + 1, n)
    with open(path, "w") as f:
        f.write("%s\n%.17g %.17g %d\n" % (t.atom, t.zv, t.amass, t.lmax))
        f.write(" ".join("%.17g" % x for x in t.rc) + "\n")
        f.write("%d %.17g\n" % (n, t.drho))
        for i in range(n):
            f.write("%.17g " % t.rho[i] + " ".join("%.17g" % x for x in vp[:, i]) + "\n")
        for i in range(n):
            f.write("%.17g " % t.rho[i] + " ".join("%.17g" % x for x in wp[:, i]) + "\n")


def read_table(path: str) -> RadialTable:
    """The text file dkbppv3.c main() reads, token by token as its fscanf
    calls take them (atom, zv, amass, lmax, rc[0..lmax], nrho, drho, rows)."""
    with open(path) as f:
        tok = f.read().split()
    atom = tok[0]
    zv, amass, lmax = float(tok[1]), float(tok[2]), int(tok[3])
    p = 4
    rc = np.array([float(x) for x in tok[p:p + lmax + 1]])
    p += lmax + 1
    nrho, drho = int(tok[p]), float(tok[p + 1])
    p += 2
    rows = np.array([float(x) for x in tok[p:p + 2 * nrho * (lmax + 2)]]).reshape(2, nrho, lmax + 2)
    rho = rows[1, :, 0].copy()  # the second table's rho column is the one kept
    vp = rows[0, :, 1:].T.copy().ravel()
    wp = rows[1, :, 1:].T.copy().ravel()
    return RadialTable(atom=atom, zv=zv, amass=amass, lmax=lmax, rc=rc, drho=drho, rho=rho, vp=vp, wp=wp)


def format_vpp(path: str, table: RadialTable, icube: int, unit: float, nfft: int, highest_l: int) -> None:
    """dkbppv3.c main(): the .vpp file (DATAOUT) of a radial table on an
    nfft grid, kbpp() on the GPU.  highest_l is the answer to its prompt:
    below the table's lmax it lowers lmax, so channel highest_l becomes the
    local one, as in the reference."""
    from . import api, inputs, refio
    _, _, unitg = inputs.get_cube(icube, unit)
    nfft3d = (nfft // 2 + 1) * nfft * nfft
    lmax = min(int(table.lmax), int(highest_l))
    n = table.nrho
    t = RadialTable(atom=table.atom, zv=table.zv, amass=table.amass, lmax=lmax, rc=table.rc[:lmax + 1],
                    drho=table.drho, rho=table.rho, vp=table.vp[:(lmax + 1) * n], wp=table.wp[:(lmax + 1) * n])
    vl, vnl, vnlnrm, _ = api.kbpp(t, inputs.get_g(nfft, unitg), nfft3d)
    refio.write_vpp(path, icube, nfft, unit, t.atom, t.amass, t.zv, lmax, t.rc, vnlnrm, vl, vnl, pad="\0")
