"""The reference's input/output files, written and read byte for byte.

* ELCIN / ELCOUT (binary): int icube, int nfft, double unit, int ispin,
  int ne[2], then (ne0+ne1)*n2ft3d doubles -- ccpsdv3/main.c:116-142 and
  :539-547, written by cmakepsi/makepsi.c:105-133.
* ``.vpp`` psp (binary): int icube, int nfft, double unit, char atom[2],
  double amass, double zv, int lmax, double rc[lmax+1], double
  vnlnrm[lmax^2], double vl[nfft3d], double vnl[lmax^2*nfft3d] --
  ckbppv3/kbppv3.c:138-150, read at ccpsdv3/main.c:264-284.
* IONIN (text): nkatm, per kind "'file' lmax", nion, per ion
  "katm r2x r2y r2z r1x r1y r1z" -- ccpsdv3/main.c:218-251.
* CONTROL (text): "ispin imove / icube unit / dt fmass / inner outer /
  tole tolc tolr" -- ccpsdv3/main.c:202-212.
"""
from __future__ import annotations

import os
import struct
from typing import Sequence, Tuple

import numpy as np


def write_elcin(path: str, icube: int, nfft: int, unit: float, ispin: int,
                ne: Sequence[int], c: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("=iidi2i", icube, nfft, unit, ispin, int(ne[0]), int(ne[1])))
        f.write(np.ascontiguousarray(c, dtype=np.float64).tobytes())


def read_elcin(path: str):
    with open(path, "rb") as f:
        hdr = f.read(struct.calcsize("=iidi2i"))
        icube, nfft, unit, ispin, ne0, ne1 = struct.unpack("=iidi2i", hdr)
        n2ft3d = (nfft + 2) * nfft * nfft
        c = np.frombuffer(f.read(8 * n2ft3d * (ne0 + ne1)), dtype=np.float64).copy()
    return dict(icube=icube, nfft=nfft, unit=unit, ispin=ispin, ne=(ne0, ne1), c=c)


def write_vpp(path: str, icube: int, nfft: int, unit: float, atom: str, amass: float,
              zv: float, lmax: int, rc: Sequence[float], vnlnrm: np.ndarray,
              vl: np.ndarray, vnl: np.ndarray, pad: str = " ") -> None:
    """pad fills a one-letter atom name: the psp formatter's own files carry
    the string terminator there (pad="\\0", its fscanf("%s") into char[2])."""
    lmmax = lmax * lmax
    nfft3d = (nfft // 2 + 1) * nfft * nfft
    a = (atom + pad + pad)[:2].encode("latin-1")
    with open(path, "wb") as f:
        f.write(struct.pack("=iid", icube, nfft, unit))
        f.write(a)
        f.write(struct.pack("=ddi", amass, zv, lmax))
        f.write(np.asarray(rc, dtype=np.float64)[:lmax + 1].tobytes())
        f.write(np.asarray(vnlnrm, dtype=np.float64)[:lmmax].tobytes())
        f.write(np.asarray(vl, dtype=np.float64)[:nfft3d].tobytes())
        f.write(np.asarray(vnl, dtype=np.float64)[:lmmax * nfft3d].tobytes())


def write_ionin(path: str, files: Sequence[Tuple[str, int]], katm: Sequence[int],
                r2: np.ndarray, r1: np.ndarray) -> None:
    r2 = np.asarray(r2).reshape(-1, 3)
    r1 = np.asarray(r1).reshape(-1, 3)
    with open(path, "w") as f:
        f.write("%d\n" % len(files))
        for name, lmax in files:
            f.write(" '%s '   %d\n" % (name, lmax))
        f.write("%d\n" % len(katm))
        for k, a, b in zip(katm, r2, r1):
            f.write("%d %.17e %.17e %.17e\n   %.17e %.17e %.17e\n" % (int(k) + 1, *a, *b))


def write_control(path: str, ispin: int, imove: int, icube: int, unit: float, dt: float,
                  fmass: float, inner: int, outer: int, tole: float = 1e-9,
                  tolc: float = 1e-9, tolr: float = 1e-4) -> None:
    with open(path, "w") as f:
        f.write("%d %d\n%d %.17e\n%.17e %.17e\n%d %d\n%.6e %.6e %.6e\n"
                % (ispin, imove, icube, unit, dt, fmass, inner, outer, tole, tolc, tolr))


def write_reference_inputs(directory: str, inp, inner: int, outer: int,
                           tole: float = 1e-9, tolc: float = 1e-9, tolr: float = 1e-4) -> None:
    """All four inputs of the reference's main() for an inputs.CpsdInputs."""
    spec = inp.spec
    os.makedirs(directory, exist_ok=True)
    write_elcin(os.path.join(directory, "ELCIN"), spec.icube, inp.nfft, spec.unit, inp.ispin,
                inp.ne, inp.c2)
    files = []
    for ia, sp in enumerate(spec.species):
        name = "%s%d.vpp" % (sp.symbol, ia)
        write_vpp(os.path.join(directory, name), spec.icube, inp.nfft, spec.unit, sp.symbol,
                  sp.amass, sp.zv, sp.lmax, [sp.rc_loc] + [sp.rc_kb] * sp.lmax,
                  inp.vnlnrm[ia * 9:(ia + 1) * 9],
                  inp.vl[ia * inp.nfft3d:(ia + 1) * inp.nfft3d],
                  inp.vnl[ia * 9 * inp.nfft3d:(ia + 1) * 9 * inp.nfft3d])
        files.append((name, sp.lmax))
    write_ionin(os.path.join(directory, "IONIN"), files, inp.katm, inp.r2, inp.r2)
    write_control(os.path.join(directory, "CONTROL"), inp.ispin, spec.move, spec.icube,
                  spec.unit, spec.dt, spec.fmass, inner, outer, tole, tolc, tolr)


def parse_reference_stdout(text: str):
    """Per outer iteration (step, E, deltae, deltac, deltar) and the final energy table."""
    rows = []
    final = {}
    keys = {
        "total     energy": 0, "total orbital energy": 1, "hartree   energy": 2,
        "exc-corr  energy": 3, "ion-ion   energy": 4, "KS kinetic energy": 5,
        "KS V_l energy": 6, "KS V_nl energy": 7, "KS V_Hart energy": 8, "KS V_xc energy": 9,
    }
    in_iter = False
    for line in text.splitlines():
        if "iteration =====" in line:
            in_iter = True
            continue
        if in_iter:
            parts = line.split()
            if len(parts) == 5:
                try:
                    rows.append((int(parts[0]),) + tuple(float(p) for p in parts[1:]))
                    continue
                except ValueError:
                    pass
            if line.strip().startswith("***"):
                continue
        s = line.strip()
        for k, idx in keys.items():
            if s.startswith(k):
                final[idx] = float(s.split(":")[1].split("(")[0])
    return rows, final


def parse_reference_epilogue(text: str):
    """The epilogue tables main.c prints: the orthonormality rows
    (ms, i, j, <c1_i|c1_j>), 1-based as printed (main.c:455-467), and the
    orbital energies in Hartree (main.c:518-530; with two spins a line holds
    one value of each)."""
    ortho, eig = [], []
    mode = None
    for line in text.splitlines():
        st = line.strip()
        if st.startswith("orthonormality"):
            mode = "o"
            continue
        if st.startswith("orbital energies"):
            mode = "e"
            continue
        if mode == "o":
            parts = st.split()
            if len(parts) == 4:
                try:
                    ortho.append((int(parts[0]), int(parts[1]), int(parts[2]), float(parts[3])))
                    continue
                except ValueError:
                    pass
            if st:
                mode = None
        elif mode == "e":
            if "eV)" not in st:
                if st:
                    mode = None
                continue
            for chunk in st.split("eV)"):
                if "(" in chunk:
                    eig.append(float(chunk.split("(")[0]))
    return ortho, eig


def read_vpp(path: str):
    """A ``.vpp`` file (the formatter's DATAOUT), as main.c:264-284 reads it."""
    with open(path, "rb") as f:
        icube, nfft, unit = struct.unpack("=iid", f.read(16))
        atom = f.read(2).decode("latin-1")
        amass, zv, lmax = struct.unpack("=ddi", f.read(20))
        nfft3d = (nfft // 2 + 1) * nfft * nfft
        lmmax = lmax * lmax
        rd = lambda m: np.frombuffer(f.read(8 * m), dtype=np.float64).copy()  # noqa: E731
        rc = rd(lmax + 1)
        vnlnrm = rd(lmmax)
        vl = rd(nfft3d)
        vnl = rd(lmmax * nfft3d)
    return dict(icube=icube, nfft=nfft, unit=unit, atom=atom, amass=amass, zv=zv, lmax=lmax, rc=rc,
                vnlnrm=vnlnrm, vl=vl, vnl=vnl)


def write_aimd_param(path: str, icube: int, unit: float, nfft: int, ispin: int, ne: Sequence[int]) -> None:
    """aimd.param as dkbppv3.c / dmakepsi.c read it: icube, unit, nfft, ispin ne0 ne1."""
    with open(path, "w") as f:
        f.write("%d %.17e %d\n%d %d %d\n" % (icube, unit, nfft, ispin, int(ne[0]), int(ne[1])))


def write_psi0(path: str, waves) -> None:
    """PSI0.DAT: one row "i j k l" per band (cmakepsi/dmakepsi.c:93-107)."""
    with open(path, "w") as f:
        for i, j, k, l in waves:
            f.write(" %d %d %d %d\n" % (i, j, k, l))

