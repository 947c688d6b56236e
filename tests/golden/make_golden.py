"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own serial C (Simple-CPSD ccpsdv3/*.c, compiled
unmodified by ``make -C oracle ref`` into oracle/_ref/) on the seeded
workloads and stores compact outputs:

* ``ref_<name>.npz`` -- per cpsd() call: E[0..9], deltae, deltac; after the
  last call: hml, lmd, the packed c2 of the first bands (coefficients on the
  cutoff sphere, in half-box index order) and the density checksums.
* ``ref_main_<name>.npz`` -- the reference's main() run from its own input
  files (ELCIN, CONTROL, IONIN, .vpp written by cpsd_b200.refio): the printed
  per-iteration lines and final energy table, the printed epilogue tables
  (orthonormality, orbital energies), the packed c1 of ELCOUT and the text
  of IONOUT.  This pins the table setup (G, mask at the grid cutoff,
  tg/vc/vg, Ewald constant) and the epilogue to main.c's.
* ``ref_epi_<name>.npz`` -- the epilogue of main.c:452-487 after the last
  call, with the reference's own gcdotc and eigsrt and the LAPACK dsyev /
  BLAS dgemm of the OpenBLAS the reference build links: the orthonormality
  matrix, eigenvalues, eigenvectors and the packed rotated c1 (first 8 bands).
* ``inputs.json`` -- SHA-256 of the generated inputs, so a change of the
  input builder is caught before parity is compared.

Usage (needs the reference tree and ``make -C oracle ref``):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "simple-cpsd_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

from cpsd_b200 import configs, inputs, refio  # noqa: E402
import oracle  # noqa: E402

# (name, spec builder, number of cpsd() calls, inner steps per call, bands of c2 kept)
CASES = [
    ("small_h2_16", lambda: configs.small_h2(16), 3, 2, 1),
    ("small_diamond_24", lambda: configs.small_diamond(24, 4), 3, 2, 4),
    ("small_diamond_32", lambda: configs.small_diamond(32, 5, ecut=25.0), 2, 2, 5),
    ("small_diamond_48", lambda: configs.small_diamond(48, 6, ecut=30.0), 2, 2, 6),
    ("h2_dimer_32", lambda: configs.h2_dimer_32(), 200, 1, 1),
    ("diamond8_64", lambda: configs.diamond8_64(), 4, 2, 4),
]

# epilogue (main.c:452-487) after the calls: (name, spec builder, calls, inner)
EPILOGUE_CASES = [
    ("small_diamond_24", lambda: configs.small_diamond(24, 4), 3, 2),
    ("small_diamond_32_40", lambda: configs.small_diamond(32, 40, ecut=25.0, seed=12), 2, 2),
]


def _moving(spec):
    spec.move = 1
    return spec


# move = 1 (ion forces and the ion SD step): positions and forces per call
MOVE_CASES = [
    ("move_small_h2_16", lambda: _moving(configs.small_h2(16)), 3, 2, 1),
    ("move_small_diamond_24", lambda: _moving(configs.small_diamond(24, 4)), 3, 2, 4),
    ("move_small_diamond_32", lambda: _moving(configs.small_diamond(32, 40, ecut=25.0, seed=12)), 2, 2, 4),
]


def input_digest(inp) -> str:
    h = hashlib.sha256()
    for a in (inp.c2, inp.vl, inp.vnl, inp.vnlnrm, inp.tg, inp.vc, inp.vg, inp.masker1, inp.r2,
              np.array([inp.cewald, inp.omega, inp.rcut])):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def packed(inp, c: np.ndarray, nbands: int) -> np.ndarray:
    pts = np.flatnonzero(inp.masker1)
    cc = c.reshape(inp.nbands, inp.nfft3d, 2)
    return np.ascontiguousarray(cc[:nbands, pts, :])


def run_case(ref, name, mk, ncalls, inner, keep):
    spec = mk()
    inp = inputs.build_inputs(spec)
    st = oracle.State(inp)
    E, de, dc, dr, r2, fion = [], [], [], [], [], []
    for _ in range(ncalls):
        ref.run(inp, inner, st)
        E.append(st.E.copy())
        de.append(st.deltae)
        dc.append(st.deltac)
        dr.append(st.deltar)
        r2.append(st.r2.copy())
        fion.append(st.fion.copy())
    dn = st.dn.reshape(inp.ispin, inp.nfft, inp.nfft, inp.nfft + 2)[..., :inp.nfft]
    out = dict(E=np.array(E), deltae=np.array(de), deltac=np.array(dc), hml=st.hml, lmd=st.lmd,
               c2=packed(inp, st.c2, keep), cpsi=packed(inp, st.cpsi, keep),
               dn_sum=dn.sum(axis=(1, 2, 3)), dn_sq=(dn * dn).sum(axis=(1, 2, 3)),
               dn_plane0=np.ascontiguousarray(dn[:, 0]), inner=np.array(inner))
    if spec.move:
        out.update(deltar=np.array(dr), r2=np.array(r2), fion=np.array(fion), r1=st.r1.copy())
    np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), **out)
    print("%-18s calls=%d inner=%d  E=%.12f" % (name, ncalls, inner, st.E[0]))
    return input_digest(inp)


def run_epilogue(ref, name, mk, ncalls, inner):
    from scipy.linalg import blas
    inp = inputs.build_inputs(mk())
    st = oracle.State(inp)
    for _ in range(ncalls):
        ref.run(inp, inner, st)

    def ref_sort(D, V):  # the reference's eigsrt on a column-major copy
        n = len(D)
        Vc = np.ascontiguousarray(V.T).ravel()
        ref.eigsrt(D, Vc, n)
        V[:, :] = Vc.reshape(n, n).T

    ep = oracle.epilogue(inp, st, ref.gcdotc, sort=ref_sort,
                         matmul=lambda A, B: blas.dgemm(1.0, np.asfortranarray(A), np.asfortranarray(B)))
    np.savez_compressed(os.path.join(HERE, "ref_epi_%s.npz" % name), ortho=ep["ortho"], eig=ep["eig"],
                        vec=ep["vec"], c1=packed(inp, ep["c1"], min(8, inp.nbands)), hml=st.hml,
                        E=st.E.copy(), ncalls=np.array(ncalls), inner=np.array(inner))
    print("epilogue(%s): eig %s" % (name, np.array2string(ep["eig"][:4], precision=6)))
    return input_digest(inp)


def run_main(name, mk, inner, outer):
    """The reference's own main() on files written in its formats (grid cutoff)."""
    spec = mk()
    _, _, unitg = inputs.get_cube(spec.icube, spec.unit)
    h = spec.nfft // 2
    spec.ecut_ry = (unitg[0] * h) ** 2 + (unitg[1] * h) ** 2 + (unitg[2] * h) ** 2  # main.c:161-164
    inp = inputs.build_inputs(spec)
    exe = os.path.join(REPO, "oracle", "_ref", "dcpsdv3.x")
    with tempfile.TemporaryDirectory() as d:
        refio.write_reference_inputs(d, inp, inner=inner, outer=outer)
        out = subprocess.run([exe], cwd=d, capture_output=True, check=True).stdout.decode("utf-8", "replace")
        elc = refio.read_elcin(os.path.join(d, "ELCOUT"))
        with open(os.path.join(d, "IONOUT")) as f:
            ionout = f.read()
    rows, final = refio.parse_reference_stdout(out)
    ortho, eig = refio.parse_reference_epilogue(out)
    np.savez_compressed(os.path.join(HERE, "ref_main_%s.npz" % name), rows=np.array(rows),
                        final=np.array([final[i] for i in range(10)]), inner=np.array(inner),
                        outer=np.array(outer), ecut=np.array(spec.ecut_ry),
                        elcout_norms=np.array([np.sum(elc["c"].reshape(inp.nbands, -1)[b] ** 2)
                                               for b in range(inp.nbands)]),
                        ortho_printed=np.array(ortho), eig_printed=np.array(eig),
                        elcout_header=np.array([elc["icube"], elc["nfft"], elc["ispin"], *elc["ne"]]),
                        elcout_unit=np.array(elc["unit"]), elcout_c1=packed(inp, elc["c"], inp.nbands),
                        ionout=np.array(ionout))
    print("main(%s): %d iterations, E=%.10f" % (name, len(rows), final[0]))
    return input_digest(inp)


def main():
    ref = oracle.ReferenceBuild()
    digests = {}
    for name, mk, ncalls, inner, keep in CASES + MOVE_CASES:
        digests[name] = run_case(ref, name, mk, ncalls, inner, keep)
    for name, mk, ncalls, inner in EPILOGUE_CASES:
        digests["epi_" + name] = run_epilogue(ref, name, mk, ncalls, inner)
    digests["main_small_diamond_24"] = run_main("small_diamond_24", lambda: configs.small_diamond(24, 4), 2, 3)
    with open(os.path.join(HERE, "inputs.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)
    with open(os.path.join(REPO, "oracle", "_ref", "BUILD_INFO.txt")) as f:
        info = f.read()
    with open(os.path.join(HERE, "REFERENCE_BUILD.txt"), "w") as f:
        f.write("Fixtures generated by tests/golden/make_golden.py from the reference build:\n" + info)


if __name__ == "__main__":
    main()
