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
* ``ref_kbpp_<name>.npz`` -- the reference's own kbpp() (ckbppv3/dkbppv3.c,
  oracle/_ref/libkbpp_ref.so) on a seeded radial table (cpsd_b200.psp):
  vl, vnl, vnlnrm and vp as the call leaves it; ``ref_kbpp_main.npz`` --
  the formatter program itself (oracle/_ref/dkbppv3.x) on aimd.param, the
  table file and its "highest L" prompt: the DATAOUT bytes.
* ``ref_makepsi.npz`` -- the reference's initial-orbital program
  (oracle/_ref/dmakepsi.x) on aimd.param and a PSI0.DAT: the ELCIN it
  writes, as header plus the nonzero entries.
* ``inputs.json`` -- SHA-256 of the generated inputs, so a change of the
  input builder is caught before parity is compared.

Usage (needs the reference tree and ``make -C oracle ref``):
    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py NAME ...   # only these ref_<NAME> cases
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

from cpsd_b200 import configs, inputs, psp, refio  # noqa: E402
import oracle  # noqa: E402

# (name, spec builder, number of cpsd() calls, inner steps per call, bands of c2 kept)
CASES = [
    ("small_h2_16", lambda: configs.small_h2(16), 3, 2, 1),
    ("small_diamond_24", lambda: configs.small_diamond(24, 4), 3, 2, 4),
    ("small_diamond_32", lambda: configs.small_diamond(32, 5, ecut=25.0), 2, 2, 5),
    ("small_diamond_48", lambda: configs.small_diamond(48, 6, ecut=30.0), 2, 2, 6),
    ("h2_dimer_32", lambda: configs.h2_dimer_32(), 200, 1, 1),
    ("diamond8_64", lambda: configs.diamond8_64(), 4, 2, 4),
    # spin-polarised, from the reference's plane-wave start (configs.spin_h2)
    ("spin_h2_16", lambda: configs.spin_h2(16), 3, 2, 3),
    ("spin_diamond_24", lambda: configs.spin_diamond(24, ne=(4, 3)), 3, 2, 7),
    # the 128^3 / 64-atom / 128-band cell of the precision study: one call of
    # two SD steps (about four minutes of reference CPU time)
    ("diamond64_128", lambda: configs.diamond64_128(), 1, 2, 1),
]

# cells of the 48-cell batched draw (configs.batched_cells(0)): one per grid
# size, the most bands, mixed H/C kinds; (index in the draw, calls, inner, bands kept)
BATCH_DRAW_CASES = [(0, 2, 2, 2), (9, 2, 2, 1), (13, 2, 2, 1), (45, 2, 2, 2)]

# epilogue (main.c:452-487) after the calls: (name, spec builder, calls, inner)
EPILOGUE_CASES = [
    ("small_diamond_24", lambda: configs.small_diamond(24, 4), 3, 2),
    ("small_diamond_32_40", lambda: configs.small_diamond(32, 40, ecut=25.0, seed=12), 2, 2),
    ("spin_diamond_24", lambda: configs.spin_diamond(24, ne=(4, 3)), 3, 2),
]


def _moving(spec):
    spec.move = 1
    return spec


# move = 1 (ion forces and the ion SD step): positions and forces per call
MOVE_CASES = [
    ("move_small_h2_16", lambda: _moving(configs.small_h2(16)), 3, 2, 1),
    ("move_small_diamond_24", lambda: _moving(configs.small_diamond(24, 4)), 3, 2, 4),
    ("move_small_diamond_32", lambda: _moving(configs.small_diamond(32, 40, ecut=25.0, seed=12)), 2, 2, 4),
    ("move_spin_diamond_24", lambda: _moving(configs.spin_diamond(24, ne=(4, 3))), 3, 2, 7),
]


# kbpp(): (name, lmax, table seed, nfft); the cube is icube 1, a = 10.26
KBPP_CASES = [("l1", 1, 1, 12), ("l2", 2, 2, 12), ("l3", 3, 3, 12)]
KBPP_UNIT = 10.26


def plane_waves(nfft: int, count: int):
    """PSI0.DAT-style rows: half-box G by increasing |k|^2 (ties in loop
    order), the first as l = 0, then each G as l = -1 and l = +1."""
    h = nfft // 2
    ks = [(i, j, k) for k in range(-h + 1, h) for j in range(-h + 1, h) for i in range(0, h)
          if (i, j, k) != (0, 0, 0) and (i > 0 or j > 0 or (j == 0 and k > 0))]
    ks.sort(key=lambda t: t[0] ** 2 + t[1] ** 2 + t[2] ** 2)
    rows = [(0, 0, 0, 0)]
    for t in ks:
        rows += [t + (-1,), t + (1,)]
    return rows[:count]


def table_digest(t) -> str:
    h = hashlib.sha256()
    for a in (t.rho, t.vp, t.wp, t.rc, np.array([t.zv, t.amass, t.drho, t.lmax])):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def run_kbpp(name, lmax, seed, nfft):
    t = psp.radial_table(lmax, seed=seed)
    _, _, unitg = inputs.get_cube(1, KBPP_UNIT)
    nfft3d = (nfft // 2 + 1) * nfft * nfft
    vl, vnl, vnlnrm, vp = oracle.reference_kbpp(t.zv, lmax, t.rho, t.vp, t.wp, t.drho,
                                                inputs.get_g(nfft, unitg), nfft3d)
    np.savez_compressed(os.path.join(HERE, "ref_kbpp_%s.npz" % name), vl=vl, vnl=vnl, vnlnrm=vnlnrm, vp=vp,
                        lmax=np.array(lmax), seed=np.array(seed), nfft=np.array(nfft))
    print("kbpp(%s): vl(G=0)=%.10f vnlnrm=%s" % (name, vl[0], np.array2string(vnlnrm, precision=6)))
    return table_digest(t)


def run_kbpp_main(lmax=3, seed=3, nfft=12, highest_l=2):
    """The formatter program: aimd.param + table file + the prompt's answer."""
    t = psp.radial_table(lmax, seed=seed)
    exe = os.path.join(REPO, "oracle", "_ref", "dkbppv3.x")
    with tempfile.TemporaryDirectory() as d:
        refio.write_aimd_param(os.path.join(d, "aimd.param"), 1, KBPP_UNIT, nfft, 1, (4, 0))
        psp.write_table(os.path.join(d, "C.dat"), t)
        subprocess.run([exe, "C.dat"], cwd=d, input=b"%d\n" % highest_l, capture_output=True, check=True)
        with open(os.path.join(d, "DATAOUT"), "rb") as f:
            data = f.read()
    np.savez_compressed(os.path.join(HERE, "ref_kbpp_main.npz"), dataout=np.frombuffer(data, dtype=np.uint8),
                        lmax=np.array(lmax), seed=np.array(seed), nfft=np.array(nfft),
                        highest_l=np.array(highest_l))
    print("dkbppv3.x: DATAOUT %d bytes" % len(data))
    return table_digest(t)


def run_makepsi(nfft=12, ispin=2, ne=(6, 4)):
    rows = plane_waves(nfft, ne[0])
    exe = os.path.join(REPO, "oracle", "_ref", "dmakepsi.x")
    with tempfile.TemporaryDirectory() as d:
        refio.write_aimd_param(os.path.join(d, "aimd.param"), 1, KBPP_UNIT, nfft, ispin, ne)
        refio.write_psi0(os.path.join(d, "PSI0.DAT"), rows)
        subprocess.run([exe, "ELCIN"], cwd=d, capture_output=True, check=True)
        elc = refio.read_elcin(os.path.join(d, "ELCIN"))
    c = elc["c"]
    nz = np.flatnonzero(c)
    np.savez_compressed(os.path.join(HERE, "ref_makepsi.npz"), rows=np.array(rows, dtype=np.int32),
                        header=np.array([elc["icube"], elc["nfft"], elc["ispin"], *elc["ne"]]),
                        unit=np.array(elc["unit"]), size=np.array(c.size), nz=nz, values=c[nz])
    print("dmakepsi.x: %d bands, %d nonzeros" % (sum(ne), len(nz)))


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
    c2all = packed(inp, st.c2, inp.nbands)
    out = dict(E=np.array(E), deltae=np.array(de), deltac=np.array(dc), hml=st.hml, lmd=st.lmd,
               c2=packed(inp, st.c2, keep), cpsi=packed(inp, st.cpsi, keep),
               dn_sum=dn.sum(axis=(1, 2, 3)), dn_sq=(dn * dn).sum(axis=(1, 2, 3)),
               dn_plane0=np.ascontiguousarray(dn[:, 0]), inner=np.array(inner),
               # every band, size-independent: sum of squares and of the
               # coefficients over the sphere
               c2_band_sq=(c2all * c2all).sum(axis=(1, 2)), c2_band_sum=c2all.sum(axis=(1, 2)))
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


def batch_draw_case(index):
    return lambda: configs.batched_cells(0)[index]


def main(only=None):
    ref = oracle.ReferenceBuild()
    path = os.path.join(HERE, "inputs.json")
    digests = {}
    if os.path.exists(path):
        with open(path) as f:
            digests = json.load(f)
    cases = CASES + MOVE_CASES + [("batch0_%02d" % i, batch_draw_case(i), nc, inner, keep)
                                  for i, nc, inner, keep in BATCH_DRAW_CASES]
    if only:
        for name, mk, ncalls, inner, keep in cases:
            if name in only:
                digests[name] = run_case(ref, name, mk, ncalls, inner, keep)
        with open(path, "w") as f:
            json.dump(digests, f, indent=1, sort_keys=True)
        return
    for name, mk, ncalls, inner, keep in cases:
        digests[name] = run_case(ref, name, mk, ncalls, inner, keep)
    for name, mk, ncalls, inner in EPILOGUE_CASES:
        digests["epi_" + name] = run_epilogue(ref, name, mk, ncalls, inner)
    digests["main_small_diamond_24"] = run_main("small_diamond_24", lambda: configs.small_diamond(24, 4), 2, 3)
    for name, lmax, seed, nfft in KBPP_CASES:
        digests["kbpp_" + name] = run_kbpp(name, lmax, seed, nfft)
    digests["kbpp_main"] = run_kbpp_main()
    run_makepsi()
    with open(os.path.join(HERE, "inputs.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)
    with open(os.path.join(REPO, "oracle", "_ref", "BUILD_INFO.txt")) as f:
        info = f.read()
    with open(os.path.join(HERE, "REFERENCE_BUILD.txt"), "w") as f:
        f.write("Fixtures generated by tests/golden/make_golden.py from the reference build:\n" + info)


if __name__ == "__main__":
    main(set(sys.argv[1:]) or None)
