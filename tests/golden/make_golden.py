"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own serial C (Simple-CPSD ccpsdv3/*.c, compiled
unmodified by ``make -C oracle ref`` into oracle/_ref/) on the seeded
workloads and stores compact outputs:

* ``ref_<name>.npz`` -- per cpsd() call: E[0..9], deltae, deltac; after the
  last call: hml, lmd, the packed c2 of the first bands (coefficients on the
  cutoff sphere, in half-box index order) and the density checksums.
* ``ref_main_<name>.npz`` -- the reference's main() run from its own input
  files (ELCIN, CONTROL, IONIN, .vpp written by cpsd_b200.refio): the printed
  per-iteration lines and final energy table.  This pins the table setup
  (G, mask at the grid cutoff, tg/vc/vg, Ewald constant) to main.c's.
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
    rows, final = refio.parse_reference_stdout(out)
    np.savez_compressed(os.path.join(HERE, "ref_main_%s.npz" % name), rows=np.array(rows),
                        final=np.array([final[i] for i in range(10)]), inner=np.array(inner),
                        outer=np.array(outer), ecut=np.array(spec.ecut_ry),
                        elcout_norms=np.array([np.sum(elc["c"].reshape(inp.nbands, -1)[b] ** 2)
                                               for b in range(inp.nbands)]))
    print("main(%s): %d iterations, E=%.10f" % (name, len(rows), final[0]))
    return input_digest(inp)


def main():
    ref = oracle.ReferenceBuild()
    digests = {}
    for name, mk, ncalls, inner, keep in CASES + MOVE_CASES:
        digests[name] = run_case(ref, name, mk, ncalls, inner, keep)
    digests["main_small_diamond_24"] = run_main("small_diamond_24", lambda: configs.small_diamond(24, 4), 2, 3)
    with open(os.path.join(HERE, "inputs.json"), "w") as f:
        json.dump(digests, f, indent=1, sort_keys=True)
    with open(os.path.join(REPO, "oracle", "_ref", "BUILD_INFO.txt")) as f:
        info = f.read()
    with open(os.path.join(HERE, "REFERENCE_BUILD.txt"), "w") as f:
        f.write("Fixtures generated by tests/golden/make_golden.py from the reference build:\n" + info)


if __name__ == "__main__":
    main()
