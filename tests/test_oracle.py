"""The oracle, pinned: FFT restatement vs numpy, tables vs the reference's
own code and its one numeric pin, the cpsd() restatement vs the golden
vectors generated by the reference build (tests/golden/make_golden.py)."""
import json
import sys
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, REPO
from cpsd_b200 import configs, inputs

import oracle

CASES = {
    "small_h2_16": (lambda: configs.small_h2(16), 3, 2),
    "small_diamond_24": (lambda: configs.small_diamond(24, 4), 3, 2),
    "small_diamond_32": (lambda: configs.small_diamond(32, 5, ecut=25.0), 2, 2),
    "small_diamond_48": (lambda: configs.small_diamond(48, 6, ecut=30.0), 2, 2),
    "h2_dimer_32": (lambda: configs.h2_dimer_32(), 200, 1),
    "diamond8_64": (lambda: configs.diamond8_64(), 4, 2),
    "spin_h2_16": (lambda: configs.spin_h2(16), 3, 2),
    "spin_diamond_24": (lambda: configs.spin_diamond(24, ne=(4, 3)), 3, 2),
    # cells of the 48-cell batched draw (make_golden.BATCH_DRAW_CASES): 32^3
    # with H and C kinds, 48^3 / 19 bands, 64^3 / 14 ions, 32^3 / 25 bands
    "batch0_00": (lambda: configs.batched_cells(0)[0], 2, 2),
    "batch0_09": (lambda: configs.batched_cells(0)[9], 2, 2),
    "batch0_13": (lambda: configs.batched_cells(0)[13], 2, 2),
    "batch0_45": (lambda: configs.batched_cells(0)[45], 2, 2),
}


def _moving(spec):
    spec.move = 1
    return spec


# move = 1: ion forces and the ion SD step (make_golden.MOVE_CASES)
MOVE_CASES = {
    "move_small_h2_16": (lambda: _moving(configs.small_h2(16)), 3, 2),
    "move_small_diamond_24": (lambda: _moving(configs.small_diamond(24, 4)), 3, 2),
    "move_small_diamond_32": (lambda: _moving(configs.small_diamond(32, 40, ecut=25.0, seed=12)), 2, 2),
    "move_spin_diamond_24": (lambda: _moving(configs.spin_diamond(24, ne=(4, 3))), 3, 2),
}
E_TOL = 1e-9  # Ha, total energy parity bar
F_TOL = 1e-9  # Ha/bohr, force parity bar


@pytest.mark.parametrize("n", [8, 12, 16, 24, 32, 48, 64])
def test_fft_restatement_matches_numpy(restatement, n):
    """cr_fft3b/rc_fft3f restatement == pocketfft up to rounding (fftpack3d.f:22-196)."""
    rng = np.random.default_rng(n)
    nh = n // 2 + 1
    x = rng.standard_normal((n, n, n))
    A = np.zeros((n, n, n + 2))
    A[:, :, :n] = x
    A = A.reshape(-1).copy()
    restatement.rc_fft3f(A, n)
    ref = np.fft.rfftn(x)
    got = A.view(np.complex128).reshape(n, n, nh)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    C = rng.standard_normal((n, n, nh)) + 1j * rng.standard_normal((n, n, nh))
    B = np.ascontiguousarray(C).view(np.float64).reshape(-1).copy()
    restatement.cr_fft3b(B, n)
    refi = np.fft.irfftn(C, s=(n, n, n), axes=(0, 1, 2)) * n ** 3
    got = B.reshape(n, n, n + 2)
    assert np.abs(got[:, :, :n] - refi).max() <= 1e-13 * np.abs(refi).max()
    assert np.all(got[:, :, n:] == 0.0)  # pad zeroed, fftpack3d.f:90-91


def test_fft_roundtrip_is_n_cubed(restatement):
    n = 24
    rng = np.random.default_rng(1)
    A = np.zeros((n, n, n + 2))
    A[:, :, :n] = rng.standard_normal((n, n, n))
    x0 = A.copy()
    A = A.reshape(-1)
    restatement.rc_fft3f(A, n)
    restatement.cr_fft3b(A, n)
    assert np.allclose(A.reshape(n, n, n + 2)[:, :, :n], n ** 3 * x0[:, :, :n], rtol=0, atol=1e-10)


def test_masker_pins_nwave_8932():
    """The reference's only numeric pin: NWAVE=8932 for the 32^3 SC examples
    (Example0-double-serial/aimd.h:1), i.e. get_masker at the grid cutoff."""
    for a in (20.0, 26.0):
        _, _, unitg = inputs.get_cube(1, a)
        h = 16
        gcut = (unitg[0] * h) ** 2 + (unitg[1] * h) ** 2 + (unitg[2] * h) ** 2
        assert int(inputs.get_masker(32, gcut, unitg).sum()) == 8932


def test_workload_sphere_sizes():
    """npw of the named workloads (half sphere, get_masker loop bounds)."""
    got = {}
    for name in ("h2_dimer_32", "diamond8_64"):
        spec = configs.NAMED[name]()
        _, _, unitg = inputs.get_cube(1, spec.unit)
        got[name] = int(inputs.get_masker(spec.nfft, spec.ecut_ry, unitg).sum())
    assert got == {"h2_dimer_32": 10924, "diamond8_64": 2483}


@pytest.mark.skipif(not os.path.exists(oracle.REFERENCE_SO), reason="reference build absent")
def test_tables_match_reference_functions():
    """inputs.py get_cube/get_g/get_masker == the reference's C (bit for bit)."""
    ref = oracle.ReferenceBuild()
    for icube, a in ((1, 20.0), (1, 10.26), (2, 12.0), (3, 9.0)):
        v, ua, ug = ref.get_cube(icube, a)
        v2, ua2, ug2 = inputs.get_cube(icube, a)
        assert v == v2 and np.array_equal(ua, ua2) and np.array_equal(ug, ug2)
        for n in (16, 24, 32):
            assert np.array_equal(ref.get_g(n, ug), inputs.get_g(n, ug2))
            for cut in (5.0, 12.0, 40.0):
                assert np.array_equal(ref.get_masker(n, cut, ug), inputs.get_masker(n, cut, ug2))


def test_inputs_match_fixture_digests():
    """The seeded inputs are the ones the fixtures were generated from."""
    sys.path.insert(0, GOLDEN)
    from make_golden import input_digest  # noqa: E402
    with open(os.path.join(GOLDEN, "inputs.json")) as f:
        want = json.load(f)
    for name, (mk, _, _) in list(CASES.items()) + list(MOVE_CASES.items()):
        assert input_digest(inputs.build_inputs(mk())) == want[name], name
    for name, mk in EPI_CASES.items():
        assert input_digest(inputs.build_inputs(mk())) == want["epi_" + name], name
    # the 128^3 cell's fixture is checked against the GPU path only (one
    # reference call of two steps takes minutes on the host)
    assert input_digest(inputs.build_inputs(configs.diamond64_128())) == want["diamond64_128"]


def test_orbitals_orthonormal_and_hermitian():
    inp = inputs.build_inputs(configs.small_diamond(24, 4))
    nh = inp.nfft // 2 + 1
    w = inputs.gamma_weights(inp.nfft)
    C = inp.c2.reshape(inp.nbands, -1).view(np.complex128)
    S = np.einsum("p,ap,bp->ab", w, C.conj(), C).real
    assert np.allclose(S, np.eye(inp.nbands), atol=1e-13)
    partner = inputs.hermitian_partner(inp.nfft)
    plane = np.arange(inp.nfft3d)[::nh]
    assert np.allclose(C[:, plane], np.conj(C[:, partner[plane]]), atol=0)
    assert np.all(C[:, inp.masker1 == 0] == 0)


def _run(R, mk, ncalls, inner):
    inp = inputs.build_inputs(mk())
    st = oracle.State(inp)
    rows = []
    for _ in range(ncalls):
        R.run(inp, inner, st)
        rows.append((st.E.copy(), st.deltae, st.deltac))
    return inp, st, rows


def packed(inp, c, nbands):
    pts = np.flatnonzero(inp.masker1)
    return c.reshape(inp.nbands, inp.nfft3d, 2)[:nbands, pts, :]


@pytest.mark.parametrize("name", list(CASES))
def test_restatement_matches_reference_build(restatement, golden, name):
    """The C restatement reproduces the reference's own cpsd() (golden vectors)."""
    mk, ncalls, inner = CASES[name]
    g = golden(name)
    inp, st, rows = _run(restatement, mk, ncalls, inner)
    E = np.array([r[0] for r in rows])
    assert np.abs(E[:, 0] - g["E"][:, 0]).max() < E_TOL
    assert np.abs(E - g["E"]).max() < 10 * E_TOL
    assert np.abs(np.array([r[1] for r in rows]) - g["deltae"]).max() < 1e-8
    assert np.abs(np.array([r[2] for r in rows]) - g["deltac"]).max() < 1e-9
    assert np.abs(st.lmd - g["lmd"]).max() < 1e-9
    assert np.abs(st.hml - g["hml"]).max() < 1e-9
    keep = g["c2"].shape[0]
    assert np.abs(packed(inp, st.c2, keep) - g["c2"]).max() < 1e-10
    assert np.abs(packed(inp, st.cpsi, keep) - g["cpsi"]).max() < 1e-10


@pytest.mark.parametrize("name", list(MOVE_CASES))
def test_restatement_matches_reference_build_with_ion_motion(restatement, golden, name):
    """move = 1: energies, forces, positions and deltar of every call against
    the reference's own cpsd() (golden vectors)."""
    mk, ncalls, inner = MOVE_CASES[name]
    g = golden(name)
    inp = inputs.build_inputs(mk())
    st = oracle.State(inp)
    for k in range(ncalls):
        restatement.run(inp, inner, st)
        assert abs(st.E[0] - g["E"][k, 0]) < E_TOL
        assert np.abs(st.fion - g["fion"][k]).max() < F_TOL
        assert np.abs(st.r2 - g["r2"][k]).max() < 1e-12
        assert abs(st.deltar - g["deltar"][k]) < F_TOL
    assert np.abs(st.lmd - g["lmd"]).max() < 1e-9


def test_restatement_matches_reference_main(restatement):
    """Same run as the reference's main() from its own files (printed digits)."""
    g = np.load(os.path.join(GOLDEN, "ref_main_small_diamond_24.npz"))
    spec = configs.small_diamond(24, 4)
    spec.ecut_ry = float(g["ecut"])
    inp = inputs.build_inputs(spec)
    st = oracle.State(inp)
    for row in g["rows"]:
        restatement.run(inp, int(g["inner"]), st)
        step, e, de, dc, dr = row
        assert abs(st.E[0] - e) <= 1e-10 * max(1.0, abs(e)) + 1e-9
        assert abs(st.deltae - de) <= 1e-5 * abs(de) + 1e-12
        assert abs(st.deltac - dc) <= 1e-5 * abs(dc) + 1e-12
    assert np.allclose(st.E, g["final"], rtol=1e-9, atol=1e-9)


def test_lagrange_off_by_one_quirk_single_band(restatement):
    """With one band the reference's convergence test reads sa1 (cpsd.c:471)
    and never passes: every step runs the full 30 iterations ("ierr=10")."""
    inp = inputs.build_inputs(configs.small_h2(16))
    st = oracle.State(inp)
    restatement.run(inp, 3, st)
    assert st.lagrange_fail == 3


# epilogue of main.c:452-487 (tests/golden/make_golden.py EPILOGUE_CASES)
EPI_CASES = {
    "small_diamond_24": lambda: configs.small_diamond(24, 4),
    "small_diamond_32_40": lambda: configs.small_diamond(32, 40, ecut=25.0, seed=12),
    "spin_diamond_24": lambda: configs.spin_diamond(24, ne=(4, 3)),
}


def eig_blocks(inp, g):
    """Per spin: (offset into hml's layout, size m, offset into eig)."""
    ne0 = int(inp.ne[0])
    return [(ms * ne0 * ne0, int(inp.ne[ms]), ms * ne0) for ms in range(inp.ispin) if int(inp.ne[ms]) > 0]


def vector_tolerances(inp, g):
    """Eigenvectors move by about (error in hml) / (eigenvalue gap): the
    bars for the vectors and the rotated orbitals grow as 1 / the smallest
    gap of the case (1e-8 and 1e-9 for gaps above 1e-3 Ha)."""
    gap = min(np.abs(np.diff(g["eig"][e0:e0 + m])).min() if m > 1 else 1.0 for _, m, e0 in eig_blocks(inp, g))
    return max(1e-8, 1e-11 / gap), max(1e-9, 1e-12 / gap)


def check_vectors(inp, g, vec, vec_tol):
    for o, m, _ in eig_blocks(inp, g):
        V, Vg = vec[o:o + m * m].reshape(m, m).T, g["vec"][o:o + m * m].reshape(m, m).T
        assert np.abs(align_columns(Vg, V) - Vg).max() < vec_tol
        assert np.abs(V.T @ V - np.eye(m)).max() < 1e-13


def align_columns(ref, got):
    """got with each column's sign chosen to match ref (an eigenvector's
    sign is not fixed by the problem); columns are the last axis."""
    s = np.sign((ref.reshape(-1, ref.shape[-1]) * got.reshape(-1, got.shape[-1])).sum(axis=0))
    s[s == 0] = 1.0
    return got * s


def align_bands(ref, got):
    """Packed orbitals (band, point, re/im): each band's sign chosen to match ref."""
    s = np.sign(np.einsum("bpc,bpc->b", ref, got))
    s[s == 0] = 1.0
    return got * s[:, None, None]


def _packed(inp, c, nb):
    pts = np.flatnonzero(inp.masker1)
    return c.reshape(inp.nbands, inp.nfft3d, 2)[:nb, pts, :]


@pytest.mark.parametrize("name", list(EPI_CASES))
def test_restatement_epilogue_matches_reference(restatement, golden, name):
    """Orthonormality table, eigenpairs of hml (descending, eigsrt order) and
    c1 <- c2 V, from the restatement's state, against the reference's own
    gcdotc / eigsrt and its LAPACK."""
    g = golden("epi_" + name)
    inp = inputs.build_inputs(EPI_CASES[name]())
    st = oracle.State(inp)
    for _ in range(int(g["ncalls"])):
        restatement.run(inp, int(g["inner"]), st)
    assert np.abs(st.hml - g["hml"]).max() < 1e-9
    ep = oracle.epilogue(inp, st, restatement.gcdotc)
    vec_tol, c1_tol = vector_tolerances(inp, g)
    assert np.abs(ep["ortho"] - g["ortho"]).max() < 1e-12
    assert np.abs(ep["eig"] - g["eig"]).max() < 1e-9
    for _, m, e0 in eig_blocks(inp, g):
        assert np.all(np.diff(ep["eig"][e0:e0 + m]) <= 0)
    check_vectors(inp, g, ep["vec"], vec_tol)
    got = _packed(inp, ep["c1"], g["c1"].shape[0])
    assert np.abs(align_bands(g["c1"], got) - g["c1"]).max() < c1_tol


def test_restatement_epilogue_matches_reference_main(restatement, tmp_path):
    """The reference main()'s printed epilogue tables, its ELCOUT and its
    IONOUT: the restatement's epilogue and this library's file writers
    (host code, no GPU) reproduce them."""
    from cpsd_b200 import api, refio
    g = np.load(os.path.join(GOLDEN, "ref_main_small_diamond_24.npz"))
    spec = configs.small_diamond(24, 4)
    spec.ecut_ry = float(g["ecut"])
    inp = inputs.build_inputs(spec)
    st = oracle.State(inp)
    for _ in g["rows"]:
        restatement.run(inp, int(g["inner"]), st)
    ep = oracle.epilogue(inp, st, restatement.gcdotc)
    m = int(inp.ne[0])
    for ms, i, j, w in g["ortho_printed"]:
        assert abs(ep["ortho"][int(i) - 1 + (int(j) - 1) * m] - w) <= 5e-8 * abs(w) + 1e-15
    assert np.allclose(ep["eig"], g["eig_printed"], rtol=1e-7, atol=0)
    got = _packed(inp, ep["c1"], inp.nbands)
    assert np.abs(align_bands(g["elcout_c1"], got) - g["elcout_c1"]).max() < 1e-9
    # ELCOUT and IONOUT through the library's writers
    path = str(tmp_path / "ELCOUT")
    api.write_elcout(path, inp, ep["c1"])
    back = refio.read_elcin(path)
    icube, nfft, ispin, ne0, ne1 = (int(x) for x in g["elcout_header"])
    assert (back["icube"], back["nfft"], back["ispin"], back["ne"]) == (icube, nfft, ispin, (ne0, ne1))
    assert back["unit"] == float(g["elcout_unit"])
    assert np.array_equal(back["c"], ep["c1"])
    assert os.path.getsize(path) == 4 * 2 + 8 + 4 * 3 + 8 * inp.nbands * inp.n2ft3d
    path = str(tmp_path / "IONOUT")
    api.write_ionout(path, inp, ["C0.vpp"], st.r2)
    with open(path) as f:
        assert f.read() == str(g["ionout"])



# input pipeline: tests/golden/make_golden.py KBPP_CASES, run_kbpp_main, run_makepsi
KBPP_CASES = {"l1": 1, "l2": 2, "l3": 3}


def kbpp_case(golden, name):
    from cpsd_b200 import psp
    g = golden("kbpp_" + name)
    t = psp.radial_table(int(g["lmax"]), seed=int(g["seed"]))
    nfft = int(g["nfft"])
    _, _, unitg = inputs.get_cube(1, 10.26)
    return g, t, inputs.get_g(nfft, unitg), (nfft // 2 + 1) * nfft * nfft


def assert_kbpp_close(got, g, rel):
    vl, vnl, vnlnrm, vp = got
    scale = np.abs(g["vl"]).max()
    assert np.abs(vl - g["vl"]).max() <= rel * scale
    if g["vnl"].size:
        assert np.abs(vnl - g["vnl"]).max() <= rel * np.abs(g["vnl"]).max()
    assert np.abs(vnlnrm - g["vnlnrm"]).max() <= rel * max(1.0, np.abs(g["vnlnrm"]).max())
    assert np.array_equal(vp, g["vp"])  # vp_l - vp_lmax, the same subtraction


def test_pipeline_tables_match_fixture_digests():
    sys.path.insert(0, GOLDEN)
    from make_golden import KBPP_CASES as KC, table_digest  # noqa: E402
    from cpsd_b200 import psp
    with open(os.path.join(GOLDEN, "inputs.json")) as f:
        want = json.load(f)
    for name, lmax, seed, _ in KC:
        assert table_digest(psp.radial_table(lmax, seed=seed)) == want["kbpp_" + name]
    assert table_digest(psp.radial_table(3, seed=3)) == want["kbpp_main"]


@pytest.mark.parametrize("name", list(KBPP_CASES))
def test_kbpp_restatement_matches_reference(golden, name):
    """kbpp() restated (numpy) against the reference's own compiled kbpp()."""
    g, t, G, nfft3d = kbpp_case(golden, name)
    got = oracle.kbpp(t.zv, t.lmax, t.rho, t.vp, t.wp, t.drho, G, nfft3d)
    assert_kbpp_close(got, g, 1e-13)


def test_psp_table_file_round_trip(tmp_path):
    """psp.write_table writes what dkbppv3.c main() reads; read_table reads it back."""
    from cpsd_b200 import psp
    t = psp.radial_table(3, seed=3)
    path = str(tmp_path / "C.dat")
    psp.write_table(path, t)
    b = psp.read_table(path)
    assert (b.atom, b.zv, b.amass, b.lmax, b.drho) == (t.atom, t.zv, t.amass, t.lmax, t.drho)
    for x, y in ((b.rc, t.rc), (b.rho, t.rho), (b.vp, t.vp), (b.wp, t.wp)):
        assert np.array_equal(x, y)


def test_makepsi_matches_reference():
    """The initial orbitals: the library's host code (no GPU needed) and the
    restatement against the ELCIN the reference's dmakepsi.x wrote, bit for
    bit (plane waves, Hermitian partners on kx = 0, spin 1 reusing rows)."""
    from cpsd_b200 import api
    g = np.load(os.path.join(GOLDEN, "ref_makepsi.npz"))
    icube, nfft, ispin, ne0, ne1 = (int(x) for x in g["header"])
    want = np.zeros(int(g["size"]))
    want[g["nz"]] = g["values"]
    for psi in (api.makepsi(nfft, ispin, (ne0, ne1), g["rows"]),
                oracle.makepsi(nfft, ispin, (ne0, ne1), g["rows"])):
        assert psi.size == want.size
        assert np.array_equal(psi, want)
    with pytest.raises(Exception):
        api.makepsi(nfft, ispin, (ne0, ne1), [(nfft, 0, 0, 0)] * ne0)  # kx outside the half box
