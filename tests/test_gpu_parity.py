"""GPU parity: the sm_100a path through the C ABI against the reference's
golden vectors and the oracle restatement.

Tolerance: the FP64 parity bar, |E - E_ref| < 1e-9 Ha for the total
energy of every cpsd() call; matrices and orbitals to ~1e-10.
"""
import os

import ctypes

import numpy as np
import pytest

from conftest import GOLDEN
from cpsd_b200 import api, configs, inputs, lib

import oracle

pytestmark = pytest.mark.gpu

E_TOL = 1e-9
CASES = {
    "small_h2_16": (lambda: configs.small_h2(16), 3, 2),
    "small_diamond_24": (lambda: configs.small_diamond(24, 4), 3, 2),
    "small_diamond_32": (lambda: configs.small_diamond(32, 5, ecut=25.0), 2, 2),
    "small_diamond_48": (lambda: configs.small_diamond(48, 6, ecut=30.0), 2, 2),
    "h2_dimer_32": (lambda: configs.h2_dimer_32(), 200, 1),
    "diamond8_64": (lambda: configs.diamond8_64(), 4, 2),
    # spin-polarised, from the reference's plane-wave start
    "spin_h2_16": (lambda: configs.spin_h2(16), 3, 2),
    "spin_diamond_24": (lambda: configs.spin_diamond(24, ne=(4, 3)), 3, 2),
    # the 128^3 / 64-atom / 128-band cell of the precision study
    "diamond64_128": (lambda: configs.diamond64_128(), 1, 2),
    # cells of the 48-cell batched draw, each on its own
    "batch0_00": (lambda: configs.batched_cells(0)[0], 2, 2),
    "batch0_09": (lambda: configs.batched_cells(0)[9], 2, 2),
    "batch0_13": (lambda: configs.batched_cells(0)[13], 2, 2),
    "batch0_45": (lambda: configs.batched_cells(0)[45], 2, 2),
}
BATCH_DRAW = {0: "batch0_00", 9: "batch0_09", 13: "batch0_13", 45: "batch0_45"}


def packed(inp, c, nbands):
    pts = np.flatnonzero(inp.masker1)
    return c.reshape(inp.nbands, inp.nfft3d, 2)[:nbands, pts, :]


def check_against_golden(inp, g, rows, st):
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
    dn = st.dn.reshape(inp.ispin, inp.nfft, inp.nfft, inp.nfft + 2)
    assert np.all(dn[..., inp.nfft:] == 0.0)
    dn = dn[..., :inp.nfft]
    assert np.allclose(dn.sum(axis=(1, 2, 3)), g["dn_sum"], rtol=1e-12, atol=0)
    assert np.allclose(dn[:, 0], g["dn_plane0"], rtol=1e-11, atol=1e-15)
    if "c2_band_sq" in g:  # every band: sums of squares and of the coefficients
        c2 = packed(inp, st.c2, inp.nbands)
        assert np.abs((c2 * c2).sum(axis=(1, 2)) - g["c2_band_sq"]).max() < 1e-10
        assert np.abs(c2.sum(axis=(1, 2)) - g["c2_band_sum"]).max() < 1e-9


@pytest.mark.parametrize("name", list(CASES))
def test_resident_cell_matches_reference(golden, name):
    """Persistent context (orbitals stay in HBM between calls) == reference build."""
    mk, ncalls, inner = CASES[name]
    inp = inputs.build_inputs(mk())
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    rows = []
    for _ in range(ncalls):
        cell.run(inner)
        rows.append((cell.E.copy(), cell.deltae, cell.deltac))
    st = api.State(inp)
    cell.get_state(st)
    cell.close()
    check_against_golden(inp, golden(name), rows, st)


@pytest.mark.parametrize("name", ["small_h2_16", "small_diamond_24", "diamond8_64", "spin_diamond_24"])
def test_dropin_cpsd_matches_reference(golden, name):
    """The reference-facing cpsd() with host buffers, called like main.c does."""
    mk, ncalls, inner = CASES[name]
    inp = inputs.build_inputs(mk())
    st = api.State(inp)
    rows = []
    for _ in range(ncalls):
        api.cpsd(inp, st, inner)
        rows.append((st.E.copy(), st.deltae, st.deltac))
    check_against_golden(inp, golden(name), rows, st)
    # cpsi leaves as c2 - c1, full box (cpsd.c:650-651)
    assert np.array_equal(st.cpsi, st.c2 - st.c1) or np.abs(st.cpsi - (st.c2 - st.c1)).max() < 1e-15


def _outside_sphere(inp, x):
    return x.reshape(-1, inp.nfft3d, 2)[:, inp.masker1 == 0, :]


def _resident_call(inp, c2, r2, inner):
    """One call of `inner` steps on a fresh resident context."""
    cell = api.GpuCell(inp)
    cell.set_state(c2, r2)
    cell.run(inner)
    st = api.State(inp)
    cell.get_state(st)
    E = cell.E.copy()
    cell.close()
    return E, st


def test_dropin_notices_changed_tables_and_mask():
    """The drop-in reuses its context and runs on the tables and mask it
    holds while host threads compare them with the caller's: tables changed
    in place between calls, and a cell of the same shape with another mask,
    give what a fresh context gives for the new inputs."""
    inp = inputs.build_inputs(configs.small_diamond(24, 4, ecut=20.0))
    st = api.State(inp)
    api.cpsd(inp, st, 2)
    inp.vg *= 1.0 + 1e-3  # the Hartree kernel, in place: same array, new values
    c2, r2 = st.c2.copy(), st.r2.copy()
    api.cpsd(inp, st, 2)
    E_ref, s_ref = _resident_call(inp, c2, r2, 2)
    assert np.array_equal(st.E, E_ref)
    assert np.array_equal(st.c2, s_ref.c2)
    # same nfft, bands, ions and kinds, another cutoff: another mask
    other = inputs.build_inputs(configs.small_diamond(24, 4, ecut=16.0))
    assert not np.array_equal(other.masker1, inp.masker1)
    so = api.State(other)
    api.cpsd(other, so, 2)
    E_ref, s_ref = _resident_call(other, other.c2, other.r2, 2)
    assert np.array_equal(so.E, E_ref)
    assert np.array_equal(so.c2, s_ref.c2)
    assert np.array_equal(so.dn, s_ref.dn)


def test_host_layout_outputs_overwrite_every_grid_point():
    """c1 and cpsi are outputs only: NaN or other values in those buffers
    before a call leave no trace (only the sphere crosses PCIe; host threads
    write the zeros), and the results are bit-identical to calls whose
    buffers started clean.  The resident get_state writes whole grids too."""
    inp = inputs.build_inputs(configs.small_diamond(24, 4, ecut=16.0))
    clean, dirty = api.State(inp), api.State(inp)
    for fill in (np.nan, -3.0):
        dirty.c1[:] = fill
        dirty.cpsi[:] = 7.0
        api.cpsd(inp, clean, 2)
        api.cpsd(inp, dirty, 2)
        for a, b in ((clean.c1, dirty.c1), (clean.c2, dirty.c2), (clean.cpsi, dirty.cpsi), (clean.dn, dirty.dn)):
            assert np.array_equal(a, b)
    for x in (clean.c1, clean.c2, clean.cpsi):
        assert not _outside_sphere(inp, x).any()
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    cell.run(2)
    ref, got = api.State(inp), api.State(inp)
    for x in (got.c1, got.c2, got.cpsi):
        x[:] = np.nan
    cell.get_state(ref)
    cell.get_state(got)
    cell.close()
    for a, b in ((ref.c1, got.c1), (ref.c2, got.c2), (ref.cpsi, got.cpsi)):
        assert np.array_equal(a, b)
        assert not _outside_sphere(inp, b).any()


def _moving(spec):
    spec.move = 1
    return spec


# move = 1: ion forces and the ion SD step (tests/golden/make_golden.py MOVE_CASES)
MOVE_CASES = {
    "move_small_h2_16": (lambda: _moving(configs.small_h2(16)), 3, 2),
    "move_small_diamond_24": (lambda: _moving(configs.small_diamond(24, 4)), 3, 2),
    "move_small_diamond_32": (lambda: _moving(configs.small_diamond(32, 40, ecut=25.0, seed=12)), 2, 2),
    # spin-polarised: the nonlocal force factor is 1 instead of 2 (cpsd.c:287-304)
    "move_spin_diamond_24": (lambda: _moving(configs.spin_diamond(24, ne=(4, 3))), 3, 2),
}
F_TOL = 1e-9  # Ha/bohr


@pytest.mark.parametrize("name", list(MOVE_CASES))
def test_ion_motion_matches_reference(golden, name):
    """move = 1 on the resident cell: energies, forces (local, nonlocal,
    k-space and real-space Ewald), positions and deltar of every call against
    the reference build."""
    mk, ncalls, inner = MOVE_CASES[name]
    g = golden(name)
    inp = inputs.build_inputs(mk())
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    st = api.State(inp)
    for k in range(ncalls):
        cell.run(inner, move=1)
        cell.get_state(st)
        assert abs(cell.E[0] - g["E"][k, 0]) < E_TOL
        assert np.abs(st.fion - g["fion"][k]).max() < F_TOL
        assert np.abs(st.r2 - g["r2"][k]).max() < 1e-12
        assert abs(cell.deltar - g["deltar"][k]) < F_TOL
    assert np.abs(st.lmd - g["lmd"]).max() < 1e-9
    cell.close()


def test_dropin_cpsd_with_ion_motion_matches_reference(golden):
    """The reference-facing cpsd() with move = 1, called like main.c does."""
    mk, ncalls, inner = MOVE_CASES["move_small_diamond_24"]
    g = golden("move_small_diamond_24")
    inp = inputs.build_inputs(mk())
    st = api.State(inp)
    for k in range(ncalls):
        api.cpsd(inp, st, inner, move=1)
        assert abs(st.E[0] - g["E"][k, 0]) < E_TOL
        assert np.abs(st.fion - g["fion"][k]).max() < F_TOL
        assert np.abs(st.r2 - g["r2"][k]).max() < 1e-12
        assert abs(st.deltar - g["deltar"][k]) < F_TOL


def test_lagrange_warning_matches_reference_quirk():
    """One band: the reference never meets its convergence test (cpsd.c:471),
    every call ends with the ierr=10 warning; so does the drop-in."""
    inp = inputs.build_inputs(configs.small_h2(16))
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    for _ in range(3):
        cell.run(2)
    assert cell.lagrange_warnings == 3
    assert lib.load().cpsd_gpu_lagrange_failures(cell.h) == 6
    cell.close()


def test_intermediates_match_restatement(restatement):
    """Density, Hamiltonian and Lagrange matrices after one step, and the
    orthonormality the constraint restores (<c2|c2> = 1 + O(dte^2))."""
    inp = inputs.build_inputs(configs.small_diamond(24, 6, ecut=22.0, seed=11))
    so = oracle.State(inp)
    restatement.run(inp, 1, so)
    sg = api.State(inp)
    api.cpsd(inp, sg, 1)
    assert np.abs(so.dn - sg.dn).max() < 1e-13
    assert np.abs(so.hml - sg.hml).max() < 1e-10
    assert np.abs(so.lmd - sg.lmd).max() < 1e-10
    assert abs(so.E[0] - sg.E[0]) < E_TOL
    w = inputs.gamma_weights(inp.nfft)
    C = sg.c2.reshape(inp.nbands, -1).view(np.complex128)
    S = np.einsum("p,ap,bp->ab", w, C.conj(), C).real
    assert np.abs(S - np.eye(inp.nbands)).max() < 1e-4


@pytest.mark.parametrize("solver", ["tile", "cluster"])
@pytest.mark.parametrize("nb", [40, 128])
def test_many_band_lagrange_solvers_match_restatement(restatement, monkeypatch, solver, nb):
    """More than 32 bands run the cluster Lagrange solvers (the 4 x 4 tiled
    one by default, the column one with CPSD_B200_LAGRANGE=cluster): lmd, hml
    and the energies of three SD steps against the restatement (40 bands:
    ragged 10 x 10 tiles; 128: full 32 x 32 tiles)."""
    if solver == "cluster":
        monkeypatch.setenv("CPSD_B200_LAGRANGE", "cluster")
    else:
        monkeypatch.delenv("CPSD_B200_LAGRANGE", raising=False)
    inp = inputs.build_inputs(configs.small_diamond(32, nb, ecut=25.0, seed=12))
    so = oracle.State(inp)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    for _ in range(3):
        restatement.run(inp, 1, so)
        cell.run(1)
        assert abs(cell.E[0] - so.E[0]) < E_TOL
    sg = api.State(inp)
    cell.get_state(sg)
    assert np.abs(so.lmd - sg.lmd).max() < 1e-10
    assert np.abs(so.hml - sg.hml).max() < 1e-10
    assert cell.lagrange_warnings == so.lagrange_fail  # same converged / not-converged steps
    cell.close()


@pytest.mark.parametrize("n", [16, 24, 32, 48, 64, 128])
def test_fft_dropins_match_oracle(restatement, n):
    """cr_fft3b_/rc_fft3f_ drop-ins (whole box) == the fftpack3d restatement."""
    rng = np.random.default_rng(100 + n)
    nh = n // 2 + 1
    C = rng.standard_normal((n, n, nh)) + 1j * rng.standard_normal((n, n, nh))
    A = np.ascontiguousarray(C).view(np.float64).reshape(-1).copy()
    B = A.copy()
    api.cr_fft3b(A, n)
    restatement.cr_fft3b(B, n)
    assert np.abs(A - B).max() <= 2e-14 * np.abs(B).max()
    x = rng.standard_normal((n, n, n + 2)).reshape(-1)
    A, B = x.copy(), x.copy()
    api.rc_fft3f(A, n)
    restatement.rc_fft3f(B, n)
    assert np.abs(A - B).max() <= 2e-14 * np.abs(B).max()


def test_fft_roundtrip_full_size():
    """rc then cr returns n^3 x at the largest supported grid."""
    n = 128
    rng = np.random.default_rng(7)
    A = np.zeros((n, n, n + 2))
    A[:, :, :n] = rng.standard_normal((n, n, n))
    x0 = A[:, :, :n].copy()
    A = A.reshape(-1)
    api.rc_fft3f(A, n)
    api.cr_fft3b(A, n)
    assert np.abs(A.reshape(n, n, n + 2)[:, :, :n] / n ** 3 - x0).max() < 1e-13


def test_full_size_cell_properties():
    """The 128^3 / 64-atom / 128-band cell (too large for the CPU oracle per
    step): energy decreases, orthonormality holds, hml and lmd symmetric,
    the density integrates to the electron count, reruns are bitwise equal."""
    inp = inputs.build_inputs(configs.diamond64_128())
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    Es = []
    for _ in range(3):
        cell.run(2)
        Es.append(cell.E[0])
    st = api.State(inp)
    cell.get_state(st)
    assert Es[0] > Es[1] > Es[2]
    m = inp.nbands
    H = st.hml[:m * m].reshape(m, m)
    assert np.abs(H - H.T).max() < 1e-12 * np.abs(H).max()
    dv = inp.omega / inp.nfft ** 3
    dn = st.dn.reshape(inp.nfft, inp.nfft, inp.nfft + 2)[..., :inp.nfft]
    assert abs(dn.sum() * dv - m) < 1e-8 * m  # ispin=1: dn holds one spin, nb electrons
    w = inputs.gamma_weights(inp.nfft)
    pts = np.flatnonzero(inp.masker1)
    C = st.c1.reshape(m, -1).view(np.complex128)[:, pts]
    S = (C.conj() * w[pts]) @ C.T
    assert np.abs(S.real - np.eye(m)).max() < 1e-6
    # determinism: same inputs, same bits
    cell.set_state(inp.c2, inp.r2)
    cell.E[:] = 0
    cell.run(2)
    e_again = cell.E[0]
    cell.close()
    cell2 = api.GpuCell(inp)
    cell2.set_state(inp.c2, inp.r2)
    cell2.run(2)
    assert cell2.E[0] == e_again
    cell2.close()


def test_error_paths(golden):
    """Bad inputs come back as status codes, never as a device fault."""
    inp = inputs.build_inputs(configs.small_h2(16))
    # move = 1 without the G vectors and masses it needs
    L = lib.load()
    cell = api.GpuCell(inp)
    nul = ctypes.c_void_p()
    assert L.cpsd_gpu_set_tables(cell.h, api._ptr(inp.katm), nul, api._ptr(inp.zv), api._ptr(inp.rcell), nul,
                                 api._ptr(inp.tg), api._ptr(inp.vc), api._ptr(inp.vg), api._ptr(inp.lmmax),
                                 api._ptr(inp.vnlnrm), api._ptr(inp.vl), api._ptr(inp.vnl)) == 0
    cell.set_state(inp.c2, inp.r2)
    with pytest.raises(lib.CpsdError) as e:
        cell.run(1, move=1)
    assert e.value.status == lib.CPSD_ERR_MOVE
    cell.close()
    bad = inputs.build_inputs(configs.small_h2(16))
    bad.c2 = bad.c2.copy()
    out_of_mask = np.flatnonzero(bad.masker1 == 0)[5]
    bad.c2[2 * out_of_mask] = 1.0
    st = api.State(bad)
    st.c1[:] = -2.0
    st.cpsi[:] = 5.0
    before = {n: getattr(st, n).copy() for n in ("c1", "c2", "cpsi", "dn", "hml", "lmd", "E", "r1", "r2")}
    with pytest.raises(lib.CpsdError) as e:
        api.cpsd(bad, st, 1)
    assert e.value.status == lib.CPSD_ERR_UNMASKED_PSI
    # the check runs beside the steps, but no output is written on a refusal
    for n, v in before.items():
        assert np.array_equal(getattr(st, n), v), n
    # and the next call with masked orbitals is the reference's
    mk, ncalls, inner = CASES["small_h2_16"]
    good = inputs.build_inputs(mk())
    sg = api.State(good)
    rows = []
    for _ in range(ncalls):
        api.cpsd(good, sg, inner)
        rows.append((sg.E.copy(), sg.deltae, sg.deltac))
    check_against_golden(good, golden("small_h2_16"), rows, sg)
    cell = api.GpuCell(inp)
    with pytest.raises(lib.CpsdError) as e:
        cell.run(0)
    assert e.value.status == lib.CPSD_ERR_ARG
    cell.close()
    spec = configs.small_h2(16)
    spec.nfft = 20  # not a supported grid
    with pytest.raises(lib.CpsdError) as e:
        api.GpuCell(inputs.build_inputs(spec))
    assert e.value.status == lib.CPSD_ERR_GRID
    A = np.zeros((20 + 2) * 20 * 20)
    with pytest.raises(lib.CpsdError):
        api.rc_fft3f(A, 20)


@pytest.mark.parametrize("nb", [4, 40])
def test_non_finite_orbitals_warn_without_fault(nb):
    """NaN orbitals (a diverged step) reach the Lagrange solver's convergence
    test, whose idamax must still return an index inside st1: the call warns
    (no convergence) and the context stays usable.  nb = 4 runs the
    single-CTA solver, nb = 40 the cluster solver."""
    inp = inputs.build_inputs(configs.small_diamond(32, nb, ecut=25.0))
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    _, c2, _ = cell.get_packed()
    c2[:] = np.nan
    cell.set_packed(c2)
    cell.run(1)
    assert cell.lagrange_warnings == 1
    assert not np.isfinite(cell.E[0])
    cell.set_state(inp.c2, inp.r2)
    cell.run(1)
    assert np.isfinite(cell.E[0])
    cell.close()


def test_graphs_and_direct_launches_agree():
    inp = inputs.build_inputs(configs.small_diamond(32, 5, ecut=25.0))
    out = []
    for graphs in (True, False):
        cell = api.GpuCell(inp)
        cell.use_graphs(graphs)
        cell.set_state(inp.c2, inp.r2)
        cell.run(3)
        out.append(cell.E.copy())
        cell.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("move", [0, 1])
def test_two_stream_step_equals_serial_step(move):
    """The production step runs the projector / kinetic / nonlocal branch on
    a second stream beside the density chain; with phase timing on, the same
    kernels run on one stream.  Both orders give the same bits."""
    inp = inputs.build_inputs(configs.small_diamond(24, 6, ecut=20.0, seed=13))
    out = []
    for serial in (False, True):
        cell = api.GpuCell(inp)
        cell.phase_timing(serial)
        cell.set_state(inp.c2, inp.r2)
        E = [cell.run(2, move=move).copy() for _ in range(3)]
        st = api.State(inp)
        cell.get_state(st)
        out.append((np.array(E), st.c2.copy(), st.r2.copy()))
        cell.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(oracle.REFERENCE_SO), "dcpsdv3_b200.x")),
                    reason="drop-in build of the reference main() absent")
def test_reference_main_linked_against_library(tmp_path):
    """The reference's unmodified main.c linked with this library's cpsd()
    (oracle/_ref/dcpsdv3_b200.x) reproduces the reference main()'s run."""
    import subprocess
    from cpsd_b200 import refio
    g = np.load(os.path.join(GOLDEN, "ref_main_small_diamond_24.npz"))
    spec = configs.small_diamond(24, 4)
    spec.ecut_ry = float(g["ecut"])
    inp = inputs.build_inputs(spec)
    refio.write_reference_inputs(str(tmp_path), inp, inner=int(g["inner"]), outer=int(g["outer"]))
    exe = os.path.join(os.path.dirname(oracle.REFERENCE_SO), "dcpsdv3_b200.x")
    out = subprocess.run([exe], cwd=str(tmp_path), capture_output=True, check=True).stdout.decode("utf-8", "replace")
    rows, final = refio.parse_reference_stdout(out)
    assert len(rows) == len(g["rows"])
    for r, w in zip(rows, g["rows"]):
        assert abs(r[1] - w[1]) <= 1e-9 * max(1.0, abs(w[1]))
    assert np.allclose([final[i] for i in range(10)], g["final"], rtol=1e-9, atol=1e-9)


def test_batched_cells_equal_individual_runs():
    """Config 4 style: uneven cells stepped in one graph per SD step give the
    same bits as each cell run on its own."""
    specs = [configs.small_diamond(24, 4, seed=21), configs.small_h2(16, seed=5),
             configs.small_diamond(32, 5, ecut=25.0, seed=8), configs.small_diamond(48, 6, ecut=30.0, seed=9)]
    inps = [inputs.build_inputs(s) for s in specs]
    solo = []
    for inp in inps:
        cell = api.GpuCell(inp)
        cell.set_state(inp.c2, inp.r2)
        cell.run(3)
        cell.run(2)
        solo.append(cell.E.copy())
        cell.close()
    cells = []
    for inp in inps:
        cell = api.GpuCell(inp)
        cell.set_state(inp.c2, inp.r2)
        cells.append(cell)
    batch = api.GpuBatch(cells)
    batch.run(3)
    E = batch.run(2)
    for i in range(len(inps)):
        assert np.array_equal(E[i], solo[i]), i
    batch.close()
    for c in cells:
        c.close()


def test_batched_draw_matches_reference(golden):
    """The 48-cell batched workload (grids 32/48/64, 4-25 bands, H and C
    kinds), all cells in one graph per SD step: the cells with fixtures from
    the reference build match them call by call (energies, deltae, deltac)
    and after the last call (hml, lmd, orbitals, density)."""
    specs = configs.batched_cells(0)
    inps = [inputs.build_inputs(s) for s in specs]
    cells = []
    for inp in inps:
        cell = api.GpuCell(inp)
        cell.set_state(inp.c2, inp.r2)
        cells.append(cell)
    batch = api.GpuBatch(cells)
    rows = {i: [] for i in BATCH_DRAW}
    for _ in range(2):
        E = batch.run(2)
        for i in BATCH_DRAW:
            rows[i].append((E[i].copy(), batch.deltae[i], batch.deltac[i]))
    for i, name in BATCH_DRAW.items():
        st = api.State(inps[i])
        cells[i].get_state(st)
        check_against_golden(inps[i], golden(name), rows[i], st)
    assert np.all(np.isfinite(batch.E))
    batch.close()
    for c in cells:
        c.close()


def test_mixed_precision_tracks_fp64(restatement):
    """FP32 transforms (orbitals, potentials and reductions FP64): the energy
    follows the FP64 oracle to ~1e-7 relative; an FP64 refinement call on
    the same state restores the parity bar on its energies' consistency."""
    inp = inputs.build_inputs(configs.small_diamond(32, 5, ecut=25.0))
    so = oracle.State(inp)
    cell = api.GpuCell(inp, precision=lib.CPSD_PREC_MIXED)
    cell.set_state(inp.c2, inp.r2)
    for _ in range(3):
        restatement.run(inp, 2, so)
        cell.run(2)
        assert abs(cell.E[0] - so.E[0]) < 1e-6 * abs(so.E[0]) + 1e-6
    # switch to FP64 for a refinement call from the mixed state: its energy is
    # that of an FP64 evaluation of the same state (checked against the oracle)
    st = api.State(inp)
    cell.get_state(st)
    cell.set_precision(lib.CPSD_PREC_FP64)
    cell.E[0] = 0.0
    cell.run(1)
    probe = oracle.State(inp)
    probe.c2[:] = st.c2
    restatement.run(inp, 1, probe)
    assert abs(cell.E[0] - probe.E[0]) < E_TOL
    cell.close()


# epilogue of main.c:452-487 (tests/golden/make_golden.py EPILOGUE_CASES)
from test_oracle import EPI_CASES, align_bands, check_vectors, eig_blocks, vector_tolerances  # noqa: E402


def _packed_bands(inp, c, nb):
    pts = np.flatnonzero(inp.masker1)
    return c.reshape(inp.nbands, inp.nfft3d, 2)[:nb, pts, :]


@pytest.mark.parametrize("name", list(EPI_CASES))
def test_epilogue_matches_reference(golden, name):
    """On the device: the orthonormality table, the eigenpairs of hml
    (descending, the reference's eigsrt order; Jacobi vectors compared up to
    each column's sign) and c1 <- c2 V, against the reference's own gcdotc,
    eigsrt and LAPACK after the same cpsd() calls."""
    g = golden("epi_" + name)
    inp = inputs.build_inputs(EPI_CASES[name]())
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    for _ in range(int(g["ncalls"])):
        cell.run(int(g["inner"]))
    before = api.State(inp)
    cell.get_state(before)
    assert np.abs(before.hml - g["hml"]).max() < 1e-9
    ep = cell.epilogue()
    after = api.State(inp)
    cell.get_state(after)
    cell.close()
    vec_tol, c1_tol = vector_tolerances(inp, g)
    assert np.abs(ep["ortho"] - g["ortho"]).max() < 1e-12
    assert np.abs(ep["eig"] - g["eig"]).max() < 1e-9
    for _, m, e0 in eig_blocks(inp, g):
        assert np.all(np.diff(ep["eig"][e0:e0 + m]) <= 0)
    check_vectors(inp, g, ep["vec"], vec_tol)
    got = _packed_bands(inp, after.c1, g["c1"].shape[0])
    assert np.abs(align_bands(g["c1"], got) - g["c1"]).max() < c1_tol
    assert np.array_equal(after.c2, before.c2)  # the epilogue leaves c2 alone


def test_epilogue_files_reproduce_reference_main(tmp_path):
    """The reference main()'s run (ELCIN/CONTROL/IONIN from the same inputs)
    finished on the device: printed orbital energies, the ELCOUT the library
    writes (header bytes, c1 up to each band's sign) and IONOUT's text."""
    from cpsd_b200 import refio
    g = np.load(os.path.join(GOLDEN, "ref_main_small_diamond_24.npz"))
    spec = configs.small_diamond(24, 4)
    spec.ecut_ry = float(g["ecut"])
    inp = inputs.build_inputs(spec)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    for _ in g["rows"]:
        cell.run(int(g["inner"]))
    ep = cell.epilogue()
    st = api.State(inp)
    cell.get_state(st)
    cell.close()
    m = int(inp.ne[0])
    for ms, i, j, w in g["ortho_printed"]:
        assert abs(ep["ortho"][int(i) - 1 + (int(j) - 1) * m] - w) <= 5e-8 * abs(w) + 1e-15
    assert np.allclose(ep["eig"], g["eig_printed"], rtol=1e-7, atol=0)
    path = str(tmp_path / "ELCOUT")
    api.write_elcout(path, inp, st.c1)
    back = refio.read_elcin(path)
    icube, nfft, ispin, ne0, ne1 = (int(x) for x in g["elcout_header"])
    assert (back["icube"], back["nfft"], back["ispin"], back["ne"]) == (icube, nfft, ispin, (ne0, ne1))
    assert back["unit"] == float(g["elcout_unit"])
    got = _packed_bands(inp, back["c"], inp.nbands)
    assert np.abs(align_bands(g["elcout_c1"], got) - g["elcout_c1"]).max() < 1e-9
    assert not np.delete(back["c"].reshape(inp.nbands, inp.nfft3d, 2), np.flatnonzero(inp.masker1), axis=1).any()
    path = str(tmp_path / "IONOUT")
    api.write_ionout(path, inp, ["C0.vpp"], st.r2)
    with open(path) as f:
        assert f.read() == str(g["ionout"])


def test_epilogue_needs_a_run():
    inp = inputs.build_inputs(configs.small_diamond(24, 4))
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    with pytest.raises(lib.CpsdError) as e:
        cell.epilogue()
    assert e.value.status == lib.CPSD_ERR_ARG
    cell.close()


# input pipeline (tests/golden/make_golden.py KBPP_CASES, run_kbpp_main)
from test_oracle import KBPP_CASES, assert_kbpp_close, kbpp_case  # noqa: E402


@pytest.mark.parametrize("name", list(KBPP_CASES))
def test_kbpp_matches_reference(golden, name):
    """cpsd_gpu_kbpp (one thread per G, the radial tables in shared memory)
    against the reference's own compiled kbpp() on the same table and grid:
    s, p and d channels, the local part with its long-range term, G = 0."""
    g, t, G, nfft3d = kbpp_case(golden, name)
    got = api.kbpp(t, G, nfft3d)
    assert_kbpp_close(got, g, 1e-13)


def test_psp_formatter_reproduces_reference_dataout(tmp_path):
    """psp.format_vpp (kbpp on the GPU) writes the .vpp file the reference's
    formatter program wrote for the same table, grid and "highest L" answer
    (a lower answer than the table's lmax makes that channel the local one)."""
    from cpsd_b200 import psp, refio
    g = np.load(os.path.join(GOLDEN, "ref_kbpp_main.npz"))
    ref_path = str(tmp_path / "DATAOUT.ref")
    with open(ref_path, "wb") as f:
        f.write(g["dataout"].tobytes())
    t = psp.radial_table(int(g["lmax"]), seed=int(g["seed"]))
    path = str(tmp_path / "DATAOUT")
    psp.format_vpp(path, t, 1, 10.26, int(g["nfft"]), int(g["highest_l"]))
    a, b = refio.read_vpp(path), refio.read_vpp(ref_path)
    assert os.path.getsize(path) == os.path.getsize(ref_path)
    with open(path, "rb") as f:
        assert f.read(38) == g["dataout"].tobytes()[:38]  # icube, nfft, unit, atom, amass, zv, lmax
    for k in ("icube", "nfft", "unit", "atom", "amass", "zv", "lmax"):
        assert a[k] == b[k], k
    assert np.array_equal(a["rc"], b["rc"])
    assert np.abs(a["vnlnrm"] - b["vnlnrm"]).max() <= 1e-15 * np.abs(b["vnlnrm"]).max()
    assert np.abs(a["vl"] - b["vl"]).max() <= 1e-13 * np.abs(b["vl"]).max()
    assert np.abs(a["vnl"] - b["vnl"]).max() <= 1e-13 * np.abs(b["vnl"]).max()


def test_pipeline_inputs_drive_the_sd_path(restatement):
    """Radial table -> kbpp on the GPU -> vl, vnl, vnlnrm; plane-wave start
    orbitals from makepsi; SD steps on those inputs on the GPU equal the
    restatement's on the same arrays."""
    from cpsd_b200 import psp
    inp = inputs.build_inputs(configs.small_diamond(24, 4, ecut=20.0))
    t = psp.radial_table(2, seed=2)
    vl, vnl, vnlnrm, _ = api.kbpp(t, inp.G, inp.nfft3d)
    inp.vl[:] = vl
    inp.vnl[:] = 0.0
    inp.vnl[:4 * inp.nfft3d] = vnl
    inp.vnlnrm[:] = 0.0
    inp.vnlnrm[:4] = vnlnrm
    inp.c2 = api.makepsi(inp.nfft, 1, (4, 0), [(0, 0, 0, 0), (1, 0, 0, -1), (1, 0, 0, 1), (0, 1, 0, -1)])
    so = oracle.State(inp)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    for _ in range(2):
        restatement.run(inp, 2, so)
        cell.run(2)
        assert abs(cell.E[0] - so.E[0]) < E_TOL
    st = api.State(inp)
    cell.get_state(st)
    cell.close()
    assert np.abs(st.c2 - so.c2).max() < 1e-10


def test_max_bands_per_spin_matches_restatement(restatement):
    """256 bands, the engine's limit per spin: the 16-CTA column-cluster
    Lagrange solver chosen on its own (no override), 4 x 4 tiles of the FP64
    tensor-core products, 256-band plane passes; one SD step against the
    restatement on the same inputs."""
    inp = inputs.build_inputs(configs.small_diamond(32, 256, ecut=40.0, seed=13))
    so = oracle.State(inp)
    restatement.run(inp, 1, so)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    cell.run(1)
    st = api.State(inp)
    cell.get_state(st)
    cell.close()
    assert abs(cell.E[0] - so.E[0]) < 1e-12 * abs(so.E[0]) + 1e-9
    assert np.abs(st.lmd - so.lmd).max() < 1e-10 * np.abs(so.lmd).max()
    assert np.abs(st.hml - so.hml).max() < 1e-10 * np.abs(so.hml).max()
    assert np.abs(st.c2 - so.c2).max() < 1e-10


def test_cell_shards_gpu_runner_equals_individual_cells():
    """shards.run_cells with the GPU runner (one batched graph per SD step
    for the rank's cells) gives each cell the energies of its own
    resident run, bit for bit."""
    from cpsd_b200 import shards
    specs = [configs.small_h2(16, seed=3), configs.small_diamond(24, 4, seed=5), configs.small_h2(16, seed=4)]
    E = shards.run_cells(specs, 2, 1)
    for spec, e in zip(specs, E):
        inp = inputs.build_inputs(spec)
        cell = api.GpuCell(inp)
        cell.set_state(inp.c2, inp.r2)
        for _ in range(2):
            cell.run(1)
        assert np.array_equal(cell.E, e)
        cell.close()
