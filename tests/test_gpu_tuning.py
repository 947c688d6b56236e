"""GPU tests of the kernel choices and the project's autotuner.

Every choice (both occupancy builds of every plane pass, density chunk
counts, split-K targets, the two cluster Lagrange solvers) keeps the FP64
parity bar against the reference build's fixtures: the choices change speed
and rounding, not the algorithm (ccpsdv3/cpsd.c:168-491).
"""
import numpy as np
import pytest

from cpsd_b200 import api, configs, inputs, lib

from test_gpu_parity import E_TOL, check_against_golden

pytestmark = pytest.mark.gpu


def _run(inp, ncalls, inner, **tuning):
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    if tuning:
        cell.set_tuning(**tuning)
    rows = []
    for _ in range(ncalls):
        cell.run(inner)
        rows.append((cell.E.copy(), cell.deltae, cell.deltac))
    st = api.State(inp)
    cell.get_state(st)
    t = cell.tuning()
    cell.close()
    return rows, st, t


def test_tuning_round_trip_and_limits():
    inp = inputs.build_inputs(configs.small_diamond(32, 40, ecut=25.0, seed=12))
    cell = api.GpuCell(inp)
    t0 = cell.tuning()
    lim = cell.tuning_limits()
    assert t0["lagrange_solver"] in (1, 2) and lim["lagrange_solver"] == 2
    assert 1 <= t0["density_chunks"] <= lim["density_chunks"]
    cell.set_tuning(tn_ctas_per_sm=4, density_chunks=lim["density_chunks"])
    t1 = cell.tuning()
    assert t1["tn_ctas_per_sm"] == 4 and t1["density_chunks"] == lim["density_chunks"]
    for bad in ({"tn_ctas_per_sm": 0}, {"tn_ctas_per_sm": 9}, {"density_chunks": lim["density_chunks"] + 1},
                {"lagrange_solver": 3}, {"plane_occupancy": [2, 0, 0, 0]}):
        with pytest.raises(lib.CpsdError) as e:
            cell.set_tuning(**bad)
        assert e.value.status == lib.CPSD_ERR_ARG
    assert cell.tuning() == t1  # a refused call changes nothing
    cell.close()


@pytest.mark.parametrize("mode", range(4))
def test_every_plane_build_keeps_parity(golden, mode):
    """Both occupancy builds of each plane pass (density, V psi, potential to
    r, density to G) on the 64^3 cell against the reference build."""
    inp = inputs.build_inputs(configs.diamond8_64())
    cell = api.GpuCell(inp)
    lim = cell.tuning_limits()["plane_occupancy"][mode]
    cell.close()
    g = golden("diamond8_64")
    for v in range(lim + 1):
        occ = [0, 0, 0, 0]
        occ[mode] = v
        rows, st, t = _run(inp, 4, 2, plane_occupancy=occ)
        assert t["plane_occupancy"] == occ
        check_against_golden(inp, g, rows, st)


@pytest.mark.parametrize("occ", [0, 1])
def test_density_row_split_keeps_parity_at_128(golden, occ):
    """The 128^3 density pass whole (one CTA per plane) and with its x rows
    split between two CTAs per plane, against the reference build."""
    inp = inputs.build_inputs(configs.diamond64_128())
    cell = api.GpuCell(inp)
    lim = cell.tuning_limits()["plane_occupancy"][0]
    planes = cell.tuning()["plane_occupancy"]
    cell.close()
    if occ > lim:
        pytest.skip("the row-split build does not fit this device")
    planes[0] = occ
    rows, st, t = _run(inp, 1, 2, plane_occupancy=planes)
    assert t["plane_occupancy"][0] == occ
    check_against_golden(inp, golden("diamond64_128"), rows, st)


def test_density_chunks_split_k_and_solvers_keep_parity(restatement):
    """Other choices on a 40-band cell against the restatement: density chunk
    counts 1 and the largest, split-K targets 1 and 4, both cluster solvers."""
    import oracle
    inp = inputs.build_inputs(configs.small_diamond(32, 40, ecut=25.0, seed=12))
    so = oracle.State(inp)
    restatement.run(inp, 2, so)
    cell = api.GpuCell(inp)
    lim = cell.tuning_limits()
    cell.close()
    for kw in ({"density_chunks": 1}, {"density_chunks": lim["density_chunks"]}, {"tn_ctas_per_sm": 1},
               {"tn_ctas_per_sm": 4}, {"lagrange_solver": 2}, {"lagrange_solver": 1}):
        rows, st, _ = _run(inp, 1, 2, **kw)
        assert abs(rows[0][0][0] - so.E[0]) < E_TOL, kw
        assert np.abs(st.lmd - so.lmd).max() < 1e-10, kw


@pytest.mark.parametrize("name", ["diamond8_64", "diamond64_128"])
def test_autotuned_cell_keeps_parity(golden, name):
    """The autotuner times its candidates on the cell, restores the orbitals,
    and the tuned run still matches the reference build; a second context of
    the same shape takes the cached choice without timing."""
    mk = {"diamond8_64": (configs.diamond8_64, 4, 2), "diamond64_128": (configs.diamond64_128, 1, 2)}
    spec, ncalls, inner = mk[name]
    inp = inputs.build_inputs(spec())
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    res = cell.autotune(steps=4 if name == "diamond64_128" else 10, force=True)
    assert res["ms_per_step_before"] > 0 and res["ms_per_step_after"] > 0
    assert res["ms_per_step_after"] <= res["ms_per_step_before"] * 1.1
    rows = []
    for _ in range(ncalls):
        cell.run(inner)
        rows.append((cell.E.copy(), cell.deltae, cell.deltac))
    st = api.State(inp)
    cell.get_state(st)
    cell.close()
    check_against_golden(inp, golden(name), rows, st)
    cell2 = api.GpuCell(inp)
    cell2.set_state(inp.c2, inp.r2)
    res2 = cell2.autotune()
    assert res2["ms_per_step_before"] == -1.0 and res2["tuning"] == res["tuning"]
    cell2.close()
