"""GPU tests of band-parallel SD of one cell (cpsd_b200.bands).

One GPU per test run here, so several ranks are emulated by contexts of one
process stepped phase by phase (LocalGroup: no kernel waits on another);
the NCCL path runs with one rank.  The decomposition over several processes
is tested on CPU with gloo ranks and the restatement (tests/test_host.py).
"""
import os
import socket

import numpy as np
import pytest

from cpsd_b200 import api, bands, configs, inputs

from test_gpu_parity import check_against_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ordinary(inp, ncalls, inner):
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    Es = []
    for _ in range(ncalls):
        Es.append(cell.run(inner).copy())
    st = api.State(inp)
    cell.get_state(st)
    cell.close()
    return np.array(Es), st


def _group(inp, ncalls, inner, world):
    ranges = bands.band_ranges(inp.nbands, world)
    cells = []
    for lo, hi in ranges:
        c = api.GpuCell(inp)
        c.set_state(inp.c2, inp.r2)
        c.set_band_range(lo, hi)
        cells.append(c)
    ex = bands.LocalGroup(torch, cells, ranges)
    Es = []
    for _ in range(ncalls):
        Es.append(bands.run(cells, ex, inner))
    states = []
    for c in cells:
        st = api.State(inp)
        c.get_state(st)
        states.append(st)
        c.close()
    return np.array(Es), states


def test_one_rank_by_phases_is_the_ordinary_step():
    """A context owning every band, stepped phase by phase with the
    exchanges in between, gives the bits of the ordinary step."""
    inp = inputs.build_inputs(configs.small_diamond(24, 6, ecut=20.0, seed=13))
    E0, s0 = _ordinary(inp, 2, 2)
    E1, s1 = _group(inp, 2, 2, 1)
    assert np.array_equal(E0, E1[:, 0])
    for a in ("c1", "c2", "cpsi", "dn", "hml", "lmd"):
        assert np.array_equal(getattr(s0, a), getattr(s1[0], a)), a


@pytest.mark.parametrize("name,world", [("diamond8_64", 2), ("diamond8_64", 3), ("spin_diamond_24", 3)])
def test_emulated_ranks_equal_one_cell(golden, name, world):
    """2 or 3 ranks each transforming their bands: every rank ends with the
    same state, equal to one context stepping all bands to rounding (the
    density is summed in another order) and to the reference build."""
    mk = {"diamond8_64": (configs.diamond8_64, 4, 2),
          "spin_diamond_24": (lambda: configs.spin_diamond(24, ne=(4, 3)), 3, 2)}
    spec, ncalls, inner = mk[name]
    inp = inputs.build_inputs(spec())
    E0, s0 = _ordinary(inp, ncalls, inner)
    E1, states = _group(inp, ncalls, inner, world)
    for r in range(world):
        assert np.array_equal(E1[:, r], E1[:, 0])
        assert np.array_equal(states[r].c2, states[0].c2)
    assert np.abs(E1[:, 0] - E0).max() < 1e-10
    assert np.abs(states[0].c2 - s0.c2).max() < 1e-12
    assert np.abs(states[0].lmd - s0.lmd).max() < 1e-11
    rows = [(E1[k, 0], 0.0, 0.0) for k in range(ncalls)]
    g = golden(name)
    assert np.abs(np.array([r[0][0] for r in rows]) - g["E"][:, 0]).max() < 1e-9
    assert np.abs(states[0].lmd - g["lmd"]).max() < 1e-9


def test_band_range_refuses_what_it_does_not_split():
    from cpsd_b200 import lib
    inp = inputs.build_inputs(configs.small_diamond(24, 4))
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    for lo, hi in ((-1, 2), (3, 2), (0, 5)):
        with pytest.raises(lib.CpsdError):
            cell.set_band_range(lo, hi)
    cell.set_band_range(0, 2)
    with pytest.raises(lib.CpsdError):
        cell.run(1)  # band-parallel contexts step by phases
    cell.set_band_range(0, -1)
    cell.run(1)
    cell.close()


def test_nccl_exchange_with_one_rank_is_the_ordinary_step():
    """The torch.distributed (NCCL) exchange on the context's stream, one
    rank: the all-reduce and the broadcasts leave the ordinary step's bits."""
    import torch.distributed as dist
    inp = inputs.build_inputs(configs.small_diamond(24, 6, ecut=20.0, seed=13))
    E0, s0 = _ordinary(inp, 2, 2)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        cell = api.GpuCell(inp)
        cell.set_state(inp.c2, inp.r2)
        ranges = bands.band_ranges(inp.nbands, 1)
        cell.set_band_range(*ranges[0])
        ex = bands.TorchExchange(torch, dist, cell, ranges)
        E1 = np.array([bands.run([cell], ex, 2)[0] for _ in range(2)])
        st = api.State(inp)
        cell.get_state(st)
        cell.close()
    finally:
        dist.destroy_process_group()
    assert np.array_equal(E0, E1)
    assert np.array_equal(s0.c2, st.c2)
