"""Host-side logic that needs no GPU: the C ABI exports, reference file
formats, workload generation, bench helpers and the multi-rank reduction."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO
from cpsd_b200 import build, configs, inputs, lib, refio


def header_functions():
    with open(os.path.join(REPO, "include", "cpsd_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "sizeof")))


def test_library_builds_and_exports_every_declared_symbol():
    so = build.build_library()
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if " T " in line)
    declared = header_functions()
    assert declared, "no declarations parsed"
    assert set(declared) <= exported, sorted(set(declared) - exported)
    assert set(declared) == set(lib.EXPORTS)


def test_library_targets_sm100a_only():
    """The build compiles for sm_100a alone (no PTX for other targets)."""
    flags = " ".join(build.NVCC_FLAGS)
    assert re.findall(r"arch=compute_(\w+),code=(\w+)", flags) == [("100a", "sm_100a")]


def test_missing_library_fails_loudly(tmp_path):
    saved = lib._lib
    lib._lib = None
    try:
        with pytest.raises(FileNotFoundError):
            lib.load(str(tmp_path / "nope.so"))
    finally:
        lib._lib = saved


def test_elcin_roundtrip(tmp_path):
    inp = inputs.build_inputs(configs.small_h2(16))
    p = str(tmp_path / "ELCIN")
    refio.write_elcin(p, 1, inp.nfft, 10.0, 1, inp.ne, inp.c2)
    back = refio.read_elcin(p)
    assert back["nfft"] == 16 and back["ne"] == (1, 0) and back["unit"] == 10.0
    assert np.array_equal(back["c"], inp.c2)
    # the header is the reference's: 4+4+8+4+8 bytes (main.c:116-121)
    assert os.path.getsize(p) == 28 + 8 * inp.c2.size


def test_reference_inputs_written(tmp_path):
    inp = inputs.build_inputs(configs.small_diamond(16, 2, ecut=10.0))
    refio.write_reference_inputs(str(tmp_path), inp, inner=2, outer=3)
    names = sorted(os.listdir(tmp_path))
    assert names == ["C0.vpp", "CONTROL", "ELCIN", "IONIN"]
    nfft3d = inp.nfft3d
    # .vpp: 4+4+8+2+8+8+4 header, rc[lmax+1], vnlnrm[lmmax], vl, vnl[lmmax]
    want = 38 + 8 * (3 + 4 + nfft3d + 4 * nfft3d)
    assert os.path.getsize(tmp_path / "C0.vpp") == want
    ion = open(tmp_path / "IONIN").read().split()
    assert ion[0] == "1" and ion[1] == "'C0.vpp" and ion[3] == "2" and ion[4] == "8"


def test_parse_reference_stdout():
    text = """          ================ iteration =========================
          >>>   iteration started on Thu Dec  3 12:00:23 2026    <<<
       2    8.6420275970e+01  7.45002e+00  4.77763e-01  0.00000e+00
       4    7.1368710863e+01 -1.29755e+00  4.82470e-01  0.00000e+00
          *** arrived at the maximum iteration.  iteration terminated.
 total     energy    : 5.6634818000e+01 ( 7.07935e+00/ion)
 KS V_xc energy      :-2.0458754790e+00 (-5.11469e-01/electron)
"""
    rows, final = refio.parse_reference_stdout(text)
    assert rows == [(2, 86.42027597, 7.45002, 0.477763, 0.0), (4, 71.368710863, -1.29755, 0.48247, 0.0)]
    assert final == {0: 56.634818, 9: -2.045875479}


def test_batched_cells_follow_the_recipe():
    cells = configs.batched_cells(seed=0)
    assert len(cells) == 48
    for c in cells:
        assert c.nfft in (32, 48, 64) and c.unit == 0.5 * c.nfft and c.ecut_ry == 30.0
        assert 2 <= len(c.katm) <= 16 and 4 <= c.ne[0] <= 32
        z = sum(4.0 if k else 1.0 for k in c.katm)
        assert c.ne[0] >= min(32, np.ceil(z / 2))
        p = c.positions
        for i in range(len(p)):
            for j in range(i):
                d = p[i] - p[j]
                d -= c.unit * np.round(d / c.unit)
                assert np.sqrt(d @ d) >= 1.5 - 1e-12


def test_analytic_psp_limits():
    """vl(G) -> -4 pi Z/G^2 at small rc, vl(0) = pi Z rc^2, projector norms."""
    sp = configs.C_SP
    spec = configs.small_diamond(24, 2, ecut=20.0)
    inp = inputs.build_inputs(spec)
    G = inp.G
    vl, vnl, vnlnrm = inputs.analytic_psp(sp, G, inp.nfft3d)
    assert vl[0] == pytest.approx(np.pi * sp.zv * sp.rc_loc ** 2)
    assert np.all(vnlnrm[:4] == [1.0 / sp.ekb[0]] + [1.0 / sp.ekb[1]] * 3)
    # |p_s>: int |p|^2 = 1  <=>  sum_G |vnl|^2 / Omega (full sphere) -> 1 for a big cell
    a = 40.0
    omega, _, unitg = inputs.get_cube(1, a)
    Gb = inputs.get_g(64, unitg)
    n3 = (64 // 2 + 1) * 64 * 64
    _, vb, _ = inputs.analytic_psp(sp, Gb, n3)
    s = inputs.gssum_np(64, vb[:n3] ** 2) / omega
    assert s == pytest.approx(1.0, rel=1e-6)


def test_bench_roofline_helpers():
    sys.path.insert(0, REPO)
    import bench
    geo = dict(npw=2483, npw_pad=2496, ncol=300, KX=11, nproj=32, dens_chunks=5)
    pb = bench.phase_bytes(geo, 16, 64, 1)
    T = 16 * 64 * 300 * 16
    assert pb["applyv_plane"] == 2 * T + 64 ** 3 * 8
    r = bench.roofline_entry({"applyv_plane": 0.01, "density_plane": 0.005}, geo, 16, 64, 1, "x", 0.1)
    assert r["kernel"] == "applyv_plane" and r["unit"] == "GB/s" and r["bound"] == "hbm"
    # transform model: one pass (read + write of the half box) per band, plus V(r)
    Nh = 33 * 64 * 64
    model = 16 * 2 * Nh * 16 + 64 ** 3 * 8
    assert r["algorithmic_bytes"] == model
    assert r["achieved"] == pytest.approx(model / 1e-5 / 1e9, rel=1e-3)
    assert r["pruned_bytes"] == pb["applyv_plane"]
    assert r["frac_pruned"] == pytest.approx(pb["applyv_plane"] / 1e-5 / 1e9 / r["peak"], rel=1e-3)
    # whole step: (2 nb + 2) transforms, six coefficient streams, six grid fields
    sb = 34 * 4 * Nh * 16 + 6 * 16 * 2483 * 16 + 6 * 64 ** 3 * 8
    assert r["sd_step"]["bytes"] == sb
    assert r["sd_step"]["achieved"] == pytest.approx(sb / 1e-4 / 1e9, rel=1e-3)


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = bench.max_over_ranks(10.0 + rank, dist, torch, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_replica_timing_takes_the_slowest_rank():
    """bench.py's multi-rank path: every rank gets the max over ranks (gloo, 2 ranks)."""
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 11.0, 1: 11.0}


@pytest.mark.parametrize("threads", ["1", "3", "16"])
def test_host_pool_runs_every_item_once(tmp_path, threads):
    """The host thread pool behind the drop-in's layout conversion: thousands
    of jobs back to back, each item exactly once, for 1, 3 and 16 threads."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "pool_check")
    src = os.path.join(REPO, "tests", "host_pool_check.cpp")
    inc = os.path.join(REPO, "simple-cpsd_b200", "csrc")
    subprocess.run([cxx, "-O2", "-std=c++17", "-pthread", "-I", inc, src, "-o", exe], check=True)
    env = dict(os.environ, CPSD_B200_HOST_THREADS=threads)
    out = subprocess.run([exe], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok %s threads" % threads)



def test_new_entry_points_report_errors_without_a_gpu(tmp_path):
    """Host-side checks of the epilogue writers and the input pipeline: bad
    arguments and unwritable files come back as status codes, before any
    device work (so they hold on a machine without a GPU)."""
    from cpsd_b200 import api
    L = lib.load()
    assert "eigen" in lib.strerror(lib.CPSD_ERR_EIG)
    assert "file" in lib.strerror(lib.CPSD_ERR_IO)
    inp = inputs.build_inputs(configs.small_h2(16))
    c1 = np.zeros(inp.nbands * inp.n2ft3d)
    with pytest.raises(lib.CpsdError) as e:
        api.write_elcout(str(tmp_path / "no_such_dir" / "ELCOUT"), inp, c1)
    assert e.value.status == lib.CPSD_ERR_IO
    with pytest.raises(ValueError):
        api.write_elcout(str(tmp_path / "ELCOUT"), inp, c1[:-1])
    ne = np.array([1, 0], dtype=np.int32)
    assert L.cpsd_write_elcout(None, 1, 16, 20.0, 1, api._ptr(ne), api._ptr(c1)) == lib.CPSD_ERR_ARG
    assert L.cpsd_write_ionout(str(tmp_path / "IONOUT").encode(), 1, None, None, 0, None, None) == lib.CPSD_ERR_ARG
    # kbpp: lmax above 3, too few radial points, and missing outputs are refused up front
    from cpsd_b200 import psp
    t = psp.radial_table(2, seed=2)
    G = inputs.get_g(16, inputs.get_cube(1, 10.26)[2])
    nfft3d = 9 * 16 * 16
    vp = t.vp.copy()
    out = np.zeros(9 * nfft3d)
    P = api._ptr
    assert L.cpsd_gpu_kbpp(4.0, 4, t.nrho, t.drho, P(t.rho), P(vp), P(t.wp), nfft3d, P(G), P(out), P(out),
                           P(out)) == lib.CPSD_ERR_ARG
    assert L.cpsd_gpu_kbpp(4.0, 2, 1, t.drho, P(t.rho), P(vp), P(t.wp), nfft3d, P(G), P(out), P(out),
                           P(out)) == lib.CPSD_ERR_ARG
    assert L.cpsd_gpu_kbpp(4.0, 2, t.nrho, t.drho, P(t.rho), P(vp), P(t.wp), nfft3d, P(G), P(out), None,
                           None) == lib.CPSD_ERR_ARG
    assert np.array_equal(vp, t.vp)  # refused calls leave vp as it was


def test_cell_shards_cover_every_cell_once_and_balance():
    """config-4 style cells over 1..8 ranks: each cell on exactly one rank,
    and no rank above the best balance the largest cell allows."""
    from cpsd_b200 import shards
    specs = configs.batched_cells(0)
    costs = [shards.cell_cost(s) for s in specs]
    for world in (1, 2, 3, 8):
        parts = shards.assign(specs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(specs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs)
    assert shards.assign(specs, 2) == shards.assign(specs, 2)  # deterministic


def _restatement_runner(specs, calls, inner):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    R = oracle.Restatement()
    out = []
    for spec in specs:
        inp = inputs.build_inputs(spec)
        st = oracle.State(inp)
        for _ in range(calls):
            R.run(inp, inner, st)
        out.append(st.E.copy())
    return np.array(out).reshape(len(specs), -1)


def _shard_specs():
    return [configs.small_h2(16, seed=3), configs.small_diamond(24, 4, seed=5), configs.small_h2(16, seed=4)]


def _shard_rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    from cpsd_b200 import shards
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    E = shards.run_cells(_shard_specs(), 2, 1, rank=rank, world=world, dist=dist, runner=_restatement_runner)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, E))


@pytest.mark.parametrize("world", [2, 4])
def test_cell_shards_gather_equals_one_process(world):
    """gloo ranks step their shares of three cells (the restatement stands
    in for the GPU runner) and gather: every rank holds every cell's
    energies, equal to one process stepping all of them.  With 4 ranks one
    rank has no cell and still joins the gather."""
    import multiprocessing as mp
    import socket
    from cpsd_b200 import shards
    specs = _shard_specs()
    if world > len(specs):
        assert any(not p for p in shards.assign(specs, world))
    want = shards.run_cells(specs, 2, 1, runner=_restatement_runner)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    for _, E in got:
        assert np.array_equal(E, want)


def test_cell_shards_rank_without_cells_runs_nothing():
    """More ranks than cells: the empty rank never calls its runner and its
    share is an empty (0 x 10) block, so it reaches the gather."""
    from cpsd_b200 import shards
    specs = _shard_specs()
    calls = []

    def runner(s, c, i):
        calls.append(len(s))
        return _restatement_runner(s, c, i)

    parts = shards.assign(specs, 5)
    empty = [r for r, p in enumerate(parts) if not p]
    assert len(empty) == 2
    with pytest.raises(RuntimeError):  # alone, an empty rank holds no cell's energies
        shards.run_cells(specs, 1, 1, rank=empty[0], world=5, runner=runner)
    assert calls == []


# ------------------------------------------------------------ band-parallel SD
def test_band_ranges_cover_every_band_once():
    from cpsd_b200 import bands
    for nb in (1, 4, 7, 128):
        for world in (1, 2, 3, 8):
            r = bands.band_ranges(nb, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == nb
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [hi - lo for lo, hi in r]
            assert max(sizes) - min(sizes) <= 1
    assert bands.spin_split(3, 5, 4) == (1, 1)
    assert bands.spin_split(0, 4, 4) == (4, 0)
    assert bands.spin_split(5, 7, 4) == (0, 2)


def _bands_specs():
    return {"diamond": lambda: configs.small_diamond(24, 5), "spin": lambda: configs.spin_diamond(24, ne=(4, 3))}


def test_band_parallel_restatement_one_rank_is_the_restatement(restatement):
    """One rank owning every band, exchanges that do nothing: the same bits
    as the plain restatement."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    for mk in _bands_specs().values():
        inp = inputs.build_inputs(mk())
        a, b = oracle.State(inp), oracle.State(inp)
        for _ in range(2):
            restatement.run(inp, 2, a)
            restatement.run_bands(inp, 2, b, 0, inp.nbands, lambda x: None, lambda x: None)
        for x, y in ((a.E, b.E), (a.c2, b.c2), (a.lmd, b.lmd), (a.dn, b.dn), (a.cpsi, b.cpsi)):
            assert np.array_equal(x, y)


def _bands_rank_main(rank, world, port, name, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    from cpsd_b200 import bands
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    inp = inputs.build_inputs(_bands_specs()[name]())
    ranges = bands.band_ranges(inp.nbands, world)
    red, gat = bands.torch_exchange(dist, ranges)
    st = oracle.State(inp)
    R = oracle.Restatement()
    for _ in range(2):
        R.run_bands(inp, 2, st, ranges[rank][0], ranges[rank][1], red, gat)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, st.E.copy(), st.c2.copy(), st.lmd.copy(), st.dn.copy()))


@pytest.mark.parametrize("name,world", [("diamond", 2), ("spin", 2), ("spin", 3)])
def test_band_parallel_restatement_gloo_ranks_equal_one_process(restatement, name, world):
    """gloo ranks each step their bands of one cell (the restatement's
    band-parallel form), exchanging the density sum and the new orbitals:
    every rank ends with the state of one process stepping all bands, to
    rounding (the density is summed in another order).  With 3 ranks over
    4 + 3 spin bands one rank holds bands of both spins."""
    import multiprocessing as mp
    import socket
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    inp = inputs.build_inputs(_bands_specs()[name]())
    want = oracle.State(inp)
    for _ in range(2):
        restatement.run(inp, 2, want)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_bands_rank_main, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    first = got[0]
    for _, E, c2, lmd, dn in got:
        assert np.array_equal(E, first[1]) and np.array_equal(c2, first[2])  # replicated state
        assert np.abs(E - want.E).max() < 1e-10
        assert np.abs(c2 - want.c2).max() < 1e-12
        assert np.abs(lmd - want.lmd).max() < 1e-11
        assert np.abs(dn - want.dn).max() < 1e-12 * np.abs(want.dn).max()
