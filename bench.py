#!/usr/bin/env python
"""Benchmark of the B200 steepest-descent engine (SD steps/s).

One bench *step* is one call of the reference's ``cpsd()`` with inner=10 (one
outer iteration of ccpsdv3/main.c:417-445): ten steepest-descent steps plus
the energy evaluation.  ``value`` is SD steps per second of the whole job
(all replicas), device-timed with CUDA events on the engine's stream, the
cell resident in HBM and L2 flushed (256 MB write) before every timed call.
``e2e`` is the same metric through the drop-in ``cpsd()`` C ABI with host
buffers in the reference's layouts, the host<->device copies inside the
timed region.  ``--impl reference`` times the reference's own serial C
(oracle/_ref, ccpsdv3/*.c compiled unmodified) on the host cores.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
Multi-GPU (torchrun, one process per GPU): `value` is every rank running its
own replica of the cell (weak scaling), timed between barriers, max over
ranks; `extra` adds the 48-cell batched draw sharded over the ranks (no
exchange in the step) and the 128^3 / 128-band cell stepped band-parallel by
all ranks (densities all-reduced and orbital rows broadcast over NCCL, per
SD step).  At one GPU the band-parallel extra runs two emulated ranks on the
one device (the phases' overhead, not a speed-up).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "simple-cpsd_b200"))

METRIC = "SD steps/s"
FALLBACK_HBM_GBS = 6650.0


# ----------------------------------------------------------------- helpers
def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def phase_bytes(geo, nb, n, ispin):
    """Algorithmic bytes per launch of the single-kernel phases (FP64).

    T  = nb*n*ncol complex (column buffer after the kz transform),
    Pk = nb*npw complex (packed orbitals), R = n^3 doubles (real grid)."""
    cb = 16
    T = nb * n * geo["ncol"] * cb
    Pk = nb * geo["npw"] * cb
    R = n ** 3 * 8
    return {
        "inv_z_bands": Pk + T,                        # packed psi in, columns out
        "density_plane": T + geo["dens_chunks"] * R,  # columns in, density partials out
        "density_xc": geo["dens_chunks"] * R + (3 + 2 * ispin) * R,
        "applyv_plane": 2 * T + ispin * R,            # columns in and out, V(r) in
        "fwd_z_sd": T + 4 * Pk,                       # columns in; c2, c1 in; cpsi, c2 out
    }


def model_bytes(geo, nb, n, ispin, s_fft=16):
    """Algorithmic bytes per launch under the transform model: a 3-D
    transform is two passes, each one read and one write of the half box
    (Nh = (n/2+1) n^2 complex, s_fft bytes each); packed coefficient streams
    are nb*npw*16 bytes, real-grid fields n^3*8.  The engine's passes are z
    (inv_z / fwd_z) and y+x planes (plane kernels), one model pass each.  The
    V psi plane kernel also redoes each band's inverse plane pass instead of
    storing psi(r); the model does not count that re-computation."""
    pass_b = 2 * (n // 2 + 1) * n * n * s_fft
    Pk = nb * geo["npw"] * 16
    R = n ** 3 * 8
    return {
        "inv_z_bands": nb * pass_b + Pk,             # c1 in; inverse z pass of every band
        "density_plane": nb * pass_b + ispin * R,    # inverse plane pass of every band; density out
        "applyv_plane": nb * pass_b + ispin * R,     # forward plane pass of every band; V(r) in
        "fwd_z_sd": nb * pass_b + 4 * Pk,            # forward z pass; c2, c1 in; cpsi, c2 out
    }


def step_model_bytes(nb, n, npw, s_fft=16):
    """The same model for a whole SD step: 2 nb + 2 transforms, six packed
    coefficient streams (c1, c2, H psi read and write), six real-grid fields."""
    return (2 * nb + 2) * 4 * (n // 2 + 1) * n * n * s_fft + 6 * nb * npw * 16 + 6 * n ** 3 * 8


def traffic_from_profile(kernel, workload):
    """dram bytes per launch from a committed ncu summary, if there is one."""
    path = os.path.join(REPO, "profiles", "%s_%s.txt" % (kernel, workload))
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x, dist, torch, device):
    """The slowest rank's time (replicas are timed independently)."""
    if dist is None:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------- CPU reference
def cpu_reference(inp, budget_s, inner, min_calls=2):
    """Time the reference's own cpsd() (oracle/_ref) on this host's cores:
    calls of `inner` SD steps + energies, the same call the GPU arm times."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # test infrastructure: only the baseline leg runs it
    try:
        impl, kind = oracle.ReferenceBuild(), "reference"
    except FileNotFoundError:
        impl, kind = oracle.Restatement(), "port"
    st = oracle.State(inp)
    calls, t0 = 0, time.perf_counter()
    while calls < min_calls or time.perf_counter() - t0 < budget_s:
        impl.run(inp, inner, st)
        calls += 1
    dt = time.perf_counter() - t0
    return calls * inner / dt, kind, calls, dt


def time_kbpp(nfft=128, lmax=3, unit=20.5, reps=3, ref=True):
    """The input pipeline's KB tables (cpsd_gpu_kbpp: host arrays in and out,
    copies included) on the 128^3 grid of the 64-atom cell, s+p+d channels,
    501 radial points; beside it the reference's own kbpp() (oracle/_ref,
    one host thread, as the formatter runs) on the same table and grid."""
    import numpy as np
    from cpsd_b200 import api, inputs, psp
    t = psp.radial_table(lmax, seed=3)
    _, _, unitg = inputs.get_cube(1, unit)
    G = inputs.get_g(nfft, unitg)
    nfft3d = (nfft // 2 + 1) * nfft * nfft
    api.kbpp(t, G, nfft3d)
    t0 = time.perf_counter()
    for _ in range(reps):
        vl, vnl, _, _ = api.kbpp(t, G, nfft3d)
    gpu_s = (time.perf_counter() - t0) / reps
    out = {"grid": nfft, "g_points": nfft3d, "radial_points": t.nrho, "lmax": lmax,
           "gpu_e2e_ms": round(gpu_s * 1e3, 3), "timing": "host wall clock around the C-ABI call, mean of %d" % reps,
           "bytes_h2d": 8 * (3 * nfft3d + (2 * lmax + 3) * t.nrho),
           "bytes_d2h": 8 * (1 + lmax * lmax) * nfft3d}
    if ref:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle  # test infrastructure: only the baseline leg runs it
        try:
            t0 = time.perf_counter()
            rvl, rvnl, _, _ = oracle.reference_kbpp(t.zv, lmax, t.rho, t.vp, t.wp, t.drho, G, nfft3d)
            ref_s = time.perf_counter() - t0
            out["reference_cpu_s"] = round(ref_s, 3)
            out["reference_cores"] = 1
            out["speedup_e2e"] = round(ref_s / gpu_s, 1)
            out["max_rel_diff_vl"] = float(np.abs(vl - rvl).max() / np.abs(rvl).max())
        except FileNotFoundError:
            out["reference_cpu_s"] = None
    return out


# ----------------------------------------------------------------- GPU arm
def time_cell(inp, steps, warmup, inner, torch, dist, want_phases=True, precision=0, gemm=0, tune=True):
    """Device time of `steps` cpsd() calls of `inner` SD steps on a resident
    cell.  The kernel choices come from the library's autotuner (timed on
    the cell before the warm-up, outside the timed region).  The timed calls
    run the production schedule (no phase events: the step's second stream
    overlaps the density chain); the per-phase times come from two extra
    calls with phase events, which serialise the step."""
    from cpsd_b200 import api
    cell = api.GpuCell(inp, precision=precision)
    if gemm:
        cell.set_gemm(gemm)
    cell.set_state(inp.c2, inp.r2)
    tuned = cell.autotune(steps=10 if inp.nbands <= 32 else 3) if tune else None
    stream = torch.cuda.ExternalStream(cell.stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(warmup):
        cell.run(inner)
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = cell.counters()[0]
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()  # L2 flush on the engine's stream, outside the event pair
        events[k][0].record(stream)
        cell.run(inner)
        events[k][1].record(stream)
    torch.cuda.synchronize()
    launches = cell.counters()[0] - l0
    if dist is not None:
        dist.barrier()
    total_ms = sum(a.elapsed_time(b) for a, b in events)
    ph = {}
    if want_phases:
        cell.phase_timing(True)
        phases = {}
        for _ in range(2):
            cell.run(inner)
            for name, ms in cell.phase_times().items():
                phases.setdefault(name, []).append(ms)
        ph = {k: sum(v) / len(v) for k, v in phases.items()}
    geo = cell.geometry()
    geo["tuning"] = tuned
    E = cell.E.copy()
    cell.close()
    return total_ms, launches, ph, geo, E


def time_cufft(n, nb, torch, double=True, reps=5):
    """The V psi application of every band through cuFFT (torch.fft), as a
    cuFFT-based engine would run it on the full half box: batched 3-D c2r,
    multiply by V(r), batched 3-D r2c.  A timed comparison only; the
    engine's own transforms are the product."""
    cdt = torch.complex128 if double else torch.complex64
    rdt = torch.float64 if double else torch.float32
    g = torch.Generator(device="cuda").manual_seed(1)
    X = torch.randn(nb, n, n, n // 2 + 1, dtype=cdt, device="cuda", generator=g)
    V = torch.randn(n, n, n, dtype=rdt, device="cuda", generator=g)
    for _ in range(2):
        torch.fft.rfftn(torch.fft.irfftn(X, s=(n, n, n), dim=(1, 2, 3)) * V, dim=(1, 2, 3))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        torch.fft.rfftn(torch.fft.irfftn(X, s=(n, n, n), dim=(1, 2, 3)) * V, dim=(1, 2, 3))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del X, V
    torch.cuda.empty_cache()
    return ms


def cufft_entry(ph, n, nb, torch, double):
    """cuFFT's batched full-box V psi against the engine's sphere-pruned
    pass of the same work (kz inverse + the V psi plane pass + kz forward
    with the SD epilogue), both device-timed."""
    eng = sum(ph.get(k, 0.0) for k in ("inv_z_bands", "applyv_plane", "fwd_z_sd"))
    cu = time_cufft(n, nb, torch, double)
    return {"cufft_ms": round(cu, 4), "engine_ms": round(eng, 4), "engine_speedup": round(cu / eng, 2) if eng else None,
            "work": "V psi of %d bands on %d^3: c2r, x V(r), r2c (%s)" % (nb, n, "FP64" if double else "FP32"),
            "cufft": "torch.fft.irfftn / rfftn, batched, full half box",
            "engine": "inv_z + plane V psi + fwd_z (sphere-pruned), phase times"}


def time_batched(specs, inner, calls):
    """Config-4 cells: one graph per SD step for all cells vs the cells one by one."""
    from cpsd_b200 import api, inputs
    inps = [inputs.build_inputs(s) for s in specs]
    cells = []
    for inp in inps:
        c = api.GpuCell(inp)
        c.set_state(inp.c2, inp.r2)
        cells.append(c)
    for c in cells:  # warm-up (captures each cell's own graphs)
        c.run(inner)
    t0 = time.perf_counter()
    for _ in range(calls):
        for c in cells:
            c.run(inner)
    t_seq = time.perf_counter() - t0
    batch = api.GpuBatch(cells)
    batch.run(inner)  # warm-up (captures the batch graphs)
    l0 = batch.launches()
    t0 = time.perf_counter()
    for _ in range(calls):
        batch.run(inner)
    t_bat = time.perf_counter() - t0
    launches = batch.launches() - l0
    batch.close()
    for c in cells:
        c.close()
    sd = len(cells) * inner * calls
    return {"cells": len(cells), "grids": sorted(set(s.nfft for s in specs)),
            "bands": [min(s.ne[0] for s in specs), max(s.ne[0] for s in specs)],
            "batched_steps_per_s": sd / t_bat, "sequential_steps_per_s": sd / t_seq,
            "speedup": t_seq / t_bat, "gpu_launches": launches, "timing": "host wall clock, synchronous calls"}


def time_band_parallel(torch, dist, world, rank, calls=2, inner=2, emulate=1):
    """Band-parallel SD of the 128^3 / 128-band cell: this rank steps its
    bands, the densities are all-reduced and the orbital rows broadcast over
    the process group (cpsd_b200.bands.TorchExchange, NCCL), device-timed on
    the cell's stream, max over ranks.  With no process group, `emulate`
    contexts on this GPU stand in for the ranks (LocalGroup, stepped phase by
    phase): that measures the phases' overhead, not a speed-up."""
    from cpsd_b200 import api, bands, configs, inputs
    inp = inputs.build_inputs(configs.diamond64_128())
    nr = world if dist is not None else emulate
    ranges = bands.band_ranges(inp.nbands, nr)
    mine = [rank] if dist is not None else list(range(nr))
    cells = []
    for r in mine:
        c = api.GpuCell(inp)
        c.set_state(inp.c2, inp.r2)
        c.set_band_range(*ranges[r])
        cells.append(c)
    ex = bands.TorchExchange(torch, dist, cells[0], ranges) if dist is not None else \
        bands.LocalGroup(torch, cells, ranges)
    bands.run(cells, ex, inner)  # warm-up
    stream = torch.cuda.ExternalStream(cells[0].stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(calls):
        bands.run(cells, ex, inner)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        dist.barrier()
    ms = max_over_ranks(ms, dist, torch, "cuda")
    E = cells[0].E.copy()
    for c in cells:
        c.close()
    return {"ranks": nr, "emulated": dist is None, "ms_per_sd_step": ms / (calls * inner),
            "final_energy": float(E[0]), "bands_per_rank": [hi - lo for lo, hi in ranges],
            "timing": "CUDA events on the stepping stream, %d calls of %d SD steps, max over ranks" % (calls, inner)}


def time_cells_sharded(torch, dist, world, rank, calls=3, inner=10):
    """The 48-cell batched draw sharded over the ranks (cpsd_b200.shards:
    longest-processing-time split, one batched graph per SD step per rank,
    no exchange in the step): SD steps of all cells per second, wall time
    between barriers, max over ranks."""
    from cpsd_b200 import api, configs, inputs, shards
    specs = configs.batched_cells(0)
    mine = shards.assign(specs, world)[rank]
    cells = []
    for i in mine:
        inp = inputs.build_inputs(specs[i])
        c = api.GpuCell(inp)
        c.set_state(inp.c2, inp.r2)
        cells.append(c)
    batch = api.GpuBatch(cells) if cells else None
    if batch:
        batch.run(inner)  # warm-up (captures the batch graphs)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(calls):
        if batch:
            batch.run(inner)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    if dist is not None:
        dist.barrier()
    dt = max_over_ranks(dt, dist, torch, "cuda")
    if batch:
        batch.close()
    for c in cells:
        c.close()
    sd = len(specs) * calls * inner
    return {"cells": len(specs), "ranks": world, "value": sd / dt, "unit": "SD steps/s (all cells)",
            "cells_on_rank0": len(shards.assign(specs, world)[0]), "scaling": "strong (fixed 48 cells)",
            "timing": "host wall clock between barriers around synchronous batched calls, max over ranks"}


def e2e_dropin(inp, calls, inner):
    """Through the reference-facing cpsd() with host buffers (copies timed)."""
    from cpsd_b200 import api
    st = api.State(inp)
    api.cpsd(inp, st, inner)  # warm-up: builds the drop-in's context
    l0, h0, d0 = api.dropin_counters()
    t0 = time.perf_counter()
    for _ in range(calls):
        api.cpsd(inp, st, inner)
    dt = time.perf_counter() - t0
    l1, h1, d1 = api.dropin_counters()
    return calls * inner / dt, (h1 - h0) / calls, (d1 - d0) / calls, l1 - l0


def roofline_entry(ph, geo, nb, n, ispin, workload, sd_step_ms):
    """The longest single-kernel phase against the measured HBM copy rate,
    with the model's bytes per launch (model_bytes); the pruned bytes the
    kernel must move at least (phase_bytes) are given beside them, and the
    whole SD step against the same model."""
    pb = phase_bytes(geo, nb, n, ispin)
    mb = model_bytes(geo, nb, n, ispin)
    cand = {k: v for k, v in ph.items() if k in mb and v > 0}
    if not cand:
        return None
    top = max(cand, key=cand.get)
    peak, src = peaks()
    t = cand[top] * 1e-3
    achieved = mb[top] / t / 1e9
    total = sum(v for v in ph.values() if v > 0)
    sb = step_model_bytes(nb, n, geo["npw"])
    step_gbs = sb / (sd_step_ms * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": top, "achieved": round(achieved, 1), "peak": peak,
            "peak_source": src, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": traffic_from_profile(top, workload), "algorithmic_bytes": mb[top],
            "bytes_model": "2 passes x (read + write) of the half box per 3-D transform, FP64",
            "pruned_bytes": pb[top], "frac_pruned": round(pb[top] / t / 1e9 / peak, 4),
            "launch_ms": round(cand[top], 5), "share_of_step": round(cand[top] / total, 3) if total else None,
            "sd_step": {"bytes": sb, "ms": round(sd_step_ms, 5), "achieved": round(step_gbs, 1),
                        "frac": round(step_gbs / peak, 4)}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="diamond8_64")
    ap.add_argument("--inner", type=int, default=10)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-vs-plain extra (about a minute)")
    ap.add_argument("--no-tune", action="store_true", help="the default kernel choices (no autotuner run)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="arithmetic of the timed workload (the default line is fp64)")
    ap.add_argument("--gemm", default="fp64", choices=["fp64", "tf32x3", "tf32x3_overlaps"],
                    help="TN-product engine of a mixed-precision run")
    args = ap.parse_args()
    prec_code = {"fp64": 0, "mixed": 1}[args.precision]
    gemm_code = {"fp64": 0, "tf32x3": 1, "tf32x3_overlaps": 3}[args.gemm] if prec_code else 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(ncores))

    from cpsd_b200 import configs, inputs
    spec = configs.NAMED[args.workload]()
    inp = inputs.build_inputs(spec)
    config = {"workload": args.workload, "nfft": inp.nfft, "nbands": inp.nbands, "nion": inp.nion,
              "npw": inp.npw, "ecut_ry": spec.ecut_ry, "inner": args.inner, "precision": args.precision,
              "gemm": args.gemm if prec_code else "fp64",
              "step": "one cpsd() call: %d SD steps + energies" % args.inner,
              "l2": "flushed (256 MB write) before every timed call", "parallelism": "replicas"}

    if args.impl == "reference":
        if rank != 0:
            return 0
        steps_done, t_all = 0, 0.0
        sample_inner = args.inner  # the same cpsd() call the GPU arm times
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle
        try:
            impl, kind = oracle.ReferenceBuild(), "reference"
        except FileNotFoundError:
            impl, kind = oracle.Restatement(), "port"
        st = oracle.State(inp)
        for _ in range(args.warmup):
            impl.run(inp, sample_inner, st)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            impl.run(inp, sample_inner, st)
            steps_done += sample_inner
        t_all = time.perf_counter() - t0
        v = steps_done / t_all
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * t_all / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": dict(config, step="one reference cpsd() call: %d SD steps + energies" % sample_inner,
                               l2="n/a: the reference runs on the host cores", precision="fp64", gemm="fp64"),
                "cpu_baseline": {"value": v, "unit": "steps/s", "cores": ncores, "kind": kind,
                                 "sample": "%d reference cpsd() calls of inner=%d on %s"
                                           % (args.steps, sample_inner, args.workload)},
                "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                              device_id=torch.device("cuda", local))
        dist = td
    else:
        torch.cuda.set_device(0)

    sampler = ClockSampler(local)
    sampler.start()
    total_ms, launches, ph, geo, E = time_cell(inp, args.steps, args.warmup, args.inner, torch, dist,
                                               precision=prec_code, gemm=gemm_code, tune=not args.no_tune)
    clocks = sampler.stop()
    total_ms = max_over_ranks(total_ms, dist, torch, "cuda")
    sd_steps = args.steps * args.inner * world
    value = sd_steps / (total_ms * 1e-3)

    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if not prec_code else "f32+f64",
            "data": "synthetic (seeded)", "config": config, "gpu_launches": int(launches), "clocks": clocks,
            "final_energy": float(E[0])}
    line["roofline"] = roofline_entry(ph, geo, inp.nbands, inp.nfft, inp.ispin, args.workload,
                                      total_ms / (args.steps * args.inner))
    if geo.get("tuning"):
        config["tuning"] = geo["tuning"]["tuning"]
        config["autotune_ms_per_sd_step"] = [geo["tuning"]["ms_per_step_before"], geo["tuning"]["ms_per_step_after"]]
    line["phases_ms"] = {k: round(v, 5) for k, v in ph.items()}

    if rank == 0 and not args.no_e2e:
        ev, hb, db, _ = e2e_dropin(inp, max(3, min(args.steps, 10)), args.inner)
        line["e2e"] = {"value": ev * world, "unit": "steps/s", "h2d_bytes_per_step": int(hb),
                       "d2h_bytes_per_step": int(db),
                       "path": "drop-in cpsd() C ABI, host buffers in the reference layout"}
    if rank == 0 and world == 1 and not args.no_cpu:
        cv, kind, calls, dt = cpu_reference(inp, args.cpu_budget, args.inner)
        line["cpu_baseline"] = {"value": cv, "unit": "steps/s", "cores": ncores, "kind": kind,
                                "sample": "%d reference cpsd() calls of inner=%d on %s (%.1f s)"
                                          % (calls, args.inner, args.workload, dt)}
    if rank == 0 and world == 1 and not args.no_extra:
        from cpsd_b200 import configs as C
        extra = {}
        # the same workload with FP32 transforms (mixed precision)
        tmx, _, phm, _, Em = time_cell(inp, args.steps, args.warmup, args.inner, torch, None,
                                       want_phases=True, precision=1)
        extra["mixed_" + args.workload] = {
            "value": sd_steps / (tmx * 1e-3), "unit": "steps/s", "ms_per_step": tmx / args.steps,
            "final_energy": float(Em[0]), "abs_dE_vs_fp64_same_steps": abs(float(Em[0]) - float(E[0])),
            "phases_ms": {k: round(v, 5) for k, v in phm.items()}}
        extra["cufft_" + args.workload] = cufft_entry(ph, inp.nfft, inp.nbands, torch, True)
        extra["cufft_mixed_" + args.workload] = cufft_entry(phm, inp.nfft, inp.nbands, torch, False)
        # config 4: 48 uneven cells, one graph launch per SD step for all of them
        extra["batched_cells"] = time_batched(C.batched_cells(0), args.inner, 3)
        # the learned path (committed network, plain SD as the fallback) against
        # plain FP64 SD run to convergence from the same start (E_conv: the
        # energy changes by < 1e-10 Ha over five blocks of 200 steps): steps and
        # wall time to |E - E_conv| <= 1e-6 Ha/atom, the learned end state's
        # distance from E_conv and its drift under continued plain SD
        from cpsd_b200 import learned
        if os.path.exists(learned.PRETRAINED) and not args.no_learned:
            mlp = learned.load_pretrained()
            evs = []
            for seed in (5000, 5001):  # gapped control: H2 molecules, one minimum
                ev = learned.study_cell(inputs.build_inputs(C.h2_molecules(seed=seed)), mlp, plain_max=100000,
                                        learned_max=20000, precision=0, gemm=0)
                ev["cell"] = "h2_molecules seed %d (held out)" % seed
                evs.append(ev)
            ev = learned.study_cell(inputs.build_inputs(C.diamond8_64(seed=5000)), mlp, plain_max=600000,
                                    learned_max=40000)
            ev["cell"] = "diamond8_64 seed 5000 (held out)"
            evs.append(ev)
            mlp.close()
            extra["learned_vs_plain"] = evs
        # the 128^3 / 64-atom / 128-band cell of the precision study, FP64
        big = inputs.build_inputs(C.diamond64_128())
        tms, lch, ph3, geo3, E3 = time_cell(big, 3, 1, args.inner, torch, None)
        tmm, _, ph3m, _, E3m = time_cell(big, 3, 1, args.inner, torch, None, precision=1)
        extra["mixed_diamond64_128"] = {"value": 3 * args.inner / (tmm * 1e-3), "unit": "steps/s",
                                        "ms_per_sd_step": tmm / (3 * args.inner),
                                        "phases_ms": {k: round(v, 4) for k, v in ph3m.items()}}
        extra["cufft_diamond64_128"] = cufft_entry(ph3, big.nfft, big.nbands, torch, True)
        extra["cufft_mixed_diamond64_128"] = cufft_entry(ph3m, big.nfft, big.nbands, torch, False)
        # the same with the TN products on the tensor cores (3xTF32, tcgen05)
        for key, mode in (("mixed_tf32x3_diamond64_128", 1), ("mixed_tf32x3_overlaps_diamond64_128", 3)):
            tmt, _, ph3t, _, _ = time_cell(big, 3, 1, args.inner, torch, None, precision=1, gemm=mode)
            extra[key] = {"value": 3 * args.inner / (tmt * 1e-3), "unit": "steps/s",
                          "ms_per_sd_step": tmt / (3 * args.inner),
                          "phases_ms": {k: round(v, 4) for k, v in ph3t.items()}}
        line["extra"] = extra
        # input pipeline: KB tables of a tabulated psp on the 128^3 grid
        extra["kbpp_128"] = time_kbpp()
        extra["diamond64_128"] = {
            "value": 3 * args.inner / (tms * 1e-3), "unit": "steps/s",
            "ms_per_sd_step": tms / (3 * args.inner), "npw": big.npw, "nbands": big.nbands,
            "tuning": (geo3.get("tuning") or {}).get("tuning"),
            "phases_ms": {k: round(v, 4) for k, v in ph3.items()},
            "roofline": roofline_entry(ph3, geo3, big.nbands, big.nfft, big.ispin, "diamond64_128",
                                       tms / (3 * args.inner))}
    if world > 1 and not args.no_extra:
        # multi-GPU: the 48-cell draw sharded over the ranks, and one 128^3
        # cell stepped band-parallel by all of them (every rank takes part)
        mg = {"cells_sharded": time_cells_sharded(torch, dist, world, rank),
              "band_parallel_diamond64_128": time_band_parallel(torch, dist, world, rank)}
        line.setdefault("extra", {}).update(mg)
    elif rank == 0 and not args.no_extra:
        line["extra"]["band_parallel_emulated_diamond64_128"] = time_band_parallel(torch, None, 1, 0, emulate=2)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
