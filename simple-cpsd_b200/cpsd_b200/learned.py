"""Learned preconditioner for the SD update: data, training, guarded use.

The network (csrc/mlp.cuh, run and trained on the GPU) maps, per band b and
|G| shell s, the features

    x = (t_s / KE_b,  log KE_b,  log |r_b|^2,  log(1 + step) / 10)

(t_s the shell's kinetic energy, KE_b the band's kinetic energy, r_b the part
of -H psi_b orthogonal to psi_b) to log K, and each SD step becomes

    c2 = c1 + dte (cpsi + (K(b, s) - 1) R),   R = cpsi - C1 (C1' W cpsi)

before the reference's Lagrange correction: only the residual R (the part of
-H psi outside the occupied subspace) is stepped by dte K, so wherever R = 0
the step is plain SD's and the fixed point H psi = psi Lambda is unchanged.

Training targets come from SD trajectories of the method itself: at a
recorded step, with C the orbitals, G the occupied-subspace-projected
gradient and C_h the orbitals `horizon` plain steps later (aligned to C by
the orthogonal Procrustes rotation, since SD fixes only the subspace), the
per-shell least-squares step that points G at C_h - C is

    K*(b, s) = sum_{p in s} w_p Re(G_bp^* (C_h - C)_bp) / (dte sum_{p in s} w_p |G_bp|^2).

For a mode of curvature lam plain SD contracts the error by (1 - dte lam) per
step, so K* is about min(horizon, 1 / (dte lam)): one learned step stands in
for up to `horizon` plain steps on slow modes and is critically damped on
stiff ones.  Targets are clipped to the kernel's range [LOGK_MIN, LOGK_MAX].

Use is guarded: energies are compared every `inner` steps and a block that
raises the energy, or whose Lagrange iteration did not converge, is redone
from its start with plain SD, so every path is monotone in the energy and the
stationary points are plain SD's (H psi = psi Lambda does not depend on K);
on cells with several stationary points a path may still end in a different
one than plain SD from the same start.  A trust region bounds log K: it
shrinks after a rejected block and grows back after accepted ones.
"""
from __future__ import annotations

import dataclasses
import math
import os
import time
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import api, inputs

NSHELL = 64  # csrc/mlp.cuh kShells
# network trained by `python -m cpsd_b200.learned --headline` (8- and 64-atom
# jittered diamond cells); loaded by load_pretrained()
PRETRAINED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "preconditioner_diamond.npy")
LOGK_MIN, LOGK_MAX = -2.0, 4.5  # csrc/mlp.cuh kLogKMin, kLogKMax
# trust region on log K: steady state near CAP_GROW / (CAP_GROW + CAP_SHRINK)
# rejected blocks (about one in eight)
CAP_SHRINK, CAP_GROW = 0.7, 0.1


@dataclasses.dataclass
class Sphere:
    w: np.ndarray      # Gamma-point weight per sphere point
    tg: np.ndarray     # |G|^2 / 2 per sphere point
    shell: np.ndarray  # shell index per point
    tmax: float


def sphere_of(cell: api.GpuCell) -> Sphere:
    idx, w, sh = cell.sphere()
    tg = cell.inp.tg[idx]
    return Sphere(w=w, tg=tg, shell=sh, tmax=float(tg.max()))


def features(sp: Sphere, c1: np.ndarray, cpsi: np.ndarray, step: int) -> np.ndarray:
    """(nb*NSHELL, 4) float32 inputs, as the step's network pass forms them
    (prec_feature in csrc/mlp.cuh)."""
    w = sp.w
    ke = np.maximum((w * sp.tg * (c1.real ** 2 + c1.imag ** 2)).sum(1), 1e-12)
    h = (w * (c1.real * cpsi.real + c1.imag * cpsi.imag)).sum(1)
    q = (w * (cpsi.real ** 2 + cpsi.imag ** 2)).sum(1)
    res = np.maximum(q - h * h, 1e-30)
    ts = (np.arange(NSHELL) + 0.5) * sp.tmax / NSHELL
    nb = c1.shape[0]
    X = np.zeros((nb, NSHELL, 4), dtype=np.float32)
    X[:, :, 0] = ts[None, :] / ke[:, None]
    X[:, :, 1] = np.log(ke)[:, None]
    X[:, :, 2] = np.log(res)[:, None]
    X[:, :, 3] = math.log1p(step) / 10.0
    return X.reshape(-1, 4)


def gamma_dot(w: np.ndarray, A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """Matrix of Gamma-point products <A_i|B_j> (real)."""
    return (A.conj() * w) @ B.T


def targets(sp: Sphere, c1: np.ndarray, cpsi: np.ndarray, cfin: np.ndarray, dte: float):
    """(nb*NSHELL,) log K* and a validity mask (shells carrying gradient)."""
    w = sp.w
    # the residual: gradient projected out of the occupied subspace (the part
    # the preconditioner steps)
    G = cpsi - gamma_dot(w, c1, cpsi).real.T @ c1
    # align the end point to C (orthogonal Procrustes on the real overlap)
    M = gamma_dot(w, cfin, c1).real
    Uo, _, Vt = np.linalg.svd(M)
    D = (Uo @ Vt).T @ cfin - c1
    # and keep only the displacement outside the occupied subspace
    D = D - gamma_dot(w, c1, D).real.T @ c1
    num = np.zeros((c1.shape[0], NSHELL))
    den = np.zeros((c1.shape[0], NSHELL))
    prod = w * (G.real * D.real + G.imag * D.imag)
    pw = w * (G.real ** 2 + G.imag ** 2)
    for s in range(NSHELL):
        m = sp.shell == s
        if m.any():
            num[:, s] = prod[:, m].sum(1)
            den[:, s] = pw[:, m].sum(1)
    k = num / np.maximum(dte * den, 1e-300)
    valid = (den > 1e-12 * max(den.max(), 1e-300)) & (k > 0)
    logk = np.log(np.clip(k, math.exp(LOGK_MIN), math.exp(LOGK_MAX)))
    return logk.reshape(-1).astype(np.float32), valid.reshape(-1)


def record_trajectory(spec: inputs.CellSpec, nsteps: int, inner: int, every: int, horizon: int = 32):
    """Plain SD; every `every` blocks of `inner` steps record (step, c1, cpsi,
    C_h) with C_h the orbitals `horizon` steps later.  Returns (sphere,
    records, dte, energies)."""
    inp = inputs.build_inputs(spec)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    sp = sphere_of(cell)
    snaps, energies = [], []
    step = 0
    for k in range(nsteps // inner):
        cell.run(inner)
        step += inner
        energies.append(float(cell.E[0]))
        if k % every == 0:
            # c1 is the input of the block's last step, taken after step - 1 steps
            c1, _, cpsi = cell.get_packed()
            cell.run(horizon)
            step += horizon
            snaps.append((step - horizon - 1, c1, cpsi, cell.get_packed()[1]))
    dte = inp.dt / math.sqrt(inp.fmass)
    cell.close()
    return sp, snaps, dte, energies


def dataset(trajs) -> Tuple[np.ndarray, np.ndarray]:
    Xs, Ts = [], []
    for sp, snaps, dte, _ in trajs:
        for step, c1, cpsi, ch in snaps:
            X = features(sp, c1, cpsi, step)
            T, valid = targets(sp, c1, cpsi, ch, dte)
            Xs.append(X[valid])
            Ts.append(T[valid])
    return np.concatenate(Xs), np.concatenate(Ts)


def train(mlp: api.Mlp, X: np.ndarray, T: np.ndarray, steps: int = 3000, batch: int = 4096,
          lr: float = 1e-3, seed: int = 0) -> np.ndarray:
    """Shuffle once (seeded) and run `steps` Adam steps on the GPU."""
    perm = np.random.default_rng(seed).permutation(X.shape[0])
    return mlp.train(X[perm], T[perm], steps, batch, lr)


@dataclasses.dataclass
class RunResult:
    energies: List[float]          # E[0] after every block
    seconds: List[float]           # wall time since the start after every block
    steps_to_tol: Optional[int]
    seconds_to_tol: Optional[float]
    rejected_blocks: int
    steps: int
    refine_step: Optional[int] = None     # step at which a mixed run switched to FP64
    final_c2: Optional[np.ndarray] = None


def run(spec_or_inp, e_conv: Optional[float], tol_per_ion: float, max_steps: int, inner: int = 20,
        mlp: Optional[api.Mlp] = None, precision: int = 0, gemm: int = 0,
        refine_per_ion: Optional[float] = None, start_c2: Optional[np.ndarray] = None,
        keep_state: bool = False) -> RunResult:
    """SD (plain, or learned-preconditioned with plain SD as the fallback)
    until the energy is within tol_per_ion * nion of e_conv, or max_steps.

    precision/gemm select the mixed path; with refine_per_ion set, a mixed
    run switches the same context to FP64 once an accepted block changes the
    energy by less than refine_per_ion * nion (the final FP64 refinement)."""
    inp = spec_or_inp if isinstance(spec_or_inp, inputs.CpsdInputs) else inputs.build_inputs(spec_or_inp)
    cell = api.GpuCell(inp, precision=precision)
    if gemm:
        cell.set_gemm(gemm)
    cell.set_state(inp.c2, inp.r2)
    if start_c2 is not None:
        cell.set_packed(start_c2)
    tol = tol_per_ion * inp.nion
    energies, seconds, rejected, steps = [], [], 0, 0
    hit_step, hit_time, refine_step = None, None, None
    prev = math.inf
    cap = LOGK_MAX
    t0 = time.perf_counter()
    if mlp is not None:
        cell.set_preconditioner(mlp)
    while steps < max_steps:
        if mlp is not None:
            # one guarded block in the library (cpsd_gpu_run_guarded): a block
            # whose energy rises, is not finite or whose Lagrange iteration did
            # not converge is redone from its start with plain SD steps
            cell.E[0] = prev
            e, rej, cap = cell.run_guarded(inner, cap)
            rejected += rej
        else:
            e = float(cell.run(inner)[0])
        steps += inner
        energies.append(e)
        seconds.append(time.perf_counter() - t0)
        if (refine_per_ion is not None and refine_step is None and precision != 0
                and abs(e - prev) < refine_per_ion * inp.nion):
            cell.set_precision(0)  # FP64 refinement from here on
            refine_step = steps
            e = math.inf  # FP64 energies are compared among themselves only
        prev = e
        if e_conv is not None and hit_step is None and abs(e - e_conv) <= tol:
            hit_step, hit_time = steps, seconds[-1]
            break
    final = cell.get_c2() if keep_state else None
    cell.close()
    return RunResult(energies, seconds, hit_step, hit_time, rejected, steps, refine_step, final)


def first_within(res: RunResult, e_conv: float, tol: float, inner: int):
    """(steps, seconds) of the first block within tol of e_conv, or (None, None)."""
    for k, e in enumerate(res.energies):
        if abs(e - e_conv) <= tol:
            return (k + 1) * inner, res.seconds[k]
    return None, None


def converged_energy(spec_or_inp, max_steps: int, inner: int = 200, tol: float = 1e-10) -> Tuple[float, int]:
    """Plain FP64 SD until the energy changes by less than tol over each of
    five consecutive blocks of `inner` steps (or max_steps).  Returns the
    energy and the steps taken (== max_steps: not converged)."""
    inp = spec_or_inp if isinstance(spec_or_inp, inputs.CpsdInputs) else inputs.build_inputs(spec_or_inp)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    prev, steps, e, quiet = math.inf, 0, math.inf, 0
    while steps < max_steps:
        e = float(cell.run(inner)[0])
        steps += inner
        quiet = quiet + 1 if abs(e - prev) < tol else 0
        if quiet >= 5:
            break
        prev = e
    cell.close()
    return e, steps


def experiment(n_train: int = 12, n_eval: int = 4, traj_steps: int = 30000, inner: int = 100, every: int = 10,
               train_steps: int = 3000, tol_per_ion: float = 1e-6, max_steps: int = 120000,
               out: Optional[str] = None, weights: Optional[str] = None, horizon: int = 32) -> dict:
    """Train on jittered 8-atom diamond cells, evaluate steps and time to
    tol_per_ion on held-out cells against plain SD."""
    import json
    from . import configs
    t0 = time.perf_counter()
    trajs = [record_trajectory(configs.diamond8_64(seed=1000 + i), traj_steps, inner, every, horizon)
             for i in range(n_train)]
    t_traj = time.perf_counter() - t0
    X, T = dataset(trajs)
    mlp = api.Mlp(seed=0)
    t0 = time.perf_counter()
    losses = train(mlp, X, T, steps=train_steps)
    t_train = time.perf_counter() - t0
    if weights:
        np.save(weights, mlp.params)
    evals = []
    for i in range(n_eval):
        inp = inputs.build_inputs(configs.diamond8_64(seed=5000 + i))
        e_conv, conv_steps = converged_energy(inp, max_steps=max_steps)
        plain = run(inp, e_conv, tol_per_ion, max_steps, inner=inner)
        lrn = run(inp, e_conv, tol_per_ion, max_steps, inner=inner, mlp=mlp)
        evals.append({"seed": 5000 + i, "e_conv": e_conv, "conv_steps": conv_steps,
                      "plain_steps": plain.steps_to_tol, "plain_s": plain.seconds_to_tol,
                      "learned_steps": lrn.steps_to_tol, "learned_s": lrn.seconds_to_tol,
                      "learned_rejected_blocks": lrn.rejected_blocks,
                      "learned_final_abs_dE_per_ion": abs(lrn.energies[-1] - e_conv) / inp.nion})
    res = {"train_cells": n_train, "samples": int(X.shape[0]), "trajectory_steps": traj_steps, "horizon": horizon,
           "trajectory_seconds": t_traj, "train_steps": train_steps, "train_seconds": t_train,
           "loss_first": float(losses[0]), "loss_last": float(np.mean(losses[-50:])),
           "tol_per_ion": tol_per_ion, "eval": evals}
    ok = [e for e in evals if e["plain_steps"] and e["learned_steps"]]
    if ok:
        res["mean_step_ratio_plain_over_learned"] = float(np.mean([e["plain_steps"] / e["learned_steps"] for e in ok]))
        res["mean_time_ratio_plain_over_learned"] = float(np.mean([e["plain_s"] / e["learned_s"] for e in ok]))
    if out:
        with open(out, "w") as f:
            json.dump(res, f, indent=1)
    mlp.close()
    return res


def load_pretrained(path: str = PRETRAINED) -> api.Mlp:
    """The committed network (FP32 master parameters of csrc/mlp.cuh)."""
    mlp = api.Mlp(seed=0)
    mlp.params = np.load(path)
    return mlp


def evaluate(inp, mlp: api.Mlp, inner: int, tol_per_ion: float, learned_steps: int, plain_steps: int,
             verify_steps: int, precision: int = 1, gemm: int = 3, refine_per_ion: float = 1e-8,
             e_ref: float = None) -> dict:
    """Steps and wall time to tol_per_ion (Ha per ion) of the learned
    mixed-precision path and of plain FP64 SD on one cell.

    SD with fixed occupations can end near a metastable stationary point
    (plain SD continued from it barely moves), and different paths can end in
    different ones.  So the reference energy is the lowest energy any run
    reaches: the learned run, plain FP64 SD continued for verify_steps from
    its end state, and plain FP64 SD run for its whole budget from the
    initial state.  Each path's time to tolerance is measured against it, and
    the learned end state's distance from it is reported.  e_ref adds an
    energy reached elsewhere (an earlier, longer plain run of the same cell)
    to that minimum; plain_steps = 0 then skips the plain run."""
    nion = inp.nion
    tol = tol_per_ion * nion
    lrn = run(inp, None, tol_per_ion, learned_steps, inner, mlp=mlp, precision=precision, gemm=gemm,
              refine_per_ion=refine_per_ion, keep_state=True)
    ver = run(inp, None, tol_per_ion, verify_steps, inner, start_c2=lrn.final_c2)
    plain = run(inp, None, tol_per_ion, plain_steps, inner) if plain_steps > 0 else None
    e_best = min(min(lrn.energies), min(ver.energies))
    if plain is not None:
        e_best = min(e_best, min(plain.energies))
    if e_ref is not None:
        e_best = min(e_best, e_ref)
    ls, lt = first_within(lrn, e_best, tol, inner)
    ps, pt = first_within(plain, e_best, tol, inner) if plain is not None else (None, None)
    out = {"nion": nion, "nbands": int(inp.nbands), "npw": int(inp.npw), "nfft": int(inp.nfft),
           "tol_per_ion": tol_per_ion, "e_best": e_best,
           "learned_end_minus_best_per_ion": (lrn.energies[-1] - e_best) / nion,
           "verify_drift_per_ion": abs(ver.energies[-1] - lrn.energies[-1]) / nion,
           "verify_steps": verify_steps,
           "learned": {"steps_to_tol": ls, "seconds_to_tol": lt, "steps_run": lrn.steps,
                       "seconds_run": lrn.seconds[-1], "rejected_blocks": lrn.rejected_blocks,
                       "fp64_refinement_from_step": lrn.refine_step, "final_energy": lrn.energies[-1],
                       "precision": "mixed" if precision else "fp64", "gemm": gemm},
           "plain_fp64": None if plain is None else
           {"steps_to_tol": ps, "seconds_to_tol": pt, "steps_run": plain.steps,
            "seconds_run": plain.seconds[-1], "final_energy": plain.energies[-1]},
           "e_ref": e_ref}
    if plain is None:
        return out
    if ps and ls:
        out["speedup_time"] = pt / lt
        out["speedup_steps"] = ps / ls
    elif ls:
        # plain SD did not get there within its budget: a lower bound
        out["speedup_time_lower_bound"] = plain.seconds[-1] / lt
        out["speedup_steps_lower_bound"] = plain.steps / ls
    return out


def plain_to_convergence(inp, max_steps: int, inner: int = 200, tol: float = 1e-10,
                         start_c2: Optional[np.ndarray] = None) -> dict:
    """Plain FP64 SD until the energy changes by less than `tol` over each of
    five consecutive blocks of `inner` steps: the converged energy E_conv
    (the reference's own test, main.c:435, watches deltae the same way).
    Returns E_conv, the steps taken (None if max_steps ran out) and the
    energy and wall time after every block."""
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    if start_c2 is not None:
        cell.set_packed(start_c2)
    energies, seconds = [], []
    prev, steps, quiet, conv = math.inf, 0, 0, None
    t0 = time.perf_counter()
    while steps < max_steps:
        e = float(cell.run(inner)[0])
        steps += inner
        energies.append(e)
        seconds.append(time.perf_counter() - t0)
        quiet = quiet + 1 if abs(e - prev) < tol else 0
        prev = e
        if quiet >= 5:
            conv = steps
            break
    cell.close()
    return {"e_conv": energies[-1], "conv_step": conv, "energies": energies, "seconds": seconds, "inner": inner}


def study_cell(inp, mlp: api.Mlp, tol_per_ion: float = 1e-6, plain_max: int = 600000, learned_max: int = 60000,
               inner: int = 100, alt_start_seed: Optional[int] = None, verify_steps: int = 5000,
               precision: int = 1, gemm: int = 3) -> dict:
    """The learned path against plain SD on one cell, with plain SD's own
    converged energy as the yardstick:

    * plain FP64 SD from the cell's start orbitals to convergence -> E_conv,
      and its time to |E - E_conv| <= tol_per_ion * nion;
    * the learned mixed-precision path (FP64 refinement at the end, plain SD
      as the fallback) from the same start until it is within the tolerance
      of E_conv, or learned_max steps; plain FP64 SD continued from its end
      state for verify_steps (a drift near zero: the end state is stationary
      for plain SD);
    * with alt_start_seed, plain SD from other seeded orbitals to convergence:
      a different E_conv there shows that the cell's fixed-occupation energy
      has several stationary points, and which one SD ends in depends on
      the path."""
    nion = inp.nion
    tol = tol_per_ion * nion
    pl = plain_to_convergence(inp, plain_max)
    e_conv = pl["e_conv"]
    p_steps, p_s = None, None
    for k, e in enumerate(pl["energies"]):
        if abs(e - e_conv) <= tol:
            p_steps, p_s = (k + 1) * pl["inner"], pl["seconds"][k]
            break
    lr = run(inp, e_conv, tol_per_ion, learned_max, inner, mlp=mlp, precision=precision, gemm=gemm,
             refine_per_ion=1e-8, keep_state=True)
    ver = run(inp, None, tol_per_ion, verify_steps, inner, start_c2=lr.final_c2)
    out = {"nion": nion, "nbands": int(inp.nbands), "nfft": int(inp.nfft), "tol_per_ion": tol_per_ion,
           "plain": {"e_conv": e_conv, "conv_step": pl["conv_step"], "steps_to_tol": p_steps, "seconds_to_tol": p_s,
                     "seconds_run": pl["seconds"][-1]},
           "learned": {"steps_to_tol": lr.steps_to_tol, "seconds_to_tol": lr.seconds_to_tol, "steps_run": lr.steps,
                       "final_energy": lr.energies[-1], "rejected_blocks": lr.rejected_blocks,
                       "precision": "mixed" if precision else "fp64", "gemm": gemm,
                       "fp64_refinement_from_step": lr.refine_step,
                       "final_minus_e_conv_per_ion": (lr.energies[-1] - e_conv) / nion,
                       "plain_continuation_drift_per_ion": abs(ver.energies[-1] - lr.energies[-1]) / nion}}
    if p_s and lr.seconds_to_tol:
        out["speedup_time"] = p_s / lr.seconds_to_tol
        out["speedup_steps"] = p_steps / lr.steps_to_tol
    if alt_start_seed is not None:
        alt = inputs.random_orbitals(inp.nfft, inp.masker1, inp.nbands, alt_start_seed)
        cell = api.GpuCell(inp)
        pts = cell.sphere()[0]
        cell.close()
        c = alt.reshape(inp.nbands, inp.nfft3d, 2)[:, pts, :]
        start = np.ascontiguousarray(c[..., 0] + 1j * c[..., 1])
        pa = plain_to_convergence(inp, plain_max, start_c2=start)
        out["plain_other_start"] = {"seed": alt_start_seed, "e_conv": pa["e_conv"], "conv_step": pa["conv_step"],
                                    "minus_e_conv_per_ion": (pa["e_conv"] - e_conv) / nion}
    return out


def headline(n8: int = 6, n64: int = 2, traj8: int = 12000, traj64: int = 4000, inner: int = 100,
             train_steps: int = 3000, eval8: int = 2, eval64: int = 1, tol_per_ion: float = 1e-6,
             learned_steps8: int = 40000, plain_steps8: int = 250000, learned_steps64: int = 30000,
             plain_steps64: int = 80000, verify_steps: int = 5000, out: Optional[str] = None,
             weights: Optional[str] = None) -> dict:
    """Train on trajectories of jittered 8- and 64-atom cells, then time the
    learned mixed-precision path against plain FP64 SD on held-out cells."""
    import json
    from . import configs
    t0 = time.perf_counter()
    trajs = [record_trajectory(configs.diamond8_64(seed=1000 + i), traj8, inner, 10) for i in range(n8)]
    trajs += [record_trajectory(configs.diamond64_128(seed=2000 + i), traj64, inner, 5) for i in range(n64)]
    t_traj = time.perf_counter() - t0
    X, T = dataset(trajs)
    mlp = api.Mlp(seed=0)
    t0 = time.perf_counter()
    losses = train(mlp, X, T, steps=train_steps)
    t_train = time.perf_counter() - t0
    if weights:
        np.save(weights, mlp.params)
    res = {"train": {"cells_8atom": n8, "cells_64atom": n64, "trajectory_steps": [traj8, traj64],
                     "samples": int(X.shape[0]), "trajectory_seconds": t_traj, "train_steps": train_steps,
                     "train_seconds": t_train, "loss_first": float(losses[0]),
                     "loss_last": float(np.mean(losses[-50:]))},
           "eval": []}
    for i in range(eval8):
        inp = inputs.build_inputs(configs.diamond8_64(seed=5000 + i))
        r = evaluate(inp, mlp, inner, tol_per_ion, learned_steps8, plain_steps8, verify_steps)
        r["cell"] = "diamond8_64 seed %d" % (5000 + i)
        res["eval"].append(r)
    for i in range(eval64):
        inp = inputs.build_inputs(configs.diamond64_128(seed=6000 + i))
        r = evaluate(inp, mlp, inner, tol_per_ion, learned_steps64, plain_steps64, verify_steps)
        r["cell"] = "diamond64_128 seed %d" % (6000 + i)
        res["eval"].append(r)
    if out:
        with open(out, "w") as f:
            json.dump(res, f, indent=1)
    mlp.close()
    return res


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=12)
    ap.add_argument("--eval", type=int, default=4)
    ap.add_argument("--traj-steps", type=int, default=30000)
    ap.add_argument("--inner", type=int, default=100)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--max-steps", type=int, default=120000)
    ap.add_argument("--out", default=None)
    ap.add_argument("--weights", default=None)
    ap.add_argument("--horizon", type=int, default=32)
    ap.add_argument("--headline", action="store_true",
                    help="8- and 64-atom training, timed learned mixed path vs plain FP64")
    ap.add_argument("--evaluate", default=None, help="time one cell (a configs name) with the committed network")
    ap.add_argument("--seed", type=int, default=6000)
    ap.add_argument("--learned-steps", type=int, default=30000)
    ap.add_argument("--plain-steps", type=int, default=200000)
    ap.add_argument("--verify-steps", type=int, default=5000)
    ap.add_argument("--e-ref", type=float, default=None,
                    help="an energy of the same cell reached by another run (joins the reference minimum)")
    ap.add_argument("--study", default=None,
                    help="study_cell on held-out cells of a configs name (comma-separated seeds in --seeds)")
    ap.add_argument("--seeds", default="5000,5001")
    ap.add_argument("--plain-max", type=int, default=600000)
    ap.add_argument("--fp64", action="store_true", help="study: the learned path in FP64 (no mixed precision)")
    a = ap.parse_args()
    if a.study:
        from . import configs
        mlp = load_pretrained()
        res = {}
        for sd in (int(x) for x in a.seeds.split(",")):
            r = study_cell(inputs.build_inputs(configs.NAMED[a.study](seed=sd)), mlp, plain_max=a.plain_max,
                           learned_max=a.learned_steps, alt_start_seed=sd + 77,
                           precision=0 if a.fp64 else 1, gemm=0 if a.fp64 else 3)
            res["%s seed %d" % (a.study, sd)] = r
            print(json.dumps({"cell": "%s seed %d" % (a.study, sd), **r}), flush=True)
            if a.out:
                with open(a.out, "w") as f:
                    json.dump(res, f, indent=1)
        mlp.close()
        raise SystemExit(0)
    if a.headline:
        print(json.dumps(headline(out=a.out, weights=a.weights), indent=1))
        raise SystemExit(0)
    if a.evaluate:
        from . import configs
        mlp = load_pretrained()
        res = evaluate(inputs.build_inputs(configs.NAMED[a.evaluate](seed=a.seed)), mlp, a.inner, 1e-6,
                       a.learned_steps, a.plain_steps, a.verify_steps, e_ref=a.e_ref)
        res["cell"] = "%s seed %d" % (a.evaluate, a.seed)
        mlp.close()
        if a.out:
            with open(a.out, "w") as f:
                json.dump(res, f, indent=1)
        print(json.dumps(res, indent=1))
        raise SystemExit(0)
    r = experiment(a.train, a.eval, a.traj_steps, a.inner, 10, a.train_steps, 1e-6, a.max_steps, a.out, a.weights,
                   a.horizon)
    print(json.dumps(r, indent=1))
