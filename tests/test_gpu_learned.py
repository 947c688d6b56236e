"""GPU tests of the learned preconditioner: the network's forward and backward
kernels against the numpy oracle (gradient check), training on the GPU, and
guarded use in SD (same converged energy as plain SD)."""
import math

import numpy as np
import pytest

from cpsd_b200 import api, configs, inputs, learned

import mlp_oracle

pytestmark = pytest.mark.gpu


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    X = np.stack([rng.uniform(0, 8, n), rng.normal(0, 1, n), rng.normal(-3, 2, n), rng.uniform(0, 1, n)], 1)
    # a smooth target of the kind the preconditioner learns (a Teter-like roll-off)
    x = X[:, 0]
    T = np.log((27 + 18 * x + 12 * x ** 2 + 8 * x ** 3) / (27 + 18 * x + 12 * x ** 2 + 8 * x ** 3 + 16 * x ** 4)) + 0.1 * X[:, 1]
    return X.astype(np.float32), T.astype(np.float32)


def test_forward_matches_oracle():
    m = api.Mlp(seed=3)
    X, _ = _data(1000)
    y = m.forward(X)
    yo, _ = mlp_oracle.forward(m.params, X)
    assert np.abs(y - yo).max() < 1e-4 * max(1.0, np.abs(yo).max())
    m.close()


def test_gradient_matches_oracle():
    """Backward kernels == analytic gradient of the numpy oracle (FP32 tolerance)."""
    m = api.Mlp(seed=5)
    X, T = _data(3000, seed=1)
    loss, g = m.gradient(X, T)
    lo, go = mlp_oracle.loss_and_grad(m.params, X, T)
    assert abs(loss - lo) < 1e-4 * lo
    scale = np.abs(go).max()
    assert np.abs(g - go).max() < 2e-4 * scale
    # and the oracle gradient itself against central finite differences on a few parameters
    p = m.params.astype(np.float64)
    for k in (mlp_oracle.B1 + 3, mlp_oracle.B3 + 7, mlp_oracle.B4):  # biases: not BF16-rounded
        e = 1e-4
        pp, pm = p.copy(), p.copy()
        pp[k] += e
        pm[k] -= e
        fd = (mlp_oracle.loss_and_grad(pp.astype(np.float32), X, T)[0] -
              mlp_oracle.loss_and_grad(pm.astype(np.float32), X, T)[0]) / (2 * e)
        assert abs(fd - go[k]) < 1e-2 * max(abs(go[k]), 1e-3)
    m.close()


def test_gradient_is_bitwise_reproducible():
    m = api.Mlp(seed=9)
    X, T = _data(5000, seed=2)
    g1 = m.gradient(X, T)[1]
    g2 = m.gradient(X, T)[1]
    assert np.array_equal(g1, g2)
    m.close()


def test_training_reduces_loss():
    m = api.Mlp(seed=11)
    X, T = _data(20000, seed=3)
    l0 = m.gradient(X, T)[0]
    losses = learned.train(m, X, T, steps=600, batch=2048, lr=2e-3)
    l1 = m.gradient(X, T)[0]
    assert l1 < 0.1 * l0, (l0, l1, losses[-5:])
    m.close()


def _h2(seed):
    # one band with a gap: plain SD converges to 1e-11 Ha in a few thousand steps
    return configs.small_h2(24, 1, seed=seed)


def test_learned_run_keeps_the_plain_sd_fixed_point():
    """An (untrained) network in the loop with the energy guard converges to
    the same energy as plain SD: only the residual is preconditioned, so the
    fixed point is plain SD's."""
    inp = inputs.build_inputs(_h2(4))
    max_steps = 100000
    e_conv, conv_steps = learned.converged_energy(inp, max_steps=max_steps, inner=200, tol=1e-12)
    assert conv_steps < max_steps
    tol = 1e-8
    plain = learned.run(inp, e_conv, tol, max_steps=max_steps, inner=50)
    assert plain.steps_to_tol is not None
    m = api.Mlp(seed=1)
    r = learned.run(inp, e_conv, tol, max_steps=4 * plain.steps_to_tol + 1000, inner=50, mlp=m)
    assert r.steps_to_tol is not None, (plain.steps_to_tol, r.rejected_blocks, r.energies[-3:], e_conv)
    assert abs(r.energies[-1] - e_conv) <= tol * inp.nion
    m.close()


def test_trained_network_needs_fewer_steps_than_plain_sd():
    """Ablation: trained on plain-SD trajectories from three initial states,
    the network reaches the converged energy (1e-8 Ha per ion) from a held-out
    initial state in fewer SD steps than plain SD, and to the same energy."""
    trajs = [learned.record_trajectory(_h2(20 + i), 4000, 50, 2, horizon=32) for i in range(3)]
    X, T = learned.dataset(trajs)
    m = api.Mlp(seed=0)
    learned.train(m, X, T, steps=1500, batch=2048, lr=2e-3)
    inp = inputs.build_inputs(_h2(99))
    e_conv, conv_steps = learned.converged_energy(inp, max_steps=100000, inner=200, tol=1e-12)
    assert conv_steps < 100000
    plain = learned.run(inp, e_conv, 1e-8, max_steps=100000, inner=50)
    lrn = learned.run(inp, e_conv, 1e-8, max_steps=100000, inner=50, mlp=m)
    assert plain.steps_to_tol is not None and lrn.steps_to_tol is not None
    assert lrn.steps_to_tol < plain.steps_to_tol, (plain.steps_to_tol, lrn.steps_to_tol, lrn.rejected_blocks)
    assert abs(lrn.energies[-1] - e_conv) <= 1e-8 * inp.nion
    m.close()


def test_unit_step_scale_is_plain_sd_bitwise():
    """With the log-K range set to [0, 0] the learned step graph takes plain
    SD steps: same energies, bit for bit, as a cell without a network."""
    inp = inputs.build_inputs(configs.small_diamond(24, 4, ecut=16.0, seed=7))
    plain = api.GpuCell(inp)
    plain.set_state(inp.c2, inp.r2)
    e_plain = [plain.run(10)[0] for _ in range(3)]
    m = api.Mlp(seed=2)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    cell.set_preconditioner(m)
    cell.set_preconditioner_range(0.0, 0.0)
    e_unit = [cell.run(10)[0] for _ in range(3)]
    assert e_unit == e_plain
    plain.close()
    cell.close()
    m.close()


def test_save_and_restore_orbitals_repeat_a_block():
    inp = inputs.build_inputs(configs.small_diamond(24, 4, ecut=16.0, seed=8))
    m = api.Mlp(seed=3)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    cell.set_preconditioner(m)
    cell.run(5)
    cell.save_orbitals()
    e1 = cell.run(10).copy()
    c_after = cell.get_c2()
    cell.restore_orbitals()
    e2 = cell.run(10).copy()
    assert np.array_equal(c_after, cell.get_c2())
    assert e1[0] == e2[0]
    cell.close()
    m.close()


def test_guarded_block_in_the_library_rejects_and_redoes_with_plain_sd():
    """cpsd_gpu_run_guarded: with the previous energy set to -inf every
    learned block counts as a rise, so each is redone from its start with
    plain SD steps -- the energies and orbitals are plain SD's, bit for bit,
    and the trust region shrinks by 0.7 per rejected block."""
    inp = inputs.build_inputs(configs.small_diamond(24, 4, ecut=16.0, seed=7))
    plain = api.GpuCell(inp)
    plain.set_state(inp.c2, inp.r2)
    e_plain = [plain.run(5).copy() for _ in range(2)]
    c_plain = plain.get_c2()
    m = api.Mlp(seed=2)
    cell = api.GpuCell(inp)
    cell.set_state(inp.c2, inp.r2)
    cell.set_preconditioner(m)
    cap = learned.LOGK_MAX
    for k in range(2):
        cell.E[0] = -math.inf
        e, rej, cap = cell.run_guarded(5, cap)
        assert rej == 1
        assert np.array_equal(cell.E[1:], e_plain[k][1:]) and e == e_plain[k][0]
    assert cap == pytest.approx(learned.LOGK_MAX - 2 * learned.CAP_SHRINK)
    assert np.array_equal(cell.get_c2(), c_plain)
    # with the previous energy +inf a block is kept as the network made it
    cell.E[0] = math.inf
    e, rej, cap2 = cell.run_guarded(5, cap)
    assert rej == 0 and math.isfinite(e) and cap2 == pytest.approx(cap + learned.CAP_GROW)
    plain.close()
    cell.close()
    m.close()
