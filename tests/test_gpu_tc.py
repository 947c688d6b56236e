"""GPU tests of the weighted TN products: the FP64 engine and the 3xTF32
tcgen05 engine of cpsd_overlap_tn against numpy, and the mixed-precision
step with tensor-core overlaps against the FP64 oracle."""
import numpy as np
import pytest

from cpsd_b200 import api, configs, inputs, lib

import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

# 3xTF32 keeps about FP32 accuracy: bound |dC| by this times the
# Cauchy-Schwarz scale max_i |w A_i| max_j |B_j|
TF32X3_TOL = 2e-6


def _case(M, N, K, seed, weighted=True):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(M, K))
    B = rng.normal(size=(N, K))
    w = rng.uniform(0.5, 2.0, size=(K + 1) // 2) if weighted else None
    wk = np.repeat(w, 2)[:K] if weighted else np.ones(K)
    ref = (A * wk) @ B.T
    scale = np.linalg.norm(A * wk, axis=1).max() * np.linalg.norm(B, axis=1).max()
    dev = lambda x: None if x is None else torch.from_numpy(x).cuda()
    return dev(A), dev(B), dev(w), ref, scale


@pytest.mark.parametrize("M,N,K", [(16, 16, 4966), (40, 40, 6002), (128, 128, 38138), (200, 72, 9000),
                                   (256, 128, 4966), (5, 3, 64), (130, 1, 130)])
def test_overlap_fp64_matches_numpy(M, N, K):
    A, B, w, ref, scale = _case(M, N, K, seed=M + N + K)
    C = api.overlap_tn(A, B, w, lib.CPSD_GEMM_FP64).cpu().numpy()
    assert np.abs(C - ref).max() <= 1e-13 * scale


@pytest.mark.parametrize("M,N,K", [(16, 16, 4966), (40, 40, 6002), (128, 128, 38138), (200, 72, 9000),
                                   (256, 128, 4966), (5, 3, 64), (130, 1, 130), (129, 129, 33)])
def test_overlap_tf32x3_matches_numpy(M, N, K):
    A, B, w, ref, scale = _case(M, N, K, seed=7 * M + N + K)
    C = api.overlap_tn(A, B, w, lib.CPSD_GEMM_TF32X3).cpu().numpy()
    assert np.abs(C - ref).max() <= TF32X3_TOL * scale, np.abs(C - ref).max() / scale


def test_overlap_unweighted_and_reproducible():
    A, B, _, ref, scale = _case(96, 64, 20000, seed=3, weighted=False)
    C1 = api.overlap_tn(A, B, None, lib.CPSD_GEMM_TF32X3).cpu().numpy()
    C2 = api.overlap_tn(A, B, None, lib.CPSD_GEMM_TF32X3).cpu().numpy()
    assert np.array_equal(C1, C2)  # fixed split plan and reduction order
    assert np.abs(C1 - ref).max() <= TF32X3_TOL * scale


def test_overlap_rejects_bad_arguments():
    A, B, w, _, _ = _case(8, 8, 64, seed=1)
    L = lib.load()
    C = torch.empty((8, 8), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert L.cpsd_overlap_tn(7, 8, 8, 64, A.data_ptr(), 64, B.data_ptr(), 64, w.data_ptr(), C.data_ptr(), 8,
                             s) == lib.CPSD_ERR_ARG
    assert L.cpsd_overlap_tn(0, 8, 8, 64, A.data_ptr(), 32, B.data_ptr(), 64, w.data_ptr(), C.data_ptr(), 8,
                             s) == lib.CPSD_ERR_ARG


def _mixed_track(restatement, mode, rel):
    inp = inputs.build_inputs(configs.small_diamond(32, 5, ecut=25.0))
    so = oracle.State(inp)
    cell = api.GpuCell(inp, precision=lib.CPSD_PREC_MIXED)
    cell.set_gemm(mode)
    cell.set_state(inp.c2, inp.r2)
    for _ in range(3):
        restatement.run(inp, 2, so)
        cell.run(2)
        assert abs(cell.E[0] - so.E[0]) < rel * abs(so.E[0]) + 1e-6
    return inp, cell


def test_mixed_step_with_tensor_core_projectors(restatement):
    """3xTF32 projector coefficients: energies follow the FP64 oracle as
    closely as the FP32 transforms alone do (1e-6 relative)."""
    _, cell = _mixed_track(restatement, lib.CPSD_GEMM_TF32X3, 1e-6)
    cell.close()


def test_mixed_step_with_tensor_core_overlaps(restatement):
    """3xTF32 overlaps too: the Lagrange solve's division by dte costs about
    1e-6 relative per step (bar 1e-5); an FP64 step from the same state
    gives the FP64 energy of that state (1e-9 Ha against the oracle)."""
    inp, cell = _mixed_track(restatement, lib.CPSD_GEMM_TF32X3_OVERLAPS, 1e-5)
    st = api.State(inp)
    cell.get_state(st)
    cell.set_precision(lib.CPSD_PREC_FP64)
    cell.E[0] = 0.0
    cell.run(1)
    probe = oracle.State(inp)
    probe.c2[:] = st.c2
    restatement.run(inp, 1, probe)
    assert abs(cell.E[0] - probe.E[0]) < 1e-9
    cell.close()


def test_tf32x3_needs_a_mixed_context():
    inp = inputs.build_inputs(configs.small_diamond(24, 4, ecut=16.0))
    cell = api.GpuCell(inp)
    with pytest.raises(lib.CpsdError):
        cell.set_gemm(lib.CPSD_GEMM_TF32X3)
    cell.close()


def test_fused_overlaps_at_128_bands():
    """The fused three-overlap tcgen05 pass (128 bands, 128^3) against the
    same mixed-precision steps with FP64 overlaps."""
    inp = inputs.build_inputs(configs.diamond64_128())
    E = []
    for mode in (lib.CPSD_GEMM_TF32X3, lib.CPSD_GEMM_TF32X3_OVERLAPS):
        cell = api.GpuCell(inp, precision=lib.CPSD_PREC_MIXED)
        cell.set_gemm(mode)
        cell.set_state(inp.c2, inp.r2)
        E.append([float(cell.run(2)[0]) for _ in range(2)])
        cell.close()
    for a, b in zip(*E):
        assert abs(a - b) < 1e-5 * abs(a), (a, b)
