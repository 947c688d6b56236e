"""GPU test of cpsd_overlap_tn_noalloc, the entry point that allocates no
device memory: through the C ABI, two calls in a row, each against
cpsd_overlap_tn (the allocating entry point) on the same inputs, and the
size limit of its static scratch.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from cpsd_b200 import lib

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

FP64_TOL = 1e-13    # as tests/test_gpu_tc.py, times the Cauchy-Schwarz scale
TF32X3_TOL = 2e-6


def _inputs(M, N, K, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(M, K))
    B = rng.normal(size=(N, K))
    w = rng.uniform(0.5, 2.0, size=(K + 1) // 2)
    wk = np.repeat(w, 2)[:K]
    scale = np.linalg.norm(A * wk, axis=1).max() * np.linalg.norm(B, axis=1).max()
    return torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), torch.from_numpy(w).cuda(), scale


def _call(fn, method, A, B, w, C):
    M, K = A.shape
    N = B.shape[0]
    s = torch.cuda.current_stream().cuda_stream
    return fn(method, M, N, K, A.data_ptr(), K, B.data_ptr(), K, w.data_ptr(), C.data_ptr(), N, s)


@pytest.mark.parametrize("method,tol", [(0, FP64_TOL), (1, TF32X3_TOL)])
def test_noalloc_matches_allocating_entry_point(method, tol):
    L = lib.load()
    for M, N, K, seed in ((128, 128, 38138, 1), (40, 72, 6002, 2)):  # two calls in a row
        A, B, w, scale = _inputs(M, N, K, seed)
        C_ref = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
        C = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
        assert _call(L.cpsd_overlap_tn, method, A, B, w, C_ref) == lib.CPSD_OK
        assert _call(L.cpsd_overlap_tn_noalloc, method, A, B, w, C) == lib.CPSD_OK
        d = (C - C_ref).abs().max().item()
        assert d <= tol * scale, (M, N, K, d / scale)


# CPSD_NOALLOC_MAX_DOUBLES of include/cpsd_b200.h: room for split-K partials
NOALLOC_MAX_DOUBLES = (1 << 20) - 32


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = lib.load()
    M = N = 1024  # a single split needs M*N = 1,048,576 > NOALLOC_MAX_DOUBLES
    assert M * N > NOALLOC_MAX_DOUBLES
    A, B, w, _ = _inputs(M, N, 64, 3)
    C = torch.zeros((M, N), dtype=torch.float64, device="cuda")
    assert _call(L.cpsd_overlap_tn_noalloc, 0, A, B, w, C) == lib.CPSD_ERR_SCRATCH
    assert float(C.abs().max()) == 0.0  # nothing was launched
