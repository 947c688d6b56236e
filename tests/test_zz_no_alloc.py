"""GPU test of cpsd_overlap_tn_noalloc, the entry point that allocates no
device memory (for host codes that hand the whole GPU to their own memory
pool, or that must not let cudaMalloc/cudaFree synchronise the device):
through the C ABI, two calls in a row, each against cpsd_overlap_tn (the
allocating entry point) and a float64 numpy product on the same inputs; the
device's free memory unchanged across calls; the largest accepted size and
the refusal beyond it.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from cpsd_b200 import lib

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

FP64_TOL = 1e-13    # as tests/test_gpu_tc.py, times the Cauchy-Schwarz scale
TF32X3_TOL = 2e-6


def _host_inputs(M, N, K, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(M, K))
    B = rng.normal(size=(N, K))
    w = rng.uniform(0.5, 2.0, size=(K + 1) // 2)
    wk = np.repeat(w, 2)[:K]
    scale = np.linalg.norm(A * wk, axis=1).max() * np.linalg.norm(B, axis=1).max()
    return A, B, w, wk, scale


def _inputs(M, N, K, seed):
    A, B, w, _, scale = _host_inputs(M, N, K, seed)
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
        A_h, B_h, w_h, wk, scale = _host_inputs(M, N, K, seed)
        A, B, w = (torch.from_numpy(x).cuda() for x in (A_h, B_h, w_h))
        C_ref = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
        C = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
        assert _call(L.cpsd_overlap_tn, method, A, B, w, C_ref) == lib.CPSD_OK
        assert _call(L.cpsd_overlap_tn_noalloc, method, A, B, w, C) == lib.CPSD_OK
        d = (C - C_ref).abs().max().item()
        assert d <= tol * scale, (M, N, K, d / scale)
        # and directly against the float64 product on the host
        d_np = np.abs(C.cpu().numpy() - (A_h * wk) @ B_h.T).max()
        assert d_np <= tol * scale, (M, N, K, d_np / scale)


def test_noalloc_leaves_device_memory_unchanged():
    """After a first call (the per-device set-up), further calls take no
    device memory: the driver's free-memory count does not move."""
    L = lib.load()
    A, B, w, scale = _inputs(96, 64, 20000, 4)
    C = torch.zeros((96, 64), dtype=torch.float64, device="cuda")
    assert _call(L.cpsd_overlap_tn_noalloc, 0, A, B, w, C) == lib.CPSD_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for method in (0, 1, 0):
        assert _call(L.cpsd_overlap_tn_noalloc, method, A, B, w, C) == lib.CPSD_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_accepts_the_largest_size():
    """M = N = 1023 (M*N = 1,046,529 <= the limit): one split fits the scratch."""
    L = lib.load()
    M = N = 1023
    A_h, B_h, w_h, wk, scale = _host_inputs(M, N, 96, 5)
    A, B, w = (torch.from_numpy(x).cuda() for x in (A_h, B_h, w_h))
    C = torch.full((M, N), np.nan, dtype=torch.float64, device="cuda")
    assert _call(L.cpsd_overlap_tn_noalloc, 0, A, B, w, C) == lib.CPSD_OK
    assert np.abs(C.cpu().numpy() - (A_h * wk) @ B_h.T).max() <= FP64_TOL * scale


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
