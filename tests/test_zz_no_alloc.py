"""The allocation-free GEMM entry point (gg_zgemm_noalloc).

Some callers may not allocate device memory at the point where they need a contraction:
services whose device memory is owned by another allocator or fixed at start-up, and
latency-bound loops where cudaMalloc's implicit synchronisation would stall other streams.
gg_zgemm_noalloc serves them with caller-owned device buffers for A, B and C and a static
device scratch array for its split-K partial sums.  These tests call it through the C ABI
twice in a row and compare it with the allocating gg_zgemm entry point and with A @ B in
numpy (1e-13 of the largest element); they run last (file name) and also pass alone.
"""
import ctypes

import numpy as np
import pytest

from green_gpu_b200 import native

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, np.complex128).view(np.float64)).cuda()
    return t


def _noalloc(lib, A, B):
    import torch
    M, K = A.shape
    N = B.shape[1]
    a, b = _dev(A), _dev(B)
    c = torch.empty((M, N * 2), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = lib.gg_zgemm_noalloc(M, N, K, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                              ctypes.c_void_p(c.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == native.GG_OK, lib.gg_last_error(None).decode()
    stream.synchronize()
    return c.cpu().numpy().view(np.complex128)


def test_noalloc_gemm_matches_allocating_entry_point_twice():
    lib = native.load()
    ctx = native.Context(2, 2, 2, 2, 4, 1, 4, 3)
    rng = np.random.default_rng(21)
    # shapes whose tile grid under-fills the GPU, so split-K (and the static scratch) is used
    for (M, N, K) in ((64, 64, 4096), (100, 70, 3000)):
        A = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
        B = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
        got = _noalloc(lib, A, B)
        want = ctx.zgemm(A, B, precision=native.PREC_FP64)
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
        ref = A @ B
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    ctx.close()


def test_noalloc_rejects_sizes_beyond_the_scratch():
    lib = native.load()
    rc = lib.gg_zgemm_noalloc(1024, 1024, 8, ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == native.GG_ERR_ARG
    assert b"exceeds the limit" in lib.gg_last_error(None)
