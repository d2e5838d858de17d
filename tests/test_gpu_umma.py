"""tcgen05 tensor-core GEMM building block (kind::tf32, 3xTF32 split) against a
host FP64 matmul: the operand layout / descriptor encoding must reproduce A B^T
to FP32 accuracy (3xTF32) and TF32 accuracy (1x)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(16, 8), (32, 32), (48, 64), (64, 64), (96, 64)])
def test_umma_tf32_tile(ctx, N, K):
    from gfb200 import _lib as L
    lib = C.CDLL(L.LIB_PATH)
    f = lib.gfx_umma_selftest
    f.argtypes = [C.c_void_p] * 3 + [C.c_int] * 3
    rng = np.random.default_rng(N + K)
    A = rng.standard_normal((128, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    for split, tol in ((1, 2e-6), (0, 2e-3)):
        D = np.zeros((128, N), np.float32)
        assert f(A.ctypes.data, B.ctypes.data, D.ctypes.data, N, K, split) == 0
        assert np.abs(D - ref).max() / np.abs(ref).max() < tol
