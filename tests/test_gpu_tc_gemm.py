"""The tcgen05 tensor-core GEMM (tbpm_nn_gemm_tn) of the learned tail.

C = alpha * A . B^T + beta * C with BF16 inputs and FP32 accumulation is
checked against a float64 numpy product of the same BF16 values (relative
1e-5, the level of FP32 accumulation) and against the mma.sync GEMM; shapes
cover single and many tiles, ragged edges in M, N and K (zero-filled TMA
boxes), K shorter than one 64-wide stage and longer than the 4-stage ring.
"""

import numpy as np
import pytest

from tbplas_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _bf16_exact(rng, shape):
    torch = _torch()
    x = rng.standard_normal(shape).astype(np.float32)
    return torch.tensor(x).to(torch.bfloat16).float().numpy().astype(np.float64)


def _status(lib):
    import ctypes
    f = ctypes.c_int(-1)
    assert lib.tbpm_nn_tc_status(ctypes.byref(f)) == 0
    return f.value


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (1, 8, 8), (257, 300, 96), (130, 129, 520),
                                   (576, 3584, 1280), (64, 256, 16)])
def test_tc_gemm_matches_numpy_and_mma(M, N, K):
    torch = _torch()
    lib = nat.load_library()
    rng = np.random.default_rng(M * 7 + N + K)
    a = _bf16_exact(rng, (M, K))
    b = _bf16_exact(rng, (N, K))
    c0 = rng.standard_normal((M, N)).astype(np.float32)
    A = torch.tensor(a, device="cuda").to(torch.bfloat16)
    B = torch.tensor(b, device="cuda").to(torch.bfloat16)
    s = torch.cuda.current_stream().cuda_stream
    ref = 0.5 * (a @ b.T) + 2.0 * c0
    C = torch.tensor(c0, device="cuda")
    assert lib.tbpm_nn_gemm_tn(A.data_ptr(), K, B.data_ptr(), K, C.data_ptr(), N, M, N, K,
                                  0.5, 2.0, s) == 0
    got = C.cpu().numpy()
    assert _status(lib) == 0
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-5
    C2 = torch.tensor(c0, device="cuda")
    assert lib.tbpm_nn_gemm_tn_mma(A.data_ptr(), K, B.data_ptr(), K, C2.data_ptr(), N, M, N, K,
                               0.5, 2.0, s) == 0
    assert np.max(np.abs(got - C2.cpu().numpy())) / np.max(np.abs(ref)) < 1e-5
    # beta = 0 overwrites C (which may hold garbage)
    C3 = torch.full((M, N), float("nan"), device="cuda")
    assert lib.tbpm_nn_gemm_tn(A.data_ptr(), K, B.data_ptr(), K, C3.data_ptr(), N, M, N, K,
                                  1.0, 0.0, s) == 0
    assert np.max(np.abs(C3.cpu().numpy() - a @ b.T)) / np.max(np.abs(a @ b.T)) < 1e-5


def test_tc_gemm_strided_operands_and_rejections():
    torch = _torch()
    lib = nat.load_library()
    rng = np.random.default_rng(5)
    M, N, K, lda, ldb, ldc = 200, 150, 72, 80, 96, 160
    a = _bf16_exact(rng, (M, lda))
    b = _bf16_exact(rng, (N, ldb))
    A = torch.tensor(a, device="cuda").to(torch.bfloat16)
    B = torch.tensor(b, device="cuda").to(torch.bfloat16)
    C = torch.zeros((M, ldc), dtype=torch.float32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert lib.tbpm_nn_gemm_tn(A.data_ptr(), lda, B.data_ptr(), ldb, C.data_ptr(), ldc, M, N,
                                  K, 1.0, 0.0, s) == 0
    ref = a[:, :K] @ b[:, :K].T
    got = C.cpu().numpy()
    assert np.max(np.abs(got[:, :N] - ref)) / np.max(np.abs(ref)) < 1e-5
    assert np.all(got[:, N:] == 0)  # columns beyond N untouched
    assert lib.tbpm_nn_gemm_tn(A.data_ptr(), 12, B.data_ptr(), 12, C.data_ptr(), 16, 16, 16,
                                  12, 1.0, 0.0, s) == nat.TBPM_ERR_ARG
    assert lib.tbpm_nn_gemm_tn(A.data_ptr() + 2, lda, B.data_ptr(), ldb, C.data_ptr(), ldc,
                                  8, 8, 8, 1.0, 0.0, s) == nat.TBPM_ERR_ARG
