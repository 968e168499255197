"""Tensor-core pieces of the learned warm start against plain PyTorch FP32."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even FP32 -> BF16 bit patterns."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def _bf16_value(bits: np.ndarray) -> np.ndarray:
    return (bits.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (256, 64, 128), (384, 128, 64), (128, 128, 8192)])
def test_gemm_bf16_matches_fp32(M, N, K):
    import torch
    from tapsim_modified_b200 import _native as N_
    rng = np.random.default_rng(M + N + K)
    a = _bf16_bits(rng.standard_normal((M, K)).astype(np.float32))
    b = _bf16_bits(rng.standard_normal((N, K)).astype(np.float32))
    c = np.empty((M, N), np.float32)
    N_.check(N_.lib().tg_gemm_bf16(N_.ptr(a), N_.ptr(b), N_.ptr(c), M, N, K))
    ref = (torch.from_numpy(_bf16_value(a)).double() @ torch.from_numpy(_bf16_value(b)).double().T).numpy()
    # FP32 accumulation of K products of magnitude ~1
    assert np.abs(c - ref).max() <= 1e-5 * K


def test_gemm_rejects_bad_shapes():
    from tapsim_modified_b200 import _native as N_
    a = np.zeros(128 * 64, np.uint16)
    c = np.zeros(128 * 64, np.float32)
    assert N_.lib().tg_gemm_bf16(N_.ptr(a), N_.ptr(a), N_.ptr(c), 100, 64, 64) == 1
    assert N_.lib().tg_gemm_bf16(N_.ptr(a), N_.ptr(a), N_.ptr(c), 128, 32, 64) == 1
