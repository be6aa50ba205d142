"""Learned denoiser on the tensor cores (needs a B200): the tcgen05 BF16 GEMM
building block against a float64 product of the same BF16 operands."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (300, 16, 144), (256, 128, 256), (128, 48, 96)])
def test_tc_gemm_matches_fp64(rg, M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((N, K)).astype(np.float32)
    got = rg.tc_gemm_bf16(A, B)
    a = rg.from_bf16_bits(rg.to_bf16_bits(A)).astype(np.float64)
    b = rg.from_bf16_bits(rg.to_bf16_bits(B)).astype(np.float64)
    ref = a @ b.T
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-4 * np.sqrt(K))
