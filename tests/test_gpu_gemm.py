"""The estimator's tcgen05 BF16 GEMM against an fp32 reference of the same
bf16-rounded operands.  Tolerance: |C - C_ref| <= 1e-3 * (sum_k |a_mk b_nk|)
+ 1e-6 per element (fp32 accumulation in a different order)."""
import numpy as np
import pytest

import asdmatch_b200 as A

pytestmark = pytest.mark.gpu


def _check(a, b):
    got = A.gemm_bf16(a, b)
    ar, br = A.from_bf16_bits(A.to_bf16_bits(a)).reshape(a.shape), A.from_bf16_bits(A.to_bf16_bits(b)).reshape(b.shape)
    want = ar.astype(np.float64) @ br.astype(np.float64).T
    scale = np.abs(ar).astype(np.float64) @ np.abs(br).astype(np.float64).T
    assert np.all(np.abs(got - want) <= 1e-3 * scale + 1e-6), np.max(np.abs(got - want))


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (128, 128, 16), (300, 200, 200), (1, 1, 1), (513, 128, 256),
                                   (128, 256, 1000)])
def test_gemm_matches_fp32_reference(M, N, K):
    rng = np.random.default_rng(M * 7 + N + K)
    _check(rng.standard_normal((M, K)).astype(np.float32), rng.standard_normal((N, K)).astype(np.float32))


def test_gemm_places_every_element():
    # identity x B picks rows of B exactly (every product is exact in fp32)
    K = 128
    eye = np.eye(K, dtype=np.float32)
    b = np.arange(128 * K, dtype=np.float32).reshape(128, K) % 97
    got = A.gemm_bf16(eye, b)
    assert np.array_equal(got, b.T)
