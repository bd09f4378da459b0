"""The tensor-core product of the learned stage's dense layers (tcgen05.mma,
BF16 operands, FP32 accumulation in tensor memory) against numpy on the same
BF16-rounded operands in FP64: tile-aligned, ragged and the layers' own
shapes.  Bar: 1e-5 of sum_k |a_k b_k| per entry (FP32 accumulation)."""
import numpy as np
import pytest

import openfea_b200 as ob
from oracle.gnn_oracle import bf16

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M, N, K", [(128, 64, 64), (200, 70, 100), (4000, 64, 320), (320, 64, 4000),
                                     (33, 6, 8), (1, 1, 1)])
def test_tc_matmul_matches_bf16_reference(gpu_ctx_factory, M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A = rng.normal(size=(M, K)).astype(np.float32)
    B = rng.normal(size=(N, K)).astype(np.float32)
    D = ob.tc_matmul(A, B)
    Ab, Bb = bf16(A), bf16(B)
    ref = Ab @ Bb.T
    scale = np.abs(Ab) @ np.abs(Bb).T
    assert np.all(np.abs(D - ref) <= 1e-5 * scale + 1e-30), np.abs(D - ref).max()
    # deterministic
    assert np.array_equal(D, ob.tc_matmul(A, B))
