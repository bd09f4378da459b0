"""The residual-norm entry point that allocates no device memory, for callers
that cannot allocate (their own pool allocator owns the GPU, or cudaMalloc's
possible device synchronization is not acceptable).  It must give the norms
that the existing solve entry point reports, call after call.  This file is
collected last so that a run stopping at its first failure has already run
every other test."""
import ctypes

import numpy as np
import pytest

import openfea_b200 as ob
from openfea_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _entry():
    fn = ob.lib().ofea_residual_norms_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def test_residual_norms_without_allocation(gpu_ctx_factory):
    import torch
    m, ffull = mg.cantilever_small()
    ctx = gpu_ctx_factory()
    fm = ctx.upload_mesh(m)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    f0 = mg.to_free(ffull, fm)
    rng = np.random.default_rng(4)
    F = np.stack([f0, 0.5 * f0 + rng.normal(0, 100.0, f0.size), -f0], axis=1)  # n x 3
    U, stats = ctx.solve(F, method="GPU_PCG", rtol=1e-9)
    nrhs = F.shape[1]
    # column-major n x nrhs on the device = row-major (nrhs, n)
    dF = torch.tensor(F.T.copy(), dtype=torch.float64, device="cuda")
    dU = torch.tensor(U.T.copy(), dtype=torch.float64, device="cuda")
    fn = _entry()
    for call in range(2):
        norms = torch.full((2 * nrhs,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = fn(ctx.h, nrhs, dF.data_ptr(), dU.data_ptr(), norms.data_ptr())
        assert rc == 0, ob.lib().ofea_last_error()
        torch.cuda.synchronize()
        # nothing was allocated on the device, on the first call either
        assert torch.cuda.mem_get_info()[0] == free_before, call
        got = norms.cpu().numpy()
        rel = got[0::2] / got[1::2]
        # against the existing entry points: the solve's reported FP64 residual
        # and f - K u from ofea_spmv
        for k in range(nrhs):
            assert abs(rel[k] - stats[k]["rel_residual"]) <= 1e-12 * stats[k]["rel_residual"] + 1e-300, (call, k)
            r = F[:, k] - ctx.spmv(U[:, k])
            assert abs(got[2 * k] - np.linalg.norm(r)) <= 1e-9 * np.linalg.norm(r), (call, k)
            assert abs(got[2 * k + 1] - np.linalg.norm(F[:, k])) <= 1e-12 * np.linalg.norm(F[:, k]), (call, k)


def test_residual_norms_without_allocation_rejects_too_many_cases(gpu_ctx_factory):
    import torch
    m, _ = mg.cantilever_small()
    ctx = gpu_ctx_factory()
    ctx.upload_mesh(m)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    n = ctx.n
    big = torch.zeros((17, n), dtype=torch.float64, device="cuda")
    norms = torch.zeros(34, dtype=torch.float64, device="cuda")
    rc = _entry()(ctx.h, 17, big.data_ptr(), big.data_ptr(), norms.data_ptr())
    assert rc == -7  # OFEA_ERR_CAPACITY
    assert b"16" in ob.lib().ofea_last_error()
