"""Parity at the workloads' full sizes, against the reference's own code.

* The jittered C3D4 block (60x20x20 cubes x 6 tets, 76,860 DOF, lognormal E,
  random top-face loads): K against the reference's build_CSR + per-element
  fill (live, 1e-13 of max|K|), and the displacement against the reference's
  solution_api("SuperLU_func") solution (committed fixture): FP64 PCG within
  1e-9, mixed and learned within 1e-8 (relative L2).
* The C3D8 cantilever 200x50x50 (1,560,600 DOF, 122.7M non-zeros) and the
  same mesh with the SIMP density field of seed 12: K against the reference's
  assembly (live), and the displacement against the reference-assembled K
  solved by the vendored Eigen CG + incomplete Cholesky to a relative residual
  near 1e-12 (committed on a sub-grid of nodes; a direct factor is out of
  reach at this size): every method within 1e-8.

Each solve runs at the relative residual the benchmark uses for that method
(`RTOL`), so these bars are the accuracy of the timed solves.
"""
import os

import numpy as np
import pytest

import openfea_b200 as ob
from openfea_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
K_TOL = 1e-13
# relative residual of each method's solves in the benchmark and here
RTOL = {"GPU_PCG": 1e-8, "GPU_MIXED": 1e-8, "GPU_LEARNED": 1e-8}
BAR = {"GPU_PCG": 1e-8, "GPU_MIXED": 1e-8, "GPU_LEARNED": 1e-8}


def rel2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def assemble(mesh):
    ctx = ob.Context(0)
    fm = ctx.upload_mesh(mesh)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    return ctx, fm


def check_K_against_reference(reference, ctx, mesh):
    rm = reference.model(mesh)
    cp, ri, val = rm.assemble()
    rp, col, kv = ctx.get_csr()
    assert np.array_equal(rp, cp) and np.array_equal(col, ri), "pattern differs from the reference's build_CSR"
    err = np.abs(kv - val).max() / np.abs(val).max()
    assert err <= K_TOL, err
    return rm


def test_tet_block_full_size_against_reference_superlu(gpu_ctx_factory, reference):
    g = np.load(os.path.join(GOLDEN, "scale_tet_60x20x20.npz"))
    m, ffull = mg.tet_block()
    ctx, fm = assemble(m)
    assert ctx.n == int(g["n"]) == 76860
    check_K_against_reference(reference, ctx, m)
    f = mg.to_free(ffull, fm)
    ctx.learned_train(None, sample_iters=600, sample_every=2, steps=200, batch=16)
    errs = {}
    for method in ("GPU_PCG", "GPU_MIXED", "GPU_LEARNED"):
        ctx.precond_reset()
        u, st = ctx.solve(f, method=method, rtol=RTOL[method])
        assert st["status"] == 0 and st["rel_residual"] <= RTOL[method], (method, st)
        errs[method] = rel2(u, g["u"])
    for method, e in errs.items():
        assert e <= BAR[method], errs
    # the plain method's own bar: 1e-9 at a tighter residual
    u, st = ctx.solve(f, method="GPU_PCG", rtol=1e-12)
    assert rel2(u, g["u"]) <= 1e-9


def scale_case(reference, name, E):
    path = os.path.join(GOLDEN, f"scale_{name}_200x50x50.npz")
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not generated (tests/golden/make_scale_golden.py)")
    g = np.load(path)
    m, ffull = mg.cantilever_large()
    m.E = E
    ctx, fm = assemble(m)
    assert ctx.n == int(g["n"]) == 1560600 and ctx.nnz == 122714982
    rm = check_K_against_reference(reference, ctx, m)
    del rm
    return g, ctx, mg.to_free(ffull, fm)


def check_methods(ctx, f, g, trainer=None):
    idx = g["idx"].astype(np.int64)
    (trainer or ctx).learned_train(None, sample_iters=1000, sample_every=1, steps=200, batch=16)
    if trainer is not None:
        ctx.set_learned_weights(trainer.learned_weights())
    errs = {}
    for method in ("GPU_PCG", "GPU_MIXED", "GPU_LEARNED"):
        ctx.precond_reset()
        u, st = ctx.solve(f, method=method, rtol=RTOL[method])
        assert st["status"] == 0 and st["rel_residual"] <= RTOL[method], (method, st)
        errs[method] = rel2(u[idx], g["u_sub"])
        # whole-vector checks of the same field
        assert abs(np.linalg.norm(u) - float(g["u_norm"])) <= BAR[method] * float(g["u_norm"])
    for method, e in errs.items():
        assert e <= BAR[method], errs
    return errs


def test_cantilever_full_size_against_reference_k_and_eigen_oracle(gpu_ctx_factory, reference):
    g, ctx, f = scale_case(reference, "cantilever", None)
    check_methods(ctx, f, g)


def test_simp_full_size_against_reference_k_and_eigen_oracle(gpu_ctx_factory, reference):
    """The learned stage trained on another density sample (seed 11), as in
    the benchmark's SIMP case."""
    g, ctx, f = scale_case(reference, "simp", 210e9 * mg.simp_density((200, 50, 50), 12, smooth=True) ** 3)
    mt, _ = mg.cantilever_large()
    mt.E = 210e9 * mg.simp_density((200, 50, 50), 11, smooth=True) ** 3
    trainer, _ = assemble(mt)
    check_methods(ctx, f, g, trainer)
