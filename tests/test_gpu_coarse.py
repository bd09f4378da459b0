"""The coarse level's two solves with E = Z^T K Z: the block LDL^T factor of
the banded E (the default; one thread-block cluster, applied as two FP32
triangular GEMVs) against the dense Gauss-Jordan inverse (one FP32 GEMV).
Both drop the directions whose pivots vanish, so they must apply the same
operator up to FP32 rounding and give the solver the same iterations."""
import numpy as np
import pytest

import openfea_b200 as ob
from openfea_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def _ctx(factory, mesh, ffull):
    ctx = factory()
    fm = ctx.upload_mesh(mesh)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    return ctx, mg.to_free(ffull, fm)


def _compare(ctx, f, method, rtol, rel_apply):
    rng = np.random.default_rng(3)
    u_f, s_f = ctx.solve(f, method=method, rtol=rtol)
    m, factored = ctx.coarse_apply()
    assert factored, "the banded coarse matrix takes the factor by default"
    C = rng.normal(size=(3, m))
    Yf = [ctx.coarse_apply(c) for c in C]
    ctx.set_coarse_solver(1)
    u_d, s_d = ctx.solve(f, method=method, rtol=rtol)
    m2, factored2 = ctx.coarse_apply()
    assert m2 == m and not factored2
    Yd = [ctx.coarse_apply(c) for c in C]
    for yf, yd in zip(Yf, Yd):
        # same operator: the two FP32 forms of E^-1 agree to their rounding
        assert np.linalg.norm(yf - yd) <= rel_apply * np.linalg.norm(yd)
    assert s_f["status"] == 0 and s_d["status"] == 0
    # FP32 rounding of a nearly singular E differs between the two forms:
    # the iteration counts may differ by some on irregular aggregates (the
    # mixed sample with 30-node aggregates: up to a fifth)
    assert abs(s_f["iterations"] - s_d["iterations"]) <= max(2, s_d["iterations"] // 5), (
        s_f["iterations"], s_d["iterations"])
    assert np.linalg.norm(u_f - u_d) <= 10 * rtol * np.linalg.norm(u_d)
    return m


def test_factor_matches_dense_inverse_on_a_cantilever(gpu_ctx_factory):
    mesh, ffull = mg.cantilever_large(60, 12, 12)
    ctx, f = _ctx(gpu_ctx_factory, mesh, ffull)
    ctx.set_coarse_nodes(40)  # about 250 aggregates: m > 64 * 20, several blocks of band
    m = _compare(ctx, f, "GPU_MIXED", 1e-10, 1e-4)
    assert m > 64 * 20


def test_factor_matches_dense_inverse_on_the_mixed_sample(gpu_ctx_factory, inp_file):
    """The reference's mixed C3D4/C3D8 sample: irregular aggregates, some too
    small for all six rigid modes (vanishing pivots)."""
    d = ob.inp_read(inp_file("implicite_test_C3D4_C3D8.inp"))
    mesh = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, d["E"], d["nu"])
    ctx = gpu_ctx_factory()
    fm = ctx.upload_mesh(mesh)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    f = ob.build_single_load(mesh.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
    ctx.set_coarse_nodes(30)
    _compare(ctx, f, "GPU_MIXED", 1e-10, 1e-3)


def test_learned_solve_uses_the_factor(gpu_ctx_factory):
    mesh, ffull = mg.cantilever_large(40, 10, 10)
    ctx, f = _ctx(gpu_ctx_factory, mesh, ffull)
    ctx.set_coarse_nodes(60)
    ctx.learned_train(sample_iters=64, sample_every=4, steps=5, batch=4)
    ctx.precond_reset()
    u_l, s_l = ctx.solve(f, method="GPU_LEARNED", rtol=1e-10)
    assert s_l["status"] == 0 and s_l["rejected_learned"] == 0
    assert ctx.coarse_apply()[1]
    ctx.set_coarse_solver(1)
    u_d, s_d = ctx.solve(f, method="GPU_LEARNED", rtol=1e-10)
    assert s_d["status"] == 0 and not ctx.coarse_apply()[1]
    assert abs(s_l["iterations"] - s_d["iterations"]) <= 2
    assert np.linalg.norm(u_l - u_d) <= 1e-9 * np.linalg.norm(u_d)


def test_coarse_solver_argument_checked(gpu_ctx_factory):
    mesh, ffull = mg.cantilever_large(10, 4, 4)
    ctx, f = _ctx(gpu_ctx_factory, mesh, ffull)
    with pytest.raises(ob.OfeaError):
        ctx.set_coarse_solver(2)
    with pytest.raises(ob.OfeaError):
        ctx.coarse_apply()  # no coarse level before a MIXED / LEARNED solve
