"""The persistent batched solver (ofea_batch_*): several SIMP design variants
of uneven length x several load cases, solved by one cooperative kernel,
against the per-variant solver, the oracle's assembly + a direct solve, its
own determinism, and the failure path of its grid barrier."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import openfea_b200 as ob
from openfea_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def variants(factory, count=4, nrhs=5, nmin=4, nmax=9):
    out = []
    for m, F in mg.design_variants(count=count, nrhs=nrhs, ny=4, nz=4, nmin=nmin, nmax=nmax):
        ctx = factory()
        fm = ctx.upload_mesh(m)
        ctx.assemble_pattern()
        ctx.assemble_linear()
        loads = np.stack([mg.to_free(F[j], fm) for j in range(nrhs)])
        out.append((ctx, m, fm, loads))
    return out


def true_rel_residual(ctx, U, F):
    rp, ci, val = ctx.get_csr()
    K = sp.csr_matrix((val, ci, rp), shape=(ctx.n, ctx.n))
    return max(np.linalg.norm(F[j] - K @ U[j]) / np.linalg.norm(F[j]) for j in range(F.shape[0]))


@pytest.mark.parametrize("method", ["GPU_MIXED", "GPU_PCG"])
def test_batched_matches_per_variant_solves(gpu_ctx_factory, tmp_path, monkeypatch, method):
    monkeypatch.setenv("OFEA_TUNE_FILE", str(tmp_path / "tune.json"))
    vs = variants(gpu_ctx_factory)
    b = ob.Batch([v[0] for v in vs], 5)
    U, st = b.solve([v[3] for v in vs], method=method, rtol=1e-10)
    for (ctx, m, fm, F), u, s in zip(vs, U, st):
        assert s["status"] == 0 and s["rel_residual"] <= 1e-10, s
        assert true_rel_residual(ctx, u, F) <= 1e-10
        ref, _ = ctx.solve(F.T, method="GPU_PCG", rtol=1e-13)
        assert np.linalg.norm(u - ref.T) / np.linalg.norm(ref) < 1e-8
    # the autotuner chose a configuration and kept it on disk
    t = b.tuning(method)
    assert t["rhs_per_lane"] in (1, 2, 4) and t["threads"] == 32 * 8 // t["rhs_per_lane"] and t["ms_per_iteration"] > 0
    data = json.load(open(tmp_path / "tune.json"))
    assert any("nrhs=5" in e["key"] for e in data["entries"])
    b.close()


def test_batched_against_oracle_direct_solve(gpu_ctx_factory, oracle):
    vs = variants(gpu_ctx_factory, count=2, nrhs=3)
    U, st = ob.solve_batched([v[0] for v in vs], [v[3] for v in vs], method="GPU_MIXED", rtol=1e-10)
    for (ctx, m, fm, F), u in zip(vs, U):
        cp, ri, val = oracle.assemble(m, fm)
        K = sp.csc_matrix((val, ri, cp), shape=(ctx.n, ctx.n))
        ref = spla.spsolve(K, F.T)
        assert np.linalg.norm(u - ref.T) / np.linalg.norm(ref) < 1e-8


# relative residual of the batched solves in the benchmark and here
BATCH_RTOL = 1e-8


@pytest.mark.parametrize("method", ["GPU_MIXED", "GPU_PCG"])
def test_batched_config4_variants_against_reference_superlu_class(gpu_ctx_factory, reference, method):
    """Real variants of the batched-reanalysis workload (64 SIMP variants
    n x 20 x 20, n ~ U{20..60}, 16 load cases): its three shortest variants
    (26,460-29,106 DOF), all 16 load cases, solved in one batch at the
    benchmark's residual, against the reference's reanalysis solver on its
    own K: solution_api("SuperLU_class") factors K and solves load case 0,
    superlu_solution_next re-solves the other 15 with that factor
    (src/linear_solution.cpp:23-39, src/solver/solver_superlu.cpp:76-94).
    Every load case within 1e-8 (relative L2)."""
    allv = mg.design_variants()
    pick = sorted(range(len(allv)), key=lambda i: (allv[i][0].nd, i))[:3]
    ctxs, loads, refs = [], [], []
    for i in pick:
        m, F = allv[i]
        ctx = gpu_ctx_factory()
        fm = ctx.upload_mesh(m)
        ctx.assemble_pattern()
        ctx.assemble_linear()
        Ff = np.stack([mg.to_free(F[j], fm) for j in range(F.shape[0])])
        rm = reference.model(m)
        rm.assemble()
        refs.append(rm.solve_multi(Ff))
        ctxs.append(ctx)
        loads.append(Ff)
    U, st = ob.solve_batched(ctxs, loads, method=method, rtol=BATCH_RTOL)
    worst = 0.0
    for u, ref, s in zip(U, refs, st):
        assert s["status"] == 0 and s["rel_residual"] <= BATCH_RTOL, s
        for j in range(ref.shape[0]):
            worst = max(worst, np.linalg.norm(u[j] - ref[j]) / np.linalg.norm(ref[j]))
    assert worst <= 1e-8, worst


def test_batched_is_deterministic_and_handles_one_load_case(gpu_ctx_factory):
    vs = variants(gpu_ctx_factory, count=3, nrhs=1)
    b = ob.Batch([v[0] for v in vs], 1)
    U1, _ = b.solve([v[3] for v in vs], method="GPU_MIXED", rtol=1e-9)
    U2, _ = b.solve([v[3] for v in vs], method="GPU_MIXED", rtol=1e-9)
    for a, c in zip(U1, U2):
        assert np.array_equal(a, c)
    b.close()


def test_batched_rejects_too_many_load_cases(gpu_ctx_factory):
    vs = variants(gpu_ctx_factory, count=1, nrhs=1)
    with pytest.raises(ob.OfeaError) as e:
        ob.Batch([vs[0][0]], 33)
    assert e.value.code == -7


def test_grid_barrier_wait_runs_out_and_context_stays_usable(gpu_ctx_factory):
    vs = variants(gpu_ctx_factory, count=1, nrhs=2)
    ctx = vs[0][0]
    assert ob.check_barrier_timeout(ctx, limit_ms=20) == 0
    b = ob.Batch([ctx], 2)
    U, st = b.solve([vs[0][3]], method="GPU_MIXED", rtol=1e-9)
    assert st[0]["status"] == 0
    b.close()


def test_batched_mixes_element_types(gpu_ctx_factory, oracle):
    """A batch holding a C3D4 tet block (per-element E) beside C3D8 variants:
    each variant is solved against its own K (checked with the oracle's)."""
    vs = variants(gpu_ctx_factory, count=2, nrhs=4)
    m, ffull = mg.tet_block(8, 4, 4)
    ctx = gpu_ctx_factory()
    fm = ctx.upload_mesh(m)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    rng = np.random.default_rng(3)
    Ft = np.stack([mg.to_free(ffull * rng.uniform(0.5, 2.0), fm) for _ in range(4)])
    items = vs + [(ctx, m, fm, Ft)]
    U, st = ob.solve_batched([v[0] for v in items], [v[3] for v in items], method="GPU_MIXED", rtol=1e-10)
    for (c, mm, ff, F), u, s in zip(items, U, st):
        assert s["status"] == 0
        cp, ri, val = oracle.assemble(mm, ff)
        K = sp.csc_matrix((val, ri, cp), shape=(c.n, c.n))
        for j in range(F.shape[0]):
            assert np.linalg.norm(F[j] - K @ u[j]) <= 1.0001e-10 * np.linalg.norm(F[j])


@pytest.mark.parametrize("method,init,per_iter", [("GPU_MIXED", 8, 10), ("GPU_PCG", 4, 4)])
def test_batched_phase_trace(gpu_ctx_factory, tmp_path, monkeypatch, method, init, per_iter):
    # one launch: the init phases, then per iteration every phase but the
    # last iteration's V-cycle (the loop ends after the convergence check)
    monkeypatch.setenv("OFEA_TUNE_FILE", str(tmp_path / "tune.json"))
    vs = variants(gpu_ctx_factory, count=2, nrhs=3)
    b = ob.Batch([v[0] for v in vs], 3)
    with pytest.raises(ob.OfeaError):
        b.phase_times()  # tracing is off
    b.set_trace(100000)
    _, st = b.solve([v[3] for v in vs], method=method, rtol=1e-9)
    assert all(s["status"] == 0 and s["refinements"] == 0 for s in st), st
    it = max(s["iterations"] for s in st)
    t = b.phase_times()
    expect = init + per_iter * it if method == "GPU_PCG" else init + per_iter * (it - 1) + 4
    assert len(t) == expect
    assert np.all(t > 0) and t.sum() <= 1e3 * st[0]["seconds"]
    # a short trace keeps the first phases only
    b.set_trace(5)
    b.solve([v[3] for v in vs], method=method, rtol=1e-9)
    assert len(b.phase_times()) == 5
    b.set_trace(0)
    with pytest.raises(ob.OfeaError):
        b.phase_times()
    b.close()
