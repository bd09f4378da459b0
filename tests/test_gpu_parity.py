"""GPU path vs the oracle and the reference's own results, through the C ABI.

Bars: integer pattern data bit-exact; K entries and element matrices within
1e-13 of max|K| (FP64, different summation order); displacements within 1e-9
(relative L2) of the reference's SuperLU solution for the FP64 PCG;
mixed precision within 1e-8.
"""
import os
import numpy as np
import pytest

import openfea_b200 as ob
from openfea_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

K_TOL = 1e-13


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def rel2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def assemble(ctx_factory, mesh, fm=None):
    ctx = ctx_factory()
    fm = ctx.upload_mesh(mesh, fm)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    return ctx, fm


def hex_block_jittered(nx=4, ny=3, nz=3, seed=5):
    m = mg.structured_hex(nx, ny, nz, 1.0, 0.8, 0.7, 210e9, 0.3)
    rng = np.random.default_rng(seed)
    h = 0.2
    m.xyz = m.xyz + rng.uniform(-0.15 * h, 0.15 * h, m.xyz.shape)
    m.E = rng.uniform(50e9, 300e9, m.ne)
    return m


def test_element_matrices_match_reference(gpu_ctx_factory, golden):
    g = golden("ref_elements.npz")
    for tag, et, npe in (("hex", 1, 8), ("tet", 0, 4)):
        for k in range(4):
            X, (E, nu) = g[f"{tag}{k}_X"], g[f"{tag}{k}_mat"]
            topo = np.zeros((1, 8), np.int32)
            topo[0, :npe] = np.arange(1, npe + 1)
            m = mg.Mesh(X, topo, np.array([et], np.int32), np.array([1], np.int32), None, E, nu)
            ctx = gpu_ctx_factory()
            ctx.upload(m.xyz, m.topo, m.etype, np.arange(npe, dtype=np.int32), E, nu)
            ctx.assemble_pattern()
            ctx.assemble_linear()
            Ke = ctx.element_matrices(0, 1, npe)[0]
            assert rel(Ke, g[f"{tag}{k}_K"]) < K_TOL, (tag, k)


def test_element_matrices_match_oracle_many(gpu_ctx_factory, oracle):
    for m in (hex_block_jittered(), mg.tet_block(5, 3, 3)[0]):
        ctx, fm = assemble(gpu_ctx_factory, m)
        npe = 8 if m.etype[0] == 1 else 4
        Kg = ctx.element_matrices(0, m.ne, npe)
        for e in range(m.ne):
            X = m.xyz[m.topo[e, :npe] - 1]
            Ko, _ = oracle.element_ke(int(m.etype[e]), X, m.E[e], m.nu)
            assert rel(Kg[e], Ko) < K_TOL, e


@pytest.mark.parametrize("case", ["hex", "tet", "mixed"])
def test_pattern_and_values_match_oracle(gpu_ctx_factory, oracle, inp_file, case):
    if case == "hex":
        m = hex_block_jittered(6, 4, 3)
    elif case == "tet":
        m = mg.tet_block(6, 4, 3)[0]
    else:
        d = ob.inp_read(inp_file("implicite_test_C3D4_C3D8.inp"))
        m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, d["E"], d["nu"])
    ctx, fm = assemble(gpu_ctx_factory, m)
    rp, col, val = ctx.get_csr()
    cp, ri, ov = oracle.assemble(m, fm)
    assert np.array_equal(rp, cp) and np.array_equal(col, ri)  # bit-exact pattern
    assert rel(val, ov) < K_TOL


def test_assembly_is_bitwise_reproducible(gpu_ctx_factory):
    m = mg.tet_block(8, 5, 5)[0]
    ctx, _ = assemble(gpu_ctx_factory, m)
    v1 = ctx.get_csr()[2]
    ctx.assemble_linear()
    v2 = ctx.get_csr()[2]
    assert np.array_equal(v1, v2)


def test_spmv_matches_oracle(gpu_ctx_factory, oracle):
    m = hex_block_jittered(7, 4, 4)
    ctx, fm = assemble(gpu_ctx_factory, m)
    cp, ri, ov = oracle.assemble(m, fm)
    x = np.random.default_rng(2).normal(size=cp.size - 1)
    y = ctx.spmv(x)
    yo = oracle.spmv(cp, ri, ov, x)
    assert rel(y, yo) < 1e-13


@pytest.mark.parametrize("case", ["hex", "tet"])
def test_nl_tangent_and_internal_force_match_oracle(gpu_ctx_factory, oracle, case):
    m = hex_block_jittered(5, 3, 3) if case == "hex" else mg.tet_block(5, 3, 3)[0]
    ctx = gpu_ctx_factory()
    fm = ctx.upload_mesh(m)
    n, _ = ctx.assemble_pattern()
    cp, ri = oracle.pattern(m, fm)
    rng = np.random.default_rng(11)
    for amp in (0.0, 1e-3, 3e-2):
        u = rng.normal(0, amp, n)
        fint = ctx.assemble_nl(u)
        rp, col, val = ctx.get_csr()
        ov, of = oracle.nl_assemble(m, fm, cp, ri, u)
        assert np.array_equal(rp, cp) and np.array_equal(col, ri)
        assert rel(val, ov) < K_TOL, amp
        scale = np.abs(ov).max() * max(np.abs(u).max(), 1e-300)
        assert np.abs(fint - of).max() <= 1e-12 * scale + 1e-300, amp


def test_cantilever_pcg64_matches_reference_superlu(gpu_ctx_factory, golden):
    g = golden("ref_models.npz")
    m, _ = mg.cantilever_small()
    ctx, fm = assemble(gpu_ctx_factory, m)
    assert ctx.nnz == 88218
    u, st = ctx.solve(g["cantilever_f"], method="GPU_PCG", rtol=1e-11)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-11
    assert rel2(u, g["cantilever_u"]) < 1e-9


def test_cantilever_mixed_matches_reference_superlu(gpu_ctx_factory, golden):
    g = golden("ref_models.npz")
    m, _ = mg.cantilever_small()
    ctx, fm = assemble(gpu_ctx_factory, m)
    u, st = ctx.solve(g["cantilever_f"], method="GPU_MIXED", rtol=1e-10)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-10
    assert rel2(u, g["cantilever_u"]) < 1e-8  # stated error bound of the mixed solver here


@pytest.mark.parametrize("graph", [True, False])
def test_solve_is_bitwise_reproducible(gpu_ctx_factory, graph):
    m, ffull = mg.cantilever_small()
    ctx, fm = assemble(gpu_ctx_factory, m)
    f = mg.to_free(ffull, fm)
    u1, s1 = ctx.solve(f, rtol=1e-10, use_graph=graph)
    u2, s2 = ctx.solve(f, rtol=1e-10, use_graph=graph)
    assert np.array_equal(u1, u2) and s1["iterations"] == s2["iterations"]


def test_golden_vtk_on_gpu(gpu_ctx_factory, golden, inp_file, tmp_path):
    d = ob.inp_read(inp_file("mesh_o.inp"))
    m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, 2.1e5, 0.3)
    ctx, fm = assemble(gpu_ctx_factory, m)
    f = ob.build_single_load(m.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
    u, st = ctx.solve(f, rtol=1e-10)
    uf = ob.full_displacement(m.nd, fm, u)
    ug = golden("cadcae_o_u.npz")["u"].ravel()
    assert rel2(uf, ug) < 3e-6  # the VTK's 6-digit print precision
    ob.write_vtk(tmp_path / "o.vtk", m.xyz, m.topo, m.etype, uf)


def test_mixed_sample_matches_reference_superlu(gpu_ctx_factory, golden, inp_file):
    g = golden("ref_models.npz")
    d = ob.inp_read(inp_file("implicite_test_C3D4_C3D8.inp"))
    m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, d["E"], d["nu"])
    ctx, fm = assemble(gpu_ctx_factory, m)
    f = ob.build_single_load(m.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
    u, st = ctx.solve(f, rtol=1e-11)
    assert rel2(u, g["implicite_test_C3D4_C3D8_u"]) < 1e-9
    u2, st2 = ctx.solve(f, method="GPU_MIXED", rtol=1e-10)
    assert rel2(u2, g["implicite_test_C3D4_C3D8_u"]) < 1e-8


def test_nl_newton_iterates_match_reference(gpu_ctx_factory, golden, inp_file):
    g = golden("ref_models.npz")
    d = ob.inp_read(inp_file("nlcae.inp"))
    m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, d["E"], d["nu"])
    ctx = gpu_ctx_factory()
    ctx.upload_mesh(m)
    ctx.assemble_pattern()
    f = g["nlcae_f"]
    u = np.zeros(f.size)
    for it in range(3):
        fint = ctx.assemble_nl(u)
        du, st = ctx.solve(f - fint, rtol=1e-11)
        u = u + du
        assert rel2(u, g["nlcae_iterates"][it]) < 1e-8, it


def test_tet_block_per_element_modulus(gpu_ctx_factory, oracle):
    """The jittered Kuhn-tet block (lognormal E, random top loads)
    at a size the CPU checker solves directly."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    m, ffull = mg.tet_block(16, 6, 6)
    ctx, fm = assemble(gpu_ctx_factory, m)
    f = mg.to_free(ffull, fm)
    cp, ri, ov = oracle.assemble(m, fm)
    uo = spl.spsolve(sp.csc_matrix((ov, ri, cp)), f)
    for method, tol, bar in (("GPU_PCG", 1e-12, 1e-9), ("GPU_MIXED", 1e-11, 1e-8)):
        u, st = ctx.solve(f, method=method, rtol=tol)
        assert st["status"] == 0
        assert rel2(u, uo) < bar, method


def test_full_size_tet_block_properties(gpu_ctx_factory):
    """The full 60x20x20 x 6-tet workload (144k elements, 76,860 DOF):
    symmetric K, positive diagonal and a converged FP64 residual."""
    m, ffull = mg.tet_block()
    ctx, fm = assemble(gpu_ctx_factory, m)
    assert ctx.n == 76860 and ctx.nnz == 3252042
    rng = np.random.default_rng(0)
    x, y = rng.normal(size=ctx.n), rng.normal(size=ctx.n)
    kx, ky = ctx.spmv(x), ctx.spmv(y)
    assert abs(x @ ky - y @ kx) <= 1e-12 * abs(x @ kx)
    f = mg.to_free(ffull, fm)
    u, st = ctx.solve(f, method="GPU_PCG", rtol=1e-8)
    assert st["status"] == 0 and st["rel_residual"] <= 1e-8
    r = f - ctx.spmv(u)
    assert np.linalg.norm(r) / np.linalg.norm(f) <= 1e-8
    u2, st2 = ctx.solve(f, method="GPU_MIXED", rtol=1e-8)
    assert st2["status"] == 0 and rel2(u2, u) < 1e-6


# ------------------------------------------------------------ error paths --

def test_errors_are_status_codes(gpu_ctx_factory):
    m, ffull = mg.cantilever_small()
    ctx = gpu_ctx_factory()
    fm = ctx.upload_mesh(m)
    with pytest.raises(ob.OfeaError) as e:
        ctx.assemble_linear()
    assert e.value.code == -6  # STATE: assembly before the pattern
    ctx.assemble_pattern()
    with pytest.raises(ob.OfeaError) as e:
        ctx.solve(np.ones(ctx.n))
    assert e.value.code == -6  # STATE: solve before assembly
    ctx.assemble_linear()
    f = mg.to_free(ffull, fm)
    u, st = ctx.solve(f, rtol=1e-12, max_iter=5, raise_on_error=False)
    assert st["status"] == -4  # NOT_CONVERGED
    bad = f.copy()
    bad[7] = np.nan
    u, st = ctx.solve(bad, raise_on_error=False)
    assert st["status"] in (-8, -4)
    with pytest.raises(ob.OfeaError) as e:
        ctx.solve(f, method=7)
    assert e.value.code == -11
    u, st = ctx.solve(np.zeros_like(f))
    assert st["status"] == 0 and not u.any()


def test_unconstrained_model_is_rejected(gpu_ctx_factory):
    m, ffull = mg.cantilever_small()
    ctx = gpu_ctx_factory()
    fm = np.arange(m.nd, dtype=np.int32)  # no boundary conditions: K singular
    ctx.upload(m.xyz, m.topo, m.etype, fm, m.E0, m.nu)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    u, st = ctx.solve(ffull, rtol=1e-10, max_iter=3000, raise_on_error=False)
    assert st["status"] in (-4, -8)


def test_bad_uploads_rejected(gpu_ctx_factory):
    m, _ = mg.cantilever_small()
    ctx = gpu_ctx_factory()
    fm = mg.free_map(m.nd, m.fix)
    topo = m.topo.copy()
    topo[0, 0] = m.nd + 5
    with pytest.raises(ob.OfeaError):
        ctx.upload(m.xyz, topo, m.etype, fm, m.E0, m.nu)
    with pytest.raises(ob.OfeaError):
        ctx.upload(m.xyz, m.topo, m.etype, fm, m.E0, 0.5)
    fm2 = fm.copy()
    fm2[fm2 == 3] = 4
    with pytest.raises(ob.OfeaError):
        ctx.upload(m.xyz, m.topo, m.etype, fm2, m.E0, m.nu)
    # the checks run over chunks of elements in parallel; the error reported is
    # still the first one in element order
    topo = m.topo.copy()
    topo[-1, 1] = topo[-1, 0]  # last element repeats a node
    with pytest.raises(ob.OfeaError, match="repeats a node"):
        ctx.upload(m.xyz, topo, m.etype, fm, m.E0, m.nu)
    topo[3, 2] = 0  # an earlier element: node id out of range
    with pytest.raises(ob.OfeaError, match="out of range"):
        ctx.upload(m.xyz, topo, m.etype, fm, m.E0, m.nu)
    et = m.etype.copy()
    et[1] = 2
    with pytest.raises(ob.OfeaError, match="element type"):
        ctx.upload(m.xyz, topo, et, fm, m.E0, m.nu)
    xyz = m.xyz.copy()
    xyz[-1, 2] = np.nan
    with pytest.raises(ob.OfeaError, match="non-finite"):
        ctx.upload(xyz, m.topo, m.etype, fm, m.E0, m.nu)
    # and a valid mesh after the failures uploads and solves
    ctx.upload(m.xyz, m.topo, m.etype, fm, m.E0, m.nu)
    ctx.assemble_pattern()
    ctx.assemble_linear()


@pytest.mark.parametrize("solver", ["GPU_PCG", "GPU_MIXED", "GPU_LEARNED"])
def test_cli_drives_the_gpu_path(golden, inp_file, tmp_path, solver):
    """The command-line driver: .inp in, .vtk out (the reference's
    OpenFEA -i ... -o ...), the GPU solver picked by -solver; the written
    u_z field matches the reference's golden result to its print precision.
    GPU_LEARNED trains on the model once, saves the weights and a second
    run reuses them."""
    import subprocess
    cli = os.path.join(os.path.dirname(ob.__file__), "ofea_cli")
    inp = inp_file("mesh_o.inp")
    out = tmp_path / "o.vtk"
    args = [cli, "-i", inp, "-o", str(out), "-solver", solver, "-rtol", "1e-10", "-E", "2.1e5", "-nu", "0.3"]
    runs = [args]
    if solver == "GPU_LEARNED":
        w = str(tmp_path / "gnn.bin")
        runs = [args + ["-save-weights", w], args + ["-weights", w]]
    ug = golden("cadcae_o_u.npz")["u"].ravel()
    for a in runs:
        r = subprocess.run(a, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        lines = out.read_text().split("\n")
        j = lines.index("SCALARS u_z double 1")
        uz = np.array([float(x) for x in lines[j + 2:j + 2 + 625]])
        assert np.abs(uz - ug[2::3]).max() <= 3e-6 * np.abs(ug[2::3]).max()
