"""The solution_api drop-in: the GPU solver called from the reference's own
flow, with the matrix the reference assembled.

* ofea_matrix_upload_csc takes the reference's CSC arrays (col_idx_, row_idx_,
  nz_val_) as solution_api receives them; the solve matches the reference's
  own SuperLU solution of the same arrays.
* oracle/_ref/ref_gpu_driver is the reference's read -> set_BCs ->
  build_CSR / fill_CSR_sparse_mat -> solution_api(solver) -> stress -> VTK
  flow, built from the reference's sources with
  openfea_b200/integration/ofea_solution_api.cpp bound in; its GPU_* output
  reproduces the shipped cadcae_o.vtk and the same driver's SuperLU run,
  for the linear path and for the -nl Newton loop (solution_nl_api).
"""
import os
import subprocess

import numpy as np
import pytest

import openfea_b200 as ob

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_driver")


def rel2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name, E, nu", [("mesh_o.inp", 2.1e5, 0.3), ("implicite_test_C3D4_C3D8.inp", None, None)])
def test_csc_upload_matches_reference_superlu(gpu_ctx_factory, reference, inp_file, name, E, nu):
    rm = reference.model_from_inp(inp_file(name), E=E, nu=nu)
    cp, ri, val = rm.assemble()
    arrays = rm.mesh_arrays()
    f = arrays["f"]
    rm.set_load(f)
    u_ref = rm.solve()
    ctx = gpu_ctx_factory()
    ctx.upload_csc(arrays["xyz"], arrays["free_map"], cp, ri, val)
    rp, col, kv = ctx.get_csr()
    assert np.array_equal(rp, cp) and np.array_equal(col, ri) and np.array_equal(kv, val)
    # (the FP64 residual floor of these samples is near 1e-11: 7.8e-12 and 7.5e-11)
    for method, rtol, bar in (("GPU_PCG", 1e-10, 1e-9), ("GPU_MIXED", 1e-10, 1e-8)):
        u, st = ctx.solve(f, method=method, rtol=rtol)
        assert st["status"] == 0
        assert rel2(u, u_ref) <= bar, (method, rel2(u, u_ref))
    # element-based calls are refused on a matrix-only context
    with pytest.raises(ob.OfeaError) as e:
        ctx.assemble_linear()
    assert e.value.code == -6


def test_csc_upload_rejects_a_matrix_without_block_structure(gpu_ctx_factory, reference, inp_file):
    rm = reference.model_from_inp(inp_file("mesh_o.inp"), E=2.1e5, nu=0.3)
    cp, ri, val = rm.assemble()
    arrays = rm.mesh_arrays()
    ctx = gpu_ctx_factory()
    bad = ri.copy()
    bad[cp[4] + 1] += 1  # a row id that breaks the 3x3 blocks (still in range)
    with pytest.raises(ob.OfeaError, match="block structured"):
        ctx.upload_csc(arrays["xyz"], arrays["free_map"], cp, bad, val)
    with pytest.raises(ob.OfeaError):
        ctx.upload_csc(arrays["xyz"], arrays["free_map"], cp[:-3], ri, val)  # n != 3 x free nodes
    # the context is usable after the failures
    ctx.upload_csc(arrays["xyz"], arrays["free_map"], cp, ri, val)
    u, st = ctx.solve(arrays["f"], method="GPU_PCG", rtol=1e-10)
    assert st["status"] == 0


def read_vtk_u(path, nd):
    lines = open(path).read().split("\n")
    out = []
    for c in "xyz":
        j = lines.index(f"SCALARS u_{c} double 1")
        out.append([float(x) for x in lines[j + 2:j + 2 + nd]])
    return np.array(out).T


def run_driver(args, tmp_path, tag):
    out = tmp_path / f"{tag}.vtk"
    r = subprocess.run([DRIVER, *args, "-o", str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return out, r.stdout


@pytest.mark.parametrize("solver, where", [("GPU_PCG", "solution_api"), ("GPU_MIXED", "solution_api"),
                                           ("GPU_LEARNED", "solution_api"), ("GPU_MIXED", "implict_analysis")])
def test_reference_flow_with_gpu_solution_api(golden, inp_file, tmp_path, solver, where):
    """The shipped sample (sample_model/CA/mesh_o.inp, E = 2.1e5, nu = 0.3):
    the reference's own driver sequence with solution_api("GPU_*") (K
    assembled by the reference), or with gpu_implicit_analysis in place of
    its assembly and solve, writes the golden cadcae_o.vtk displacement to its
    6 printed digits."""
    if not os.path.exists(DRIVER):
        pytest.skip("oracle/_ref/ref_gpu_driver not built (needs the reference tree)")
    args = ["-i", inp_file("mesh_o.inp"), "-E", "2.1e5", "-nu", "0.3"]
    extra = ["-gpu-assembly"] if where == "implict_analysis" else []
    out_gpu, _ = run_driver(args + ["-solver", solver] + extra, tmp_path, solver + where)
    out_cpu, _ = run_driver(args + ["-solver", "SuperLU_func"], tmp_path, "superlu")
    ug = golden("cadcae_o_u.npz")["u"].reshape(-1, 3)
    u_gpu, u_cpu = read_vtk_u(out_gpu, ug.shape[0]), read_vtk_u(out_cpu, ug.shape[0])
    assert np.abs(u_gpu - ug).max() <= 3e-6 * np.abs(ug).max()
    assert np.abs(u_gpu - u_cpu).max() <= 3e-6 * np.abs(u_cpu).max()


def test_reference_newton_loop_with_gpu_solution_nl_api(inp_file, tmp_path):
    """-nl on the shipped nlcae.inp: the reference's Newton loop with
    solution_nl_api("GPU_PCG") takes the same number of iterations as with
    SuperLU and writes the same displacement to the printed digits."""
    if not os.path.exists(DRIVER):
        pytest.skip("oracle/_ref/ref_gpu_driver not built (needs the reference tree)")
    args = ["-i", inp_file("nlcae.inp"), "-nl"]
    out_gpu, log_gpu = run_driver(args + ["-solver", "GPU_PCG"], tmp_path, "nl_gpu")
    out_cpu, log_cpu = run_driver(args + ["-solver", "SuperLU_func"], tmp_path, "nl_cpu")
    it_gpu = [ln for ln in log_gpu.split("\n") if ln.startswith("newton")]
    it_cpu = [ln for ln in log_cpu.split("\n") if ln.startswith("newton")]
    assert len(it_gpu) == len(it_cpu) >= 2
    nd = int(open(out_cpu).read().split("POINTS")[1].split()[0])
    u_gpu, u_cpu = read_vtk_u(out_gpu, nd), read_vtk_u(out_cpu, nd)
    assert np.abs(u_gpu - u_cpu).max() <= 3e-6 * np.abs(u_cpu).max()
