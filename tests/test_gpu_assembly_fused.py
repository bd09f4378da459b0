"""One-pass C3D8 assembly (integration fused with the owner-computes gather).

The fused kernel must give K, its block-Jacobi inverse and every solve the
same bits as the two-pass assembly (element matrices, then the gather) that
the oracle tests pin to the reference (src/assemble.cpp:95-151 through
src/Elements/C3D8_Gauss.cpp:19-107), and meshes it does not cover must take
the two-pass path.
"""
import numpy as np
import pytest

from openfea_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def jittered(nx, ny, nz, seed=3):
    ext = np.array([1.0, 0.6, 0.9])
    m = mg.structured_hex(nx, ny, nz, *ext, 210e9, 0.3)
    rng = np.random.default_rng(seed)
    interior = np.all((m.xyz > 1e-9) & (m.xyz < ext - 1e-9), axis=1)
    h = 0.15 * min(ext / np.array([nx, ny, nz]))  # distorted, never inverted
    m.xyz[interior] += rng.uniform(-h, h, (int(interior.sum()), 3))
    m.E = rng.uniform(20e9, 300e9, m.ne)
    return m


def both_paths(ctx_factory, mesh):
    out = []
    for path in (0, 1):
        ctx = ctx_factory()
        ctx.set_assembly_path(path)
        fm = ctx.upload_mesh(mesh)
        ctx.assemble_pattern()
        ctx.assemble_linear()
        out.append((ctx, fm))
    return out


@pytest.mark.parametrize("shape", [(12, 5, 4), (7, 3, 40), (30, 2, 2)])
def test_fused_assembly_matches_two_pass_bitwise(gpu_ctx_factory, shape):
    # z-lines of 5, 41 and 3 nodes: slices inside one line, across two and
    # across many; per-element moduli and distorted elements
    m = jittered(*shape)
    (cf, fm), (ct, _) = both_paths(gpu_ctx_factory, m)
    assert cf.assembly_path() == 0 and ct.assembly_path() == 1
    rf, colf, vf = cf.get_csr()
    rt, colt, vt = ct.get_csr()
    assert np.array_equal(rf, rt) and np.array_equal(colf, colt)
    assert np.array_equal(vf, vt)
    x = np.random.default_rng(1).normal(size=rf.size - 1)
    assert np.array_equal(cf.spmv(x), ct.spmv(x))
    f = np.random.default_rng(2).normal(size=rf.size - 1)
    uf, sf = cf.solve(f, rtol=1e-10, method="GPU_PCG")
    ut, st = ct.solve(f, rtol=1e-10, method="GPU_PCG")
    # the same K and block-Jacobi inverse give the same PCG64 iterates
    assert np.array_equal(uf, ut) and sf["iterations"] == st["iterations"]


def test_fused_assembly_is_bitwise_reproducible(gpu_ctx_factory):
    m = jittered(9, 6, 5)
    ctx = gpu_ctx_factory()
    ctx.upload_mesh(m)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    assert ctx.assembly_path() == 0
    x = np.random.default_rng(4).normal(size=ctx.n)
    y1 = ctx.spmv(x)
    ctx.assemble_linear()
    assert np.array_equal(y1, ctx.spmv(x))


def test_fused_assembly_element_matrices_on_demand(gpu_ctx_factory):
    m = jittered(4, 3, 3)
    (cf, _), (ct, _) = both_paths(gpu_ctx_factory, m)
    assert np.array_equal(cf.element_matrices(0, m.ne, 8), ct.element_matrices(0, m.ne, 8))


def test_meshes_outside_the_fused_kernel_take_two_pass(gpu_ctx_factory):
    tet = mg.tet_block(5, 3, 3)[0]
    ctx = gpu_ctx_factory()
    ctx.upload_mesh(tet)
    ctx.assemble_pattern()
    ctx.assemble_linear()
    assert ctx.assembly_path() == 1
