"""Combined-approximations reanalysis on the device (ofea_ca_reanalysis)
against the reference's shipped CA output and the oracle's restatement of
src/ca_analysis.cpp."""
import dataclasses

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import openfea_b200 as ob
from openfea_b200 import meshgen as mg
from oracle import ca_oracle

pytestmark = pytest.mark.gpu


def contexts(factory, m0, m1):
    out = []
    for m in (m0, m1):
        c = factory()
        fm = c.upload_mesh(m)
        c.assemble_pattern()
        c.assemble_linear()
        out.append(c)
    return out[0], out[1], fm


def test_ca_reproduces_the_shipped_output(gpu_ctx_factory, ca_sample, golden):
    """n_basis = 1 is the reference's shipped run (its basis stays at u_0);
    u_0 is solved on the device here."""
    s = ca_sample
    base, mod, fm = contexts(gpu_ctx_factory, s["m0"], s["m1"])
    assert np.array_equal(fm, s["fm"])
    u, st = ob.ca_reanalysis(base, mod, s["f"], None, n_basis=1)
    assert st["status"] == 0 and st["basis_used"] == 1 and st["solve_iterations"] > 0
    un = ca_oracle.to_modified_nodes(u, fm, s["ci"]["node_map"])
    ug = golden("cadcae_ca_u.npz")["u"]
    assert np.linalg.norm(un - ug) / np.linalg.norm(ug) < 1e-5  # 6 printed digits
    u0 = spla.spsolve(s["K0"].tocsc(), s["f"])
    ref = ca_oracle.ca_reanalysis(s["K0"], s["dK"], s["f"], u0, 1)
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-9


@pytest.mark.parametrize("nb", [2, 4])
def test_ca_basis_matches_oracle(gpu_ctx_factory, ca_sample, nb):
    s = ca_sample
    base, mod, fm = contexts(gpu_ctx_factory, s["m0"], s["m1"])
    u0 = spla.spsolve(s["K0"].tocsc(), s["f"])
    u, st = ob.ca_reanalysis(base, mod, s["f"], u0, n_basis=nb, rtol=1e-10)
    assert st["status"] == 0 and st["basis_used"] == nb and st["basis_requested"] == nb
    ref = ca_oracle.ca_reanalysis(s["K0"], s["dK"], s["f"], u0, nb)
    assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-7
    K = s["K0"] + s["dK"]
    rr = np.linalg.norm(s["f"] - K @ ref) / np.linalg.norm(s["f"])
    assert st["rel_residual"] == pytest.approx(rr, rel=1e-5)
    # reproducible: the same call gives the same bits
    u2, _ = ob.ca_reanalysis(base, mod, s["f"], u0, n_basis=nb, rtol=1e-10)
    assert np.array_equal(u, u2)


def test_ca_hex_with_moved_nodes_and_deleted_elements(gpu_ctx_factory, oracle):
    """C3D8 cantilever: a band of elements deleted and interior nodes moved;
    the oracle builds ΔK = K(modified) - K0 on its own assembly."""
    m0, ffull = mg.cantilever_small()
    rng = np.random.default_rng(3)
    xyz1 = m0.xyz.copy()
    inner = np.flatnonzero((m0.xyz[:, 0] > 0.3) & (m0.xyz[:, 0] < 0.7) & (m0.xyz[:, 1] > 0) & (m0.xyz[:, 1] < 0.2)
                           & (m0.xyz[:, 2] > 0) & (m0.xyz[:, 2] < 0.2))
    xyz1[inner] += rng.uniform(-0.004, 0.004, (inner.size, 3))
    E1 = np.full(m0.ne, m0.E0)
    E1[40:48] = 0.0
    m1 = dataclasses.replace(m0, xyz=xyz1, E=E1)
    base, mod, fm = contexts(gpu_ctx_factory, m0, m1)
    n = base.n
    f = mg.to_free(ffull, fm)
    K = []
    for m in (m0, m1):
        cp, ri, val = oracle.assemble(m, fm)
        K.append(sp.csc_matrix((val, ri, cp), shape=(n, n)))
    u0 = spla.spsolve(K[0], f)
    for nb in (1, 3):
        u, st = ob.ca_reanalysis(base, mod, f, None, n_basis=nb, method="GPU_MIXED", rtol=1e-10)
        assert st["status"] == 0 and st["basis_used"] == nb
        ref = ca_oracle.ca_reanalysis(K[0], K[1] - K[0], f, u0, nb)
        assert np.linalg.norm(u - ref) / np.linalg.norm(ref) < 1e-7
    # a larger basis is closer to the modified model's own solution
    uex = spla.spsolve(K[1], f)
    e1 = np.linalg.norm(ob.ca_reanalysis(base, mod, f, u0, n_basis=1)[0] - uex)
    e3 = np.linalg.norm(ob.ca_reanalysis(base, mod, f, u0, n_basis=3)[0] - uex)
    assert e3 < e1


def test_ca_rejects_bad_arguments(gpu_ctx_factory):
    m0, ffull = mg.cantilever_small()
    base, mod, fm = contexts(gpu_ctx_factory, m0, m0)
    f = mg.to_free(ffull, fm)
    for nb in (0, 33):
        with pytest.raises(ob.OfeaError) as e:
            ob.ca_reanalysis(base, mod, f, None, n_basis=nb)
        assert e.value.code == -1
    with pytest.raises(ob.OfeaError):
        ob.ca_reanalysis(base, base, f, None, n_basis=2)
    # different sizes
    small = mg.structured_hex(20, 4, 3, 1.0, 0.2, 0.15)
    c = gpu_ctx_factory()
    c.upload_mesh(small)
    c.assemble_pattern()
    c.assemble_linear()
    with pytest.raises(ob.OfeaError) as e:
        ob.ca_reanalysis(base, c, f, None, n_basis=2)
    assert e.value.code == -1
    # same sizes and pattern, different numbering: the free nodes numbered in reverse
    fm2 = fm.copy()
    fr = fm2 >= 0
    fm2[fr] = fm2[fr].max() - fm2[fr]
    c2 = gpu_ctx_factory()
    c2.upload_mesh(m0, free_map=fm2)
    c2.assemble_pattern()
    c2.assemble_linear()
    assert c2.n == base.n and c2.nnz == base.nnz
    with pytest.raises(ob.OfeaError) as e:
        ob.ca_reanalysis(base, c2, f, None, n_basis=2)
    assert e.value.code == -1
    # same numbering, different elements: one element's nodes changed
    topo = m0.topo.copy()
    topo[0, 0] = topo[200, 6]
    c3 = gpu_ctx_factory()
    c3.upload_mesh(dataclasses.replace(m0, topo=topo))
    c3.assemble_pattern()
    c3.assemble_linear()
    with pytest.raises(ob.OfeaError) as e:
        ob.ca_reanalysis(base, c3, f, None, n_basis=2)
    assert e.value.code == -1


def test_cli_ca_mode_writes_the_modified_model(golden, inp_file, tmp_path):
    """ofea_cli -ca: the analysis of mesh_o.inp, then the reanalysis from the
    change file onto mesh_m.inp's nodes; with one basis vector the written
    field is the reference's shipped cadcae_ca.vtk to its print precision."""
    import os
    import subprocess
    cli = os.path.join(os.path.dirname(ob.__file__), "ofea_cli")
    ug = golden("cadcae_ca_u.npz")["u"]
    for nb in (1, 4):
        out, out_ca = tmp_path / f"o{nb}.vtk", tmp_path / f"ca{nb}.vtk"
        args = [cli, "-i", inp_file("mesh_o.inp"), "-o", str(out), "-rtol", "1e-10", "-E", "2.1e5", "-nu", "0.3",
                "-ca", inp_file("CA_info.txt"), "-mesh-m", inp_file("mesh_m.inp"), "-nbasis", str(nb),
                "-o-ca", str(out_ca)]
        r = subprocess.run(args, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        lines = out_ca.read_text().split("\n")
        assert "POINTS\t525\tdouble" in lines and any(s_.startswith("CELLS\t1920") for s_ in lines)
        u = np.stack([np.array([float(x) for x in lines[lines.index(f"SCALARS {c} double 1") + 2:][:525]])
                      for c in ("u_x", "u_y", "u_z")], axis=1)
        assert np.all(np.isfinite(u))
        if nb == 1:
            assert np.linalg.norm(u - ug) / np.linalg.norm(ug) < 1e-5
