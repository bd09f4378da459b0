"""The oracle (oracle/ofea_oracle.c) pinned against the reference's own
results: element matrices from its element routines, K and SuperLU
displacements from its assembly + solution_api, its -nl Newton iterates and
the shipped golden output sample_model/CA/cadcae_o.vtk."""
import numpy as np
import pytest

from openfea_b200 import meshgen as mg


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def csc(cp, ri, val):
    import scipy.sparse as sp
    return sp.csc_matrix((val, ri, cp), shape=(cp.size - 1, cp.size - 1))


def direct_solve(cp, ri, val, f):
    """Sparse LU as a checker (scipy's SuperLU, the library family of the
    reference's SuperLU_func path)."""
    import scipy.sparse.linalg as spl
    return spl.spsolve(csc(cp, ri, val), f)


def test_element_matrices_match_reference_routines(oracle, golden):
    g = golden("ref_elements.npz")
    for k in range(4):
        for tag, et in (("hex", 1), ("tet", 0)):
            X, U, (E, nu) = g[f"{tag}{k}_X"], g[f"{tag}{k}_U"], g[f"{tag}{k}_mat"]
            K, _ = oracle.element_ke(et, X, E, nu)
            assert rel(K, g[f"{tag}{k}_K"]) < 1e-13
            KT, f = oracle.element_nl(et, X, U, E, nu)
            assert rel(KT, g[f"{tag}{k}_KT"]) < 1e-13
            assert rel(f, g[f"{tag}{k}_f"]) < 1e-12


def test_inverted_tet_keeps_signed_determinant(oracle, golden):
    g = golden("ref_elements.npz")
    K, det = oracle.element_ke(0, g["tetinv_X"], *g["tetinv_mat"])
    assert det < 0
    assert rel(K, g["tetinv_K"]) < 1e-14
    assert np.trace(K) < 0  # negative stiffness, no abs() (C3D4_hammer.cpp:70)


@pytest.mark.parametrize("et", [0, 1])
def test_element_rigid_body_modes_and_symmetry(oracle, et):
    rng = np.random.default_rng(3)
    X = (mg.HEX_SIGNS * 0.5 if et else np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]]))
    X = X + rng.uniform(-0.1, 0.1, X.shape)
    K, _ = oracle.element_ke(et, X, 210e9, 0.3)
    assert rel(K, K.T) < 1e-14
    npe = X.shape[0]
    modes = []
    for c in range(3):
        t = np.zeros((npe, 3)); t[:, c] = 1; modes.append(t.ravel())
    for axis in range(3):
        w = np.zeros(3); w[axis] = 1
        modes.append(np.cross(w, X).ravel())
    for m in modes:
        assert np.abs(K @ m).max() < 1e-9 * np.abs(K).max()


def test_tiny_models_K_and_u_match_reference(oracle, golden):
    g = golden("ref_models.npz")
    cases = {"hex_tiny": mg.structured_hex(4, 2, 2, 0.2, 0.1, 0.1, 210e9, 0.3),
             "tet_tiny": mg.tet_block(4, 2, 2)[0]}
    for tag, m in cases.items():
        fm = oracle.free_index(m.nd, m.fix)
        cp, ri, val = oracle.assemble(m, fm)
        assert np.array_equal(cp, g[f"{tag}_colptr"]) and np.array_equal(ri, g[f"{tag}_rowidx"])
        assert rel(val, g[f"{tag}_val"]) < 1e-13
        u, st, _, rr = oracle.pcg(cp, ri, val, g[f"{tag}_f"], rtol=1e-12)
        assert st == 0
        assert np.linalg.norm(u - g[f"{tag}_u"]) / np.linalg.norm(g[f"{tag}_u"]) < 1e-9


def test_cantilever_matches_reference_superlu(oracle, golden):
    g = golden("ref_models.npz")
    m, _ = mg.cantilever_small()
    fm = oracle.free_index(m.nd, m.fix)
    cp, ri, val = oracle.assemble(m, fm)
    assert val.size == int(g["cantilever_nnz"]) == 88218
    u, st, _, _ = oracle.pcg(cp, ri, val, g["cantilever_f"], rtol=1e-11)
    assert st == 0
    assert np.linalg.norm(u - g["cantilever_u"]) / np.linalg.norm(g["cantilever_u"]) < 1e-9


def test_golden_vtk_reproduced(oracle, golden, inp_file):
    """sample_model/CA/cadcae_o.vtk, written by the reference with E=2.1e5,
    nu=0.3 at 6 significant digits."""
    import openfea_b200 as ob
    d = ob.inp_read(inp_file("mesh_o.inp"))
    m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, 2.1e5, 0.3)
    fm = oracle.free_index(m.nd, m.fix)
    cp, ri, val = oracle.assemble(m, fm)
    f = ob.build_single_load(m.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
    u = direct_solve(cp, ri, val, f)
    uf = np.zeros(3 * m.nd)
    oracle.L.orc_full_displacement(m.nd, fm.ctypes.data, u.ctypes.data, uf.ctypes.data)
    ug = golden("cadcae_o_u.npz")["u"].ravel()
    assert np.linalg.norm(uf - ug) / np.linalg.norm(ug) < 3e-6  # print precision


def test_sample_models_match_reference_superlu(oracle, golden, inp_file):
    import openfea_b200 as ob
    g = golden("ref_models.npz")
    for name, E, nu in (("mesh_o", 2.1e5, 0.3), ("implicite_test_C3D4_C3D8", None, None)):
        d = ob.inp_read(inp_file(name + ".inp"))
        m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, E or d["E"], nu or d["nu"])
        fm = oracle.free_index(m.nd, m.fix)
        cp, ri, val = oracle.assemble(m, fm)
        assert val.size == int(g[f"{name}_nnz"])
        f = ob.build_single_load(m.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
        assert np.array_equal(f, g[f"{name}_f"])
        # the reference's SuperLU solution satisfies the oracle's K
        ur = g[f"{name}_u"]
        r = f - oracle.spmv(cp, ri, val, ur)
        assert np.linalg.norm(r) / np.linalg.norm(f) < 1e-9


def test_nl_newton_iterates_match_reference(oracle, golden, inp_file):
    """Newton iterates of the -nl path (src/cae.cpp:209-253) on nlcae.inp."""
    import openfea_b200 as ob
    g = golden("ref_models.npz")
    d = ob.inp_read(inp_file("nlcae.inp"))
    m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, d["E"], d["nu"])
    fm = oracle.free_index(m.nd, m.fix)
    cp, ri = oracle.pattern(m, fm)
    f = g["nlcae_f"]
    u = np.zeros(f.size)
    for it in range(3):
        # K_T(u_k) du = f - f_int(u_k) holds for the reference's own increment
        val, fint = oracle.nl_assemble(m, fm, cp, ri, u)
        un = g["nlcae_iterates"][it]
        b = f - fint
        r = b - oracle.spmv(cp, ri, val, un - u)
        assert np.linalg.norm(r) / np.linalg.norm(f) < 1e-9, it
        u = un


def test_oracle_against_live_reference(oracle, reference):
    """Where the reference build is present: pattern + values + NL on a
    per-element-modulus tet mesh and a mixed sample."""
    m, ffull = mg.tet_block(6, 3, 3)
    fm = oracle.free_index(m.nd, m.fix)
    cp, ri, val = oracle.assemble(m, fm)
    rcp, rri, rval = reference.model(m).assemble()
    assert np.array_equal(cp, rcp) and np.array_equal(ri, rri)
    assert rel(val, rval) < 1e-13
    rm = reference.model(m)
    rm.assemble()
    u = np.random.default_rng(1).normal(0, 1e-4, cp.size - 1)
    _, _, rv, rf = rm.nl_assemble(u)
    ov, of = oracle.nl_assemble(m, fm, cp, ri, u)
    assert rel(ov, rv) < 1e-13
    scale = np.abs(val).max() * np.abs(u).max()
    assert np.abs(of - rf).max() < 1e-12 * scale


def test_free_index_rejects_bad_sets(oracle):
    with pytest.raises(ValueError):
        oracle.free_index(10, [])
    with pytest.raises(ValueError):
        oracle.free_index(10, [3, 3])
    with pytest.raises(ValueError):
        oracle.free_index(10, [11])
    fm = oracle.free_index(6, [5, 2])
    assert fm.tolist() == [0, -1, 1, 2, -1, 3]
