"""Stress recovery on the CPU: the oracle's restatement of
get_cauchy_stress_3d (src/post_process.cpp:79-167) against the reference's
shipped S_* fields, and a patch test of the Cauchy mode."""
import dataclasses

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import openfea_b200 as ob
from openfea_b200 import meshgen as mg
from oracle import stress_oracle as so


def test_oracle_reproduces_shipped_stress_fields(oracle, golden, inp_file):
    """S_xx .. S_Mises of sample_model/CA/cadcae_o.vtk from a full-precision
    solution of the same model: the file's 6 printed digits."""
    d = ob.inp_read(inp_file("mesh_o.inp"))
    m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, 2.1e5, 0.3)
    fm = oracle.free_index(m.nd, m.fix)
    n = 3 * int((fm >= 0).sum())
    cp, ri, val = oracle.assemble(m, fm)
    f = ob.build_single_load(m.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
    u = spla.spsolve(sp.csc_matrix((val, ri, cp), shape=(n, n)), f)
    uf = ob.full_displacement(m.nd, fm, u).reshape(-1, 3)
    node = so.node_values(m, so.element_values(m, uf, "reference"))
    S = golden("cadcae_o_stress.npz")["S"]
    for k in range(7):
        assert np.linalg.norm(node[k] - S[k]) <= 5e-6 * np.linalg.norm(S[k]), k


def test_oracle_cauchy_patch_test():
    """u = x (a, b, c) on a C3D8 block and on a C3D4 block: every element
    carries the stress D eps of that uniform strain."""
    a, b, c = 1e-3, -2e-4, 5e-4
    eps = np.array([a, 0, 0, b, 0, c])
    for m in (mg.structured_hex(4, 2, 2, 0.2, 0.1, 0.1, 210e9, 0.3), mg.tet_block(4, 2, 2)[0]):
        m = dataclasses.replace(m, xyz=m.xyz + 0.01 * np.sin(7 * m.xyz))  # distorted elements
        uf = m.xyz[:, :1] * np.array([a, b, c])
        el = so.element_values(m, uf, "cauchy")
        E = np.full(m.ne, m.E0) if m.E is None else np.asarray(m.E)
        lam = (E * m.nu / ((1 + m.nu) * (1 - 2 * m.nu)))[:, None]
        mu = (E / (2 * (1 + m.nu)))[:, None]
        s = np.concatenate([lam * eps[:3].sum() + 2 * mu * eps[:3], mu * eps[3:]], axis=1)
        assert np.allclose(el[:, :6], s, rtol=1e-9, atol=1e-9 * np.abs(s).max())
        assert np.allclose(el[:, 6], so.mises(s.T), rtol=1e-9)
