"""Stress recovery on the device (ofea_stress) against the oracle's
restatement of get_cauchy_stress_3d and the reference's shipped S_* fields,
through the C ABI, the VTK writer and the command line."""
import dataclasses
import os
import subprocess

import numpy as np
import pytest

import openfea_b200 as ob
from openfea_b200 import meshgen as mg
from oracle import stress_oracle as so

pytestmark = pytest.mark.gpu


def solved(factory, m):
    c = factory()
    fm = c.upload_mesh(m)
    c.assemble_pattern()
    c.assemble_linear()
    return c, fm


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_stress_reproduces_shipped_fields(gpu_ctx_factory, golden, inp_file):
    d = ob.inp_read(inp_file("mesh_o.inp"))
    m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, 2.1e5, 0.3)
    c, fm = solved(gpu_ctx_factory, m)
    f = ob.build_single_load(m.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
    u, st = c.solve(f, rtol=1e-10)
    elem, node = c.stress(u, "reference")
    S = golden("cadcae_o_stress.npz")["S"]
    for k in range(7):
        assert rel(node[k], S[k]) <= 5e-6, k  # the file's 6 printed digits
    uf = ob.full_displacement(m.nd, fm, u).reshape(-1, 3)
    ref_el = so.element_values(m, uf, "reference")
    assert rel(elem, ref_el) <= 1e-12
    assert rel(node, so.node_values(m, ref_el)) <= 1e-12


@pytest.mark.parametrize("mode", ["reference", "cauchy"])
def test_stress_mixed_mesh_matches_oracle(gpu_ctx_factory, inp_file, mode):
    """C3D4 + C3D8 sample: element values in caller order and node means."""
    d = ob.inp_read(inp_file("implicite_test_C3D4_C3D8.inp"))
    m = mg.Mesh(d["xyz"], d["topo"], d["etype"], d["fix"], None, d["E"], d["nu"])
    c, fm = solved(gpu_ctx_factory, m)
    f = ob.build_single_load(m.nd, fm, d["load_set"], d["load_dof"], d["load_value"])
    u, _ = c.solve(f, rtol=1e-10)
    elem, node = c.stress(u, mode)
    uf = ob.full_displacement(m.nd, fm, u).reshape(-1, 3)
    ref_el = so.element_values(m, uf, mode)
    assert rel(elem, ref_el) <= 1e-11
    assert rel(node, so.node_values(m, ref_el)) <= 1e-11
    if mode == "reference":
        assert np.all(elem[m.etype == 1] == 0.0)  # the reference computes nothing for C3D8


def test_stress_cauchy_patch_test_on_device(gpu_ctx_factory):
    """u = x (a, b, c) on a distorted C3D8 cantilever (zero on the clamped
    face x = 0): every element carries D eps of that uniform strain."""
    m, _ = mg.cantilever_small()
    m = dataclasses.replace(m, xyz=m.xyz + 0.004 * np.sin(9 * m.xyz) * (m.xyz[:, :1] > 0))
    c, fm = solved(gpu_ctx_factory, m)
    a, b, cc = 1e-3, -2e-4, 5e-4
    uf = m.xyz[:, :1] * np.array([a, b, cc])
    u = np.zeros(c.n)
    fr = fm >= 0
    u.reshape(-1, 3)[fm[fr]] = uf[fr]
    elem, _ = c.stress(u, "cauchy")
    eps = np.array([a, 0, 0, b, 0, cc])
    lam = m.E0 * m.nu / ((1 + m.nu) * (1 - 2 * m.nu))
    mu = m.E0 / (2 * (1 + m.nu))
    s = np.concatenate([lam * eps[:3].sum() + 2 * mu * eps[:3], mu * eps[3:]])
    assert np.allclose(elem[:, :6], s, rtol=1e-9, atol=1e-9 * np.abs(s).max())


def test_stress_rejects_bad_mode(gpu_ctx_factory):
    m, _ = mg.cantilever_small()
    c, _ = solved(gpu_ctx_factory, m)
    rc = ob.lib().ofea_stress(c.h, np.zeros(c.n).ctypes.data, 5, None, None)
    assert rc == -1


def test_cli_writes_the_reference_stress_fields(golden, inp_file, tmp_path):
    cli = os.path.join(os.path.dirname(ob.__file__), "ofea_cli")
    out = tmp_path / "o.vtk"
    r = subprocess.run([cli, "-i", inp_file("mesh_o.inp"), "-o", str(out), "-rtol", "1e-10", "-E", "2.1e5",
                        "-nu", "0.3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = out.read_text().split("\n")
    S = golden("cadcae_o_stress.npz")["S"]
    for k, name in enumerate(["S_xx", "S_yy", "S_zz", "S_xy", "S_yz", "S_xz", "S_Mises"]):
        j = lines.index(f"SCALARS {name} double 1")
        assert lines[j + 1] == f"LOOKUP_TABLE  table{k + 5}"
        v = np.array([float(x) for x in lines[j + 2:j + 2 + 625]])
        assert rel(v, S[k]) <= 5e-6, name
