"""Host side of the boundary, no GPU: the C-ABI library loads and exports
every symbol include/*.h declares; the .inp reader, DOF numbering, load
vector and VTK writer keep the reference's formats."""
import os
import re

import numpy as np
import pytest

import openfea_b200 as ob
from tests.conftest import ROOT, has_gpu


def declared_symbols():
    names = []
    for h in ("ofea_gpu.h", "ofea_host.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"OFEA_API\s+[\w\s\*]*?\b(ofea_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = ob.lib()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    assert b"sm_100a" in L.ofea_version()


def test_no_device_is_an_error_not_a_fallback():
    if has_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(ob.OfeaError) as e:
        ob.Context()
    assert e.value.code == -9


def test_reader_sample_models(inp_file):
    d = ob.inp_read(inp_file("mesh_o.inp"))
    assert d["xyz"].shape == (625, 3) and d["topo"].shape == (2304, 8)
    assert (d["etype"] == 0).all() and not d["has_elastic"]
    assert d["load_dof"] == 3 and d["load_value"] == -10.0
    assert d["fix"].tolist()[:3] == [202, 422, 342] and d["load_set"].size == 12
    d = ob.inp_read(inp_file("implicite_test_C3D4_C3D8.inp"))
    assert d["xyz"].shape[0] == 6318 and (d["etype"] == 1).sum() == 1328 and (d["etype"] == 0).sum() == 20413
    assert d["E"] == 2.1e9 and d["nu"] == 0.3 and d["density"] == 7800.0
    assert d["load_value"] == -100000.0
    d = ob.inp_read(inp_file("nlcae.inp"))
    assert d["E"] == 210000.0 and d["load_dof"] == 2


def test_reader_matches_reference_reader(reference, inp_file):
    for name in ("mesh_o.inp", "implicite_test_C3D4_C3D8.inp", "nlcae.inp"):
        d = ob.inp_read(inp_file(name))
        a = reference.model_from_inp(inp_file(name)).mesh_arrays()
        assert np.array_equal(d["xyz"], a["xyz"])
        assert np.array_equal(d["topo"], a["topo"]) and np.array_equal(d["etype"], a["etype"])
        fm = ob.build_free_index(d["xyz"].shape[0], d["fix"])
        assert np.array_equal(fm, a["free_map"])
        if d["has_elastic"]:
            assert d["E"] == a["E"] and d["nu"] == a["nu"]
        f = ob.build_single_load(fm.size, fm, d["load_set"], d["load_dof"], d["load_value"])
        assert np.array_equal(f, a["f"])


def test_reader_errors(tmp_path):
    with pytest.raises(ob.OfeaError) as e:
        ob.inp_read(tmp_path / "missing.inp")
    assert e.value.code == -10
    p = tmp_path / "bad.inp"
    p.write_text("*Node\n1, 0., 0., 0.\n*Element, type=C3D20\n1, 1, 1\n*End Assembly\n")
    with pytest.raises(ob.OfeaError):
        ob.inp_read(p)


def test_free_index_and_load(oracle):
    fix = np.array([9, 2, 5])
    fm = ob.build_free_index(10, fix)
    assert np.array_equal(fm, oracle.free_index(10, fix))
    for bad in ([], [2, 2], [0], [11]):
        with pytest.raises(ob.OfeaError):
            ob.build_free_index(10, np.array(bad, dtype=np.int32))
    f = ob.build_single_load(10, fm, [1, 2, 10], 2, -5.0)
    assert f.size == 21 and f[1] == -5.0 and f[3 * fm[9] + 1] == -5.0 and np.count_nonzero(f) == 2
    u = np.arange(21, dtype=float)
    uf = ob.full_displacement(10, fm, u)
    assert uf[3:6].tolist() == [0, 0, 0] and uf[0:3].tolist() == [0, 1, 2]


def test_vtk_writer_layout(tmp_path, golden, inp_file):
    """Same header, cell order/types and u fields as the reference's output."""
    d = ob.inp_read(inp_file("mesh_o.inp"))
    ug = golden("cadcae_o_u.npz")["u"].ravel()
    out = tmp_path / "o.vtk"
    ob.write_vtk(out, d["xyz"], d["topo"], d["etype"], ug)
    lines = out.read_text().split("\n")
    assert lines[:4] == ["# vtk DataFile Version 3.0", "The density field of the optimized results",
                         "ASCII", "DATASET UNSTRUCTURED_GRID"]
    assert lines[5] == "POINTS\t625\tdouble"
    i = lines.index("CELLS\t2304\t11520")
    t = d["topo"][0]
    assert lines[i + 1] == "\t".join(map(str, [4, t[0] - 1, t[2] - 1, t[1] - 1, t[3] - 1]))
    j = lines.index("SCALARS u_z double 1")
    uz = np.array([float(x) for x in lines[j + 2:j + 2 + 625]])
    assert np.allclose(uz, ug[2::3], rtol=1e-5, atol=0)
    # a hex mesh: VTK_VOXEL order (src/data2vtk.cpp:159-162)
    m = __import__("openfea_b200.meshgen", fromlist=["x"]).structured_hex(1, 1, 1, 1, 1, 1)
    ob.write_vtk(tmp_path / "h.vtk", m.xyz, m.topo, m.etype, np.zeros(24))
    L2 = (tmp_path / "h.vtk").read_text().split("\n")
    k = L2.index("CELLS\t1\t9")
    t = m.topo[0]
    assert L2[k + 1] == "\t".join(map(str, [8] + [t[a] - 1 for a in (0, 1, 3, 2, 4, 5, 7, 6)]))
    assert L2[L2.index("CELL_TYPES\t\t1") + 1] == "11"


def test_solution_api_binding_forwards_cpu_solvers(golden, inp_file, tmp_path):
    """The reference-side binding (openfea_b200/integration/ofea_solution_api.cpp)
    compiles against the reference's headers and, for the reference's own
    solver strings, hands the call to the reference's dispatch unchanged: the
    reference's flow through it with "SuperLU_func" writes the shipped
    cadcae_o.vtk displacement (6 printed digits).  No GPU is involved."""
    import subprocess
    drv = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_driver")
    if not os.path.exists(drv):
        pytest.skip("oracle/_ref/ref_gpu_driver not built (needs the reference tree)")
    out = tmp_path / "o.vtk"
    r = subprocess.run([drv, "-i", inp_file("mesh_o.inp"), "-o", str(out), "-solver", "SuperLU_func",
                        "-E", "2.1e5", "-nu", "0.3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = out.read_text().split("\n")
    ug = golden("cadcae_o_u.npz")["u"].reshape(-1, 3)
    for c, name in enumerate("xyz"):
        j = lines.index(f"SCALARS u_{name} double 1")
        v = np.array([float(x) for x in lines[j + 2:j + 2 + ug.shape[0]]])
        assert np.abs(v - ug[:, c]).max() <= 3e-6 * np.abs(ug).max()
    if not has_gpu():
        # a GPU solver string without a GPU fails with the library's status, no exit()
        r = subprocess.run([drv, "-i", inp_file("mesh_o.inp"), "-o", str(tmp_path / "g.vtk"), "-solver",
                            "GPU_PCG", "-E", "2.1e5", "-nu", "0.3"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 1 and "no CUDA device" in r.stderr
