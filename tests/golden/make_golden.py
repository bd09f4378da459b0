"""Generate the golden fixtures under tests/golden/ from the reference.

Run where the reference tree and oracle/_ref/libofea_ref.so (make -C oracle)
exist:

    python tests/golden/make_golden.py <reference tree>   (or OFEA_REFERENCE_DIR)

Writes:
  *.inp.gz              the reference's sample models used as test inputs
                        (sample_model/CA/mesh_o.inp, sample_model/L_NL/nlcae.inp,
                        sample_model/test/implicite_test_C3D4_C3D8.inp)
  cadcae_o_u.npz        u_x, u_y, u_z of the reference's shipped output
                        sample_model/CA/cadcae_o.vtk (E = 2.1e5, nu = 0.3)
  CA_info.txt.gz        the CA change file of that sample (384 deleted C3D4)
  mesh_m.inp.gz         the sample's modified mesh (525 nodes, 1,920 C3D4)
  cadcae_o_stress.npz   S_xx .. S_Mises of the shipped sample_model/CA/cadcae_o.vtk
                        (the reference's nodal stress recovery, 625 nodes)
  cadcae_ca_u.npz       u_x, u_y, u_z of the shipped CA reanalysis output
                        sample_model/CA/cadcae_ca.vtk (525 nodes of the
                        modified model)

    python tests/golden/make_golden.py --ca-only <reference tree>

writes only the sample_model/CA fixtures (no oracle/_ref needed).
  ref_elements.npz      element matrices from the reference's element routines
  ref_models.npz        K (CSC) and SuperLU displacements from the reference's
                        own build_CSR / fill_CSR_sparse_mat / solution_api
                        ("SuperLU_func") on small models, and the Newton
                        iterates of its -nl path on nlcae.inp
"""
from __future__ import annotations

import gzip
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402
from openfea_b200 import meshgen as mg  # noqa: E402

SAMPLES = {
    "mesh_o.inp": "sample_model/CA/mesh_o.inp",
    "nlcae.inp": "sample_model/L_NL/nlcae.inp",
    "implicite_test_C3D4_C3D8.inp": "sample_model/test/implicite_test_C3D4_C3D8.inp",
}


def vtk_displacement(path, nd):
    lines = open(path).read().split("\n")
    out = []
    for name in ("u_x", "u_y", "u_z"):
        i = [k for k, s in enumerate(lines) if s.startswith("SCALARS " + name)][0]
        out.append(np.array([float(x) for x in lines[i + 2:i + 2 + nd]]))
    return np.stack(out, axis=1)


def vtk_fields(path, names, nd):
    lines = open(path).read().split("\n")
    out = []
    for name in names:
        i = [k for k, s in enumerate(lines) if s.startswith("SCALARS " + name + " ")][0]
        out.append(np.array([float(x) for x in lines[i + 2:i + 2 + nd]]))
    return np.stack(out)


def ca_fixtures(ref_root):
    S = vtk_fields(os.path.join(ref_root, "sample_model/CA/cadcae_o.vtk"),
                   ["S_xx", "S_yy", "S_zz", "S_xy", "S_yz", "S_xz", "S_Mises"], 625)
    np.savez_compressed(os.path.join(HERE, "cadcae_o_stress.npz"), S=S, E=2.1e5, nu=0.3)
    with open(os.path.join(ref_root, "sample_model/CA/CA_info.txt"), "rb") as fi, \
            gzip.GzipFile(os.path.join(HERE, "CA_info.txt.gz"), "wb", mtime=0) as fo:
        shutil.copyfileobj(fi, fo)
    with open(os.path.join(ref_root, "sample_model/CA/mesh_m.inp"), "rb") as fi, \
            gzip.GzipFile(os.path.join(HERE, "mesh_m.inp.gz"), "wb", mtime=0) as fo:
        shutil.copyfileobj(fi, fo)
    u = vtk_displacement(os.path.join(ref_root, "sample_model/CA/cadcae_ca.vtk"), 525)
    np.savez_compressed(os.path.join(HERE, "cadcae_ca_u.npz"), u=u, E=2.1e5, nu=0.3, n_basis=4)


def main(ref_root):
    ca_fixtures(ref_root)
    R = Reference()
    for name, rel in SAMPLES.items():
        with open(os.path.join(ref_root, rel), "rb") as fi, gzip.open(os.path.join(HERE, name + ".gz"), "wb") as fo:
            shutil.copyfileobj(fi, fo)
    u = vtk_displacement(os.path.join(ref_root, "sample_model/CA/cadcae_o.vtk"), 625)
    np.savez_compressed(os.path.join(HERE, "cadcae_o_u.npz"), u=u, E=2.1e5, nu=0.3)

    # element matrices (reference routines) on seeded distorted elements
    rng = np.random.default_rng(7)
    ele = {}
    for k in range(4):
        X8 = mg.HEX_SIGNS * 0.5 * (1 + 0.3 * k) + rng.uniform(-0.12, 0.12, (8, 3))
        X4 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]]) * (1 + k) + rng.uniform(-0.1, 0.1, (4, 3))
        E = float(rng.uniform(1e5, 3e11))
        nu = float(rng.uniform(0.1, 0.45))
        U8 = rng.normal(0, 0.03, (3, 8))
        U4 = rng.normal(0, 0.03, (3, 4))
        ele[f"hex{k}_X"], ele[f"hex{k}_U"], ele[f"hex{k}_mat"] = X8, U8, np.array([E, nu])
        ele[f"hex{k}_K"] = R.element_ke(1, X8, E, nu)
        ele[f"hex{k}_KT"], ele[f"hex{k}_f"] = R.element_nl(1, X8, U8, E, nu)
        ele[f"tet{k}_X"], ele[f"tet{k}_U"], ele[f"tet{k}_mat"] = X4, U4, np.array([E, nu])
        ele[f"tet{k}_K"] = R.element_ke(0, X4, E, nu)
        ele[f"tet{k}_KT"], ele[f"tet{k}_f"] = R.element_nl(0, X4, U4, E, nu)
    # an inverted tet: the reference keeps the signed determinant
    Xi = np.array([[0, 0, 0], [0, 1, 0], [1, 0, 0], [0, 0, 1.0]])
    ele["tetinv_X"], ele["tetinv_mat"] = Xi, np.array([2.1e5, 0.3])
    ele["tetinv_K"] = R.element_ke(0, Xi, 2.1e5, 0.3)
    np.savez_compressed(os.path.join(HERE, "ref_elements.npz"), **ele)

    models = {}
    # tiny meshes: full K
    for tag, (m, ffull) in {"hex_tiny": mg.cantilever_small(), "tet_tiny": mg.tet_block(4, 2, 2)}.items():
        if tag == "hex_tiny":
            m = mg.structured_hex(4, 2, 2, 0.2, 0.1, 0.1, 210e9, 0.3)
            ffull = mg.end_traction_loads(m, -1e6)
        fm = mg.free_map(m.nd, m.fix)
        rm = R.model(m)
        cp, ri, val = rm.assemble()
        f = mg.to_free(ffull, fm)
        rm.set_load(f)
        models[f"{tag}_colptr"], models[f"{tag}_rowidx"], models[f"{tag}_val"] = cp, ri, val
        models[f"{tag}_f"], models[f"{tag}_u"] = f, rm.solve()
    # the 20x4x4 C3D8 cantilever: displacement only
    m, ffull = mg.cantilever_small()
    fm = mg.free_map(m.nd, m.fix)
    rm = R.model(m)
    _, _, val = rm.assemble()
    f = mg.to_free(ffull, fm)
    rm.set_load(f)
    models["cantilever_f"], models["cantilever_u"] = f, rm.solve()
    models["cantilever_nnz"] = val.size
    # sample models through the reference reader + SuperLU
    for name, E, nu in (("mesh_o.inp", 2.1e5, 0.3), ("implicite_test_C3D4_C3D8.inp", None, None)):
        rm = R.model_from_inp(os.path.join(ref_root, SAMPLES[name]), E, nu)
        _, _, val = rm.assemble()
        tag = name.split(".")[0]
        models[f"{tag}_u"] = rm.solve()
        models[f"{tag}_f"] = rm.mesh_arrays()["f"]
        models[f"{tag}_nnz"] = val.size
        models[f"{tag}_Kdiag_sum"] = float(np.sum(np.abs(val)))
    # -nl Newton iterates on nlcae.inp (implict_analysis, src/cae.cpp:209-253) with SuperLU
    rm = R.model_from_inp(os.path.join(ref_root, SAMPLES["nlcae.inp"]))
    f = rm.mesh_arrays()["f"]
    u = np.zeros(rm.n)
    its = []
    for it in range(3):
        _, _, _, fint = rm.nl_assemble(u)
        r = f - fint
        du = rm.nl_solve(r)
        u = u + du
        its.append(u.copy())
    models["nlcae_iterates"] = np.array(its)
    models["nlcae_f"] = f
    np.savez_compressed(os.path.join(HERE, "ref_models.npz"), **models)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if a != "--ca-only"]
    root = args[0] if args else os.environ.get("OFEA_REFERENCE_DIR")
    if not root:
        sys.exit("usage: make_golden.py [--ca-only] <reference tree>  (or set OFEA_REFERENCE_DIR)")
    if "--ca-only" in sys.argv:
        ca_fixtures(root)
    else:
        main(root)
