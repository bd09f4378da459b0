"""CPU restatement of the reference's combined-approximations reanalysis.

TEST INFRASTRUCTURE ONLY: imported by tests/, where it is the checker of
ofea_ca_reanalysis, never the product.

Follows src/ca_analysis.cpp:
* ΔK assembled element by element from the change list
  (ca_fill_CSR_sparse_mat, :52-145): a deleted element adds -Ke, a moved one
  Ke(new coordinates) - Ke(old), an added one +Ke;
* basis r_0 = u_0, r_i = -K0^-1 ΔK r_(i-1) with the kept factor of K0
  (ca_build_rom, :146-178);
* thin U of the basis' SVD (ca_SVD, :180-207; the reference runs it in
  FP32, here FP64);
* reduced system U^T K U y = U^T f with K = K0 + ΔK and the original load
  (ca_solve, :209-250; ca_reduced_K :262-283; ca_reduced_F :303-311),
  u = U y.

Parity: pinned by sample_model/CA/cadcae_ca.vtk, the reference's shipped CA
output.  Its driver solves the original model with "Pardiso_class"
(src/cae.cpp:274), so the SuperLU factor that ca_build_rom re-solves with is
never built and r_1.. stay zero: the shipped output is the Galerkin solution
on span(u_0), i.e. n_basis = 1 here.  Larger bases follow the same code with
the factor present ("SuperLU_class"), which the shipped driver never runs.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from openfea_b200 import meshgen as mg


def delta_k(oracle, ca_info, fix, free_map, n, E0, nu, xyz_old=None):
    """ΔK from the change list, element by element (ca_fill_CSR_sparse_mat):
    kind 0 (deleted) -Ke, 1 (moved) Ke(new) - Ke(old coordinates), 2 (added)
    +Ke, with the modified coordinates of ca_info['xyz']."""
    topo = np.where(ca_info["topo"] >= 0, ca_info["topo"] + 1, 0)  # 1-based, 0 padded
    kind = ca_info["kind"]
    sign = np.where(kind == 0, -1.0, 1.0)

    def K_of(xyz, sel, s):
        if not np.any(sel):
            return sp.csc_matrix((n, n))
        m = mg.Mesh(xyz, topo[sel], ca_info["etype"][sel], fix, E0 * s[sel], E0, nu)
        cp, ri, val = oracle.assemble(m, free_map)
        return sp.csc_matrix((val, ri, cp), shape=(n, n))

    dK = K_of(ca_info["xyz"], np.ones(kind.size, bool), sign)
    moved = kind == 1
    if np.any(moved):
        if xyz_old is None:
            raise ValueError("moved elements need the original coordinates")
        dK = dK - K_of(xyz_old, moved, np.ones(kind.size))
    return dK


def ca_reanalysis(K0, dK, f, u0, n_basis):
    """The CA solution from n_basis basis vectors (exact K0 solves)."""
    lu = spla.splu(sp.csc_matrix(K0))
    basis = [np.asarray(u0, dtype=np.float64)]
    for _ in range(1, n_basis):
        basis.append(-lu.solve(dK @ basis[-1]))
    V = np.stack(basis, axis=1)
    U, s, _ = np.linalg.svd(V, full_matrices=False)
    U = U[:, s > 1e-13 * s[0]]
    K = K0 + dK
    KR = U.T @ (K @ U)
    fR = U.T @ f
    return U @ np.linalg.solve(KR, fR)


def to_modified_nodes(u, free_map, node_map):
    """reset_ca_displacement (src/post_process.cpp:42-75): the free-DOF
    solution onto every original node (zeros on fixed ones), then onto the
    modified model's nodes through the node map (-1: removed)."""
    nd = free_map.size
    uf = np.zeros((nd, 3))
    fr = free_map >= 0
    uf[fr] = np.asarray(u).reshape(-1, 3)[free_map[fr]]
    keep = node_map >= 0
    out = np.zeros((int(node_map.max()) + 1, 3))
    out[node_map[keep]] = uf[keep]
    return out
