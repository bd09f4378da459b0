"""CPU restatement of the reference's stress recovery.

TEST INFRASTRUCTURE ONLY: imported by tests/, where it is the checker of
ofea_stress, never the product.

Follows simulation_post::get_cauchy_stress_3d (src/post_process.cpp:79-167):
per element six components (xx yy zz xy yz xz) and the von Mises
expression of :103-109 applied to them, then per node the sum over the
elements that use it, in element order, divided by their count.

* mode "reference": what the reference computes.  For C3D4 its
  get_stress_node_hammer (src/Elements/C3D4_hammer.cpp:185-226) returns the
  engineering strain B u (the D product is commented out), B from
  dN/dxyz = J^-1 dN/drst with J = dN/drst X and the rows of
  build_strain_node_mat_hammer.  C3D8 has no get_stress_node (the base-class
  stub of src/Elements/include/ele_base.h:66 leaves the values unset); zero
  here.
* mode "cauchy": D B u with the isotropic D of build_cons_mat; for C3D8 the
  mean over the 8 Gauss points at +-1/sqrt(3) (node order of
  src/Elements/C3D8_Gauss.cpp:27-52).

Parity: pinned by the S_xx .. S_Mises fields of the reference's shipped
sample_model/CA/cadcae_o.vtk (all C3D4, mode "reference").
"""
from __future__ import annotations

import numpy as np

_TET_DN = np.array([[-1.0, 1.0, 0.0, 0.0], [-1.0, 0.0, 1.0, 0.0], [-1.0, 0.0, 0.0, 1.0]])
_SR = np.array([-1, 1, 1, -1, -1, 1, 1, -1], dtype=float)
_SS = np.array([-1, -1, 1, 1, -1, -1, 1, 1], dtype=float)
_ST = np.array([-1, -1, -1, -1, 1, 1, 1, 1], dtype=float)


def _hex_dn(r, s, t):
    return 0.125 * np.stack([_SR * (1 + _SS * s) * (1 + _ST * t),
                             _SS * (1 + _SR * r) * (1 + _ST * t),
                             _ST * (1 + _SR * r) * (1 + _SS * s)])


def _strain(dn_dxyz, U):
    """Rows of build_strain_node_mat_hammer times u: xx yy zz, then the
    engineering shears xy, yz, xz."""
    g, u = dn_dxyz, U
    return np.array([g[0] @ u[:, 0], g[1] @ u[:, 1], g[2] @ u[:, 2],
                     g[1] @ u[:, 0] + g[0] @ u[:, 1],
                     g[2] @ u[:, 1] + g[1] @ u[:, 2],
                     g[2] @ u[:, 0] + g[0] @ u[:, 2]])


def _d_times(eps, E, nu):
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    tr = eps[0] + eps[1] + eps[2]
    return np.concatenate([lam * tr + 2 * mu * eps[:3], mu * eps[3:]])


def mises(s):
    return np.sqrt(0.5 * ((s[0] - s[1]) ** 2 + (s[1] - s[2]) ** 2 + (s[2] - s[0]) ** 2
                          + 6.0 * (s[3] ** 2 + s[4] ** 2 + s[5] ** 2)))


def element_values(mesh, u_full, mode="reference"):
    """(ne, 7) per element; u_full (nd, 3) on every node (zeros on fixed ones)."""
    xyz = np.asarray(mesh.xyz, dtype=float)
    U = np.asarray(u_full, dtype=float).reshape(-1, 3)
    E = np.full(mesh.ne, mesh.E0) if mesh.E is None else np.asarray(mesh.E, dtype=float)
    out = np.zeros((mesh.ne, 7))
    g = 1.0 / np.sqrt(3.0)
    for e in range(mesh.ne):
        t = np.asarray(mesh.topo[e])
        if mesh.etype[e] == 0:
            nodes = t[:4] - 1
            X, Ue = xyz[nodes], U[nodes]
            J = _TET_DN @ X
            eps = _strain(np.linalg.inv(J) @ _TET_DN, Ue)
            s = eps if mode == "reference" else _d_times(eps, E[e], mesh.nu)
        else:
            s = np.zeros(6)
            if mode == "cauchy":
                nodes = t[:8] - 1
                X, Ue = xyz[nodes], U[nodes]
                for q in range(8):
                    dn = _hex_dn(_SR[q] * g, _SS[q] * g, _ST[q] * g)
                    J = dn @ X
                    s += 0.125 * _d_times(_strain(np.linalg.inv(J) @ dn, Ue), E[e], mesh.nu)
        out[e, :6] = s
        out[e, 6] = mises(s) if (mesh.etype[e] == 0 or mode == "cauchy") else 0.0
    return out


def node_values(mesh, elem):
    """(7, nd): the element values summed per node in element order, divided
    by the node's element count (nodes on no element: 0)."""
    node = np.zeros((7, mesh.nd))
    cnt = np.zeros(mesh.nd)
    for e in range(mesh.ne):
        t = np.asarray(mesh.topo[e])
        for n in t[: (8 if mesh.etype[e] == 1 else 4)] - 1:
            node[:, n] += elem[e]
            cnt[n] += 1
    nz = cnt > 0
    node[:, nz] /= cnt[nz]
    return node
