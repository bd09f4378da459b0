"""Seeded synthetic meshes, materials and loads for the implicit-static workloads.

All arrays use the reference's conventions so they can be handed to the
reference reader/assembler and to this library alike:

* ``xyz``   float64 (nd, 3) node coordinates;
* ``topo``  int32 (ne, 8) 1-based node ids, C3D4 elements use the first 4
  slots (``data_management::node_topos_``, src/include/data_management.h:49);
* ``etype`` int32 (ne,), 0 = C3D4, 1 = C3D8 (``ELE_TYPES``,
  src/include/data_management.h:76);
* ``fix``   int32 1-based fixed node ids (whole-node ENCASTRE, ``Set-fix``);
* C3D8 node order is the reference's (src/Elements/C3D8_Gauss.cpp:27-52):
  nodes 1-4 counter-clockwise on the face t = -1, nodes 5-8 above them.

Node numbering is x-slowest, z-fastest, so a structured block's nodes at x = 0
come first and the matrix bandwidth is set by the (y, z) cross-section.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# Corner signs (r, s, t) of the reference's 8-node brick.
HEX_SIGNS = np.array(
    [[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
     [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.int64)


@dataclass
class Mesh:
    xyz: np.ndarray
    topo: np.ndarray
    etype: np.ndarray
    fix: np.ndarray
    E: np.ndarray | None = None       # per-element Young's modulus or None
    E0: float = 210e9
    nu: float = 0.3
    shape: tuple = ()
    info: dict = field(default_factory=dict)

    @property
    def nd(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def ne(self) -> int:
        return int(self.topo.shape[0])


def _node_id(i, j, k, ny, nz):
    return (i * (ny + 1) + j) * (nz + 1) + k


def grid_nodes(nx, ny, nz, lx, ly, lz):
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    xyz = np.stack([i * (lx / nx), j * (ly / ny), k * (lz / nz)], axis=-1).reshape(-1, 3)
    return xyz.astype(np.float64)


def structured_hex(nx, ny, nz, lx, ly, lz, E0=210e9, nu=0.3) -> Mesh:
    """nx*ny*nz C3D8 block over [0,lx]x[0,ly]x[0,lz], clamped at x = 0."""
    xyz = grid_nodes(nx, ny, nz, lx, ly, lz)
    ei, ej, ek = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ei, ej, ek = ei.ravel(), ej.ravel(), ek.ravel()
    topo = np.zeros((ei.size, 8), dtype=np.int32)
    for a, (sr, ss, st) in enumerate(HEX_SIGNS):
        topo[:, a] = _node_id(ei + (sr > 0), ej + (ss > 0), ek + (st > 0), ny, nz) + 1
    etype = np.ones(ei.size, dtype=np.int32)
    fix = (np.arange((ny + 1) * (nz + 1)) + 1).astype(np.int32)  # the x = 0 face
    return Mesh(xyz, topo, etype, fix, None, E0, nu, (nx, ny, nz),
                {"kind": "hex", "lx": lx, "ly": ly, "lz": lz})


# Kuhn subdivision of the unit cube into 6 tetrahedra sharing the diagonal
# (0,0,0)-(1,1,1): one tet per permutation of the axes.
_PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def kuhn_tets(nx, ny, nz, h=1.0, jitter=0.0, seed=1, E0=70e9, nu=0.33) -> Mesh:
    """nx*ny*nz cubes of size h, 6 C3D4 each, clamped at z = 0.

    Interior nodes are moved by U(-jitter*h, +jitter*h) per coordinate (faces
    stay planar).  Every tet is oriented with a positive Jacobian determinant.
    """
    xyz = grid_nodes(nx, ny, nz, nx * h, ny * h, nz * h)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter * h, jitter * h, size=xyz.shape)
        n = np.array([nx, ny, nz], dtype=np.float64) * h
        interior = np.all((xyz > 1e-9 * h) & (xyz < n - 1e-9 * h), axis=1)
        xyz[interior] += d[interior]
    ei, ej, ek = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = np.stack([ei.ravel(), ej.ravel(), ek.ravel()], axis=1)
    tets = []
    for p in _PERMS:
        v = [base.copy()]
        cur = base.copy()
        for ax in p:
            cur = cur.copy()
            cur[:, ax] += 1
            v.append(cur)
        ids = [(_node_id(q[:, 0], q[:, 1], q[:, 2], ny, nz) + 1) for q in v]
        tets.append(np.stack(ids, axis=1))
    t4 = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int32)
    # orient: det([x1-x0, x2-x0, x3-x0]) > 0, else swap nodes 1 and 2
    X = xyz[t4 - 1]
    det = np.linalg.det(np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=1))
    neg = det < 0
    t4[neg, 1], t4[neg, 2] = t4[neg, 2].copy(), t4[neg, 1].copy()
    topo = np.zeros((t4.shape[0], 8), dtype=np.int32)
    topo[:, :4] = t4
    etype = np.zeros(t4.shape[0], dtype=np.int32)
    k = np.arange(xyz.shape[0]) % (nz + 1)
    fix = (np.nonzero(k == 0)[0] + 1).astype(np.int32)  # the z = 0 face
    return Mesh(xyz, topo, etype, fix, None, E0, nu, (nx, ny, nz),
                {"kind": "tet", "h": h, "jitter": jitter})


def free_map(nd: int, fix: np.ndarray) -> np.ndarray:
    """resort_free_nodes_ (src/set_bc.cpp:20-43) for a duplicate-free fixed set."""
    fm = np.zeros(nd, dtype=np.int32)
    fixed = np.zeros(nd, dtype=bool)
    fixed[np.asarray(fix, dtype=np.int64) - 1] = True
    fm[fixed] = -1
    fm[~fixed] = np.arange(int((~fixed).sum()), dtype=np.int32)
    return fm


def end_traction_loads(mesh: Mesh, traction: float, axis: int = 2) -> np.ndarray:
    """Consistent bilinear nodal forces of a uniform traction on the x = L face
    of a structured hex block, on the full 3*nd DOF vector."""
    nx, ny, nz = mesh.shape
    ly, lz = mesh.info["ly"], mesh.info["lz"]
    area = (ly / ny) * (lz / nz)
    w = np.zeros((ny + 1, nz + 1))
    w[:-1, :-1] += 0.25
    w[1:, :-1] += 0.25
    w[:-1, 1:] += 0.25
    w[1:, 1:] += 0.25
    f = np.zeros(3 * mesh.nd)
    j, k = np.meshgrid(np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    nodes = _node_id(nx, j, k, ny, nz)
    f[3 * nodes.ravel() + axis] = traction * area * w.ravel()
    return f


def to_free(f_full: np.ndarray, fm: np.ndarray) -> np.ndarray:
    """Restrict a full 3*nd vector to the free DOFs 3*fm[node]+c."""
    n = 3 * int((fm >= 0).sum())
    f = np.zeros(n)
    nodes = np.nonzero(fm >= 0)[0]
    for c in range(3):
        f[3 * fm[nodes] + c] = f_full[3 * nodes + c]
    return f


def face_nodes_x(mesh: Mesh, i: int) -> np.ndarray:
    nx, ny, nz = mesh.shape
    j, k = np.meshgrid(np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    return _node_id(i, j, k, ny, nz).ravel()


# ----------------------------------------------------------------- workloads --

def cantilever_small() -> tuple[Mesh, np.ndarray]:
    """C3D8 20x4x4 over 1.0x0.2x0.2 m, E = 210 GPa, nu = 0.3, clamped at x = 0,
    1 MPa traction in -z on x = L as consistent nodal loads (40 kN total)."""
    m = structured_hex(20, 4, 4, 1.0, 0.2, 0.2, 210e9, 0.3)
    return m, end_traction_loads(m, -1e6)


def tet_block(nx=60, ny=20, nz=20, seed_mesh=1, seed_E=2, seed_load=3) -> tuple[Mesh, np.ndarray]:
    """nx*ny*nz unit cubes x 6 C3D4, jitter +-0.15 h, E_e = 70 GPa*exp(0.5 z),
    z ~ N(0,1), nu = 0.33, clamped at z = 0, N(0, (1 kN)^2) nodal forces per
    component on the top face."""
    m = kuhn_tets(nx, ny, nz, 1.0, 0.15, seed_mesh, 70e9, 0.33)
    rng = np.random.default_rng(seed_E)
    m.E = 70e9 * np.exp(0.5 * rng.standard_normal(m.ne))
    rng = np.random.default_rng(seed_load)
    top = np.nonzero(np.arange(m.nd) % (nz + 1) == nz)[0]
    f = np.zeros(3 * m.nd)
    f.reshape(-1, 3)[top] = rng.normal(0.0, 1e3, size=(top.size, 3))
    return m, f


def cantilever_large(nx=200, ny=50, nz=50) -> tuple[Mesh, np.ndarray]:
    """C3D8 200x50x50 over 1.0x0.25x0.25 m (h = 5 mm), E = 210 GPa, nu = 0.3,
    clamped at x = 0, 1 MPa end traction in -z."""
    m = structured_hex(nx, ny, nz, nx * 0.005, ny * 0.005, nz * 0.005, 210e9, 0.3)
    return m, end_traction_loads(m, -1e6)


def simp_density(shape, seed, smooth=False) -> np.ndarray:
    """Per-element density rho ~ U[0.1, 1] (x-slowest element order), optionally
    smoothed by a 3x3x3 box filter (edges clamped)."""
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.1, 1.0, size=shape)
    if smooth:
        p = np.pad(rho, 1, mode="edge")
        acc = np.zeros_like(rho)
        for di in range(3):
            for dj in range(3):
                for dk in range(3):
                    acc += p[di:di + shape[0], dj:dj + shape[1], dk:dk + shape[2]]
        rho = acc / 27.0
    return rho.ravel()


def design_variants(count=64, seed_len=4, seed_rho=5, seed_load=6, nrhs=16, ny=20, nz=20,
                    h=0.005, nmin=20, nmax=60):
    """Batched-reanalysis workload: `count` C3D8 blocks n x ny x nz, n ~ U{nmin..nmax},
    SIMP stiffness E = 210 GPa * rho^3 with rho ~ U[0.1, 1], clamped at x = 0,
    `nrhs` load cases of N(0, (1 kN)^2) nodal forces on the x = L face."""
    rng = np.random.default_rng(seed_len)
    lens = rng.integers(nmin, nmax + 1, size=count)
    rrho = np.random.default_rng(seed_rho)
    rload = np.random.default_rng(seed_load)
    out = []
    for n in lens:
        m = structured_hex(int(n), ny, nz, n * h, ny * h, nz * h, 210e9, 0.3)
        m.E = 210e9 * rrho.uniform(0.1, 1.0, size=m.ne) ** 3
        face = face_nodes_x(m, int(n))
        F = np.zeros((nrhs, 3 * m.nd))
        for r in range(nrhs):
            F[r].reshape(-1, 3)[face] = rload.normal(0.0, 1e3, size=(face.size, 3))
        out.append((m, F))
    return out
