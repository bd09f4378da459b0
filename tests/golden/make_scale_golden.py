"""Generate the full-size parity fixtures under tests/golden/ from the
reference's own code (oracle/_ref/libofea_ref.so, built by `make -C oracle
REF=<reference tree>`).  Test infrastructure only.

    python tests/golden/make_scale_golden.py [tet] [cantilever] [simp] [--threads N]

Writes:
  scale_tet_60x20x20.npz      the jittered C3D4 block (60x20x20 cubes x 6 tets,
                              76,860 DOF, lognormal E, random top-face loads):
                              the reference's build_CSR + per-element fill +
                              solution_api("SuperLU_func") displacement, all
                              76,860 values, and the reference's timings
  scale_cantilever_200x50x50.npz
                              the C3D8 cantilever (1,560,600 DOF, 122.7M
                              non-zeros): the reference-assembled K solved by the
                              vendored Eigen ConjugateGradient + IncompleteCholesky
                              in FP64 to a true relative residual near 1e-12
                              (a direct factor is out of reach at this size)
  scale_simp_200x50x50.npz    the same mesh with the SIMP density field of
                              seed 12 (rho ~ U[0.1,1], 3x3x3 box filter, E = 210
                              GPa rho^3), same oracle

The 1.56M-DOF fixtures keep the displacement on a sub-grid of nodes (every 5th
node along each axis: 14,520 values) plus whole-vector checks (2-norm, sum, and
dot products with seeded Gaussian vectors w_k = default_rng(100 + k)), so the
file stays small; the relative L2 error on the sub-grid estimates the
whole-field error.  They also keep the oracle's iteration count to relative
residual 1e-8 and the timings of the reference's assembly, IC set-up and CG.
"""
from __future__ import annotations

import os
import platform
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

N_PROJ = 4


def projections(u):
    return np.array([float(np.random.default_rng(100 + k).standard_normal(u.size) @ u) for k in range(N_PROJ)])


def subgrid_dofs(shape, fm, step=5):
    """Free DOFs of the nodes (i, j, k) with i, j, k multiples of `step`."""
    nx, ny, nz = shape
    i, j, k = np.meshgrid(np.arange(0, nx + 1, step), np.arange(0, ny + 1, step),
                          np.arange(0, nz + 1, step), indexing="ij")
    nodes = ((i * (ny + 1) + j) * (nz + 1) + k).ravel()
    nodes = nodes[fm[nodes] >= 0]
    return (3 * fm[nodes][:, None] + np.arange(3)[None, :]).ravel().astype(np.int64)


def cpu_name():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor()


def tet(R):
    from openfea_b200 import meshgen as mg
    m, ff = mg.tet_block()
    fm = mg.free_map(m.nd, m.fix)
    f = mg.to_free(ff, fm)
    rm = R.model(m)
    cp, ri, val = rm.assemble()
    rm.set_load(f)
    t0 = time.perf_counter()
    u = rm.solve()
    t_solve = time.perf_counter() - t0
    t = rm.times()
    r = f - (np.bincount(ri, weights=val * np.repeat(u, np.diff(cp)), minlength=rm.n))
    rel = float(np.linalg.norm(r) / np.linalg.norm(f))
    out = os.path.join(HERE, "scale_tet_60x20x20.npz")
    np.savez_compressed(out, u=u, n=rm.n, nnz=val.size, rel_residual=rel, build_csr_s=t["build_csr"],
                        fill_s=t["fill"], superlu_s=t_solve, cpu=cpu_name(),
                        oracle="reference build_CSR + per-element fill + solution_api(SuperLU_func)")
    print(f"tet: n={rm.n} nnz={val.size} SuperLU {t_solve:.1f} s, rel. residual {rel:.2e} -> {out}", flush=True)


def cantilever(R, name, E, threads):
    from openfea_b200 import meshgen as mg
    shape = (200, 50, 50)
    m, ff = mg.cantilever_large(*shape)
    m.E = E
    fm = mg.free_map(m.nd, m.fix)
    f = mg.to_free(ff, fm)
    rm = R.model(m)
    t0 = time.perf_counter()
    cp, ri, val = rm.assemble()
    t_asm = time.perf_counter() - t0
    t = rm.times()
    del cp, ri, val
    print(f"{name}: assembled n={rm.n} in {t_asm:.1f} s ({t})", flush=True)
    _, s8 = rm.cg_ic(f, rtol=1e-8, threads=threads)
    print(f"{name}: to 1e-8: {s8}", flush=True)
    # CG's recursive residual drifts from the true one (about 2e-10 at this
    # size), so restart from the current u on the true residual while that
    # keeps falling (each restart redoes the IC set-up); it levels off near
    # 2e-11, the rounding floor of f - K u in FP64 for these matrices
    u, last = None, np.inf
    for _ in range(6):
        u, st = rm.cg_ic(f, rtol=1e-12, max_iter=200000, threads=threads, u0=u)
        print(f"{name}: to 1e-12: {st}", flush=True)
        if st["rel_residual"] <= 2e-12 or st["rel_residual"] > 0.5 * last:
            break
        last = st["rel_residual"]
    idx = subgrid_dofs(shape, fm)
    out = os.path.join(HERE, f"scale_{name}_200x50x50.npz")
    np.savez_compressed(out, idx=idx.astype(np.int32), u_sub=u[idx], n=rm.n, u_norm=np.linalg.norm(u),
                        u_sum=u.sum(), u_proj=projections(u), rel_residual=st["rel_residual"],
                        iterations=st["iterations"], iterations_1e8=s8["iterations"],
                        rel_residual_1e8=s8["rel_residual"], ic_setup_s=s8["setup_s"], cg_1e8_s=s8["cg_s"],
                        build_csr_s=t["build_csr"], fill_s=t["fill"], threads=threads, cpu=cpu_name(),
                        oracle=("reference build_CSR + fill_CSR_sparse_mat K, vendored Eigen 3.4.0 "
                                "ConjugateGradient<Lower|Upper, IncompleteCholesky<natural ordering>> FP64"))
    print(f"{name}: -> {out}", flush=True)


def main():
    from oracle.oracle import Reference
    if not Reference.available():
        sys.exit("oracle/_ref/libofea_ref.so is missing: make -C oracle REF=<reference tree>")
    args = sys.argv[1:]
    threads = 8
    if "--threads" in args:
        i = args.index("--threads")
        threads = int(args[i + 1])
        del args[i:i + 2]
    which = set(args) or {"tet", "cantilever", "simp"}
    R = Reference()
    if "tet" in which:
        tet(R)
    if "cantilever" in which:
        cantilever(R, "cantilever", None, threads)
    if "simp" in which:
        from openfea_b200 import meshgen as mg
        cantilever(R, "simp", 210e9 * mg.simp_density((200, 50, 50), 12, smooth=True) ** 3, threads)


if __name__ == "__main__":
    main()
