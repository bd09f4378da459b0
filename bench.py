#!/usr/bin/env python
"""Benchmark of the implicit-static hot path on B200.

Workload: C3D8 cantilever 200 x 50 x 50 (h = 5 mm, 522,801 nodes, 1,560,600
free DOF, 122.7M non-zeros), E = 210 GPa, nu = 0.3, clamped at x = 0, 1 MPa end
traction in -z (synthetic, seeded; the reference ships no benchmark input).

One step = one solve K u = f to a true FP64 relative residual of 1e-8 with the
learned + mixed-precision solver (FP64 flexible PCG, FP32 two-level V-cycle
preconditioner plus the learned coarse stage, including the per-matrix setup
of both levels and the network's evaluation), K assembled and f resident in
HBM.  The learned stage is trained once, before the warm-up, on residuals of
plain-PCG solves of a seeded random load (not the benchmark's load); its
training time is reported beside the number.  `value` = seconds per step
(device time, CUDA events on the launching stream, max over ranks).  The
mixed solver without the learned stage and the plain FP64 PCG are timed on
the same K and f for comparison.  `e2e` = the reference-facing path through
the C ABI with host buffers: mesh upload, pattern, FP64 assembly, solve
(trained weights handed to the new context), u back to the host - the span
the reference times with clock() (src/cae.cpp:257-281).

    python bench.py [--gpus N --steps K --warmup W]      # this library
    python bench.py --impl reference                    # the reference's CPU path

Multi-GPU (torchrun, one rank per GPU): every rank solves its own replica of
the workload (the single-matrix solve does not shard; no data-path
collective); timings are reduced with MAX over ranks.  The batched
reanalysis measurement partitions its variants over the ranks instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve s to 1e-8 rel. residual: learned+mixed vs plain GPU PCG; SpMV HBM GB/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--shape", default="200x50x50", help="cantilever elements nx x ny x nz")
    p.add_argument("--rtol", type=float, default=1e-8)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-reanalysis measurement")
    p.add_argument("--no-simp", action="store_true", help="skip the learned-preconditioner SIMP measurement")
    p.add_argument("--no-ca", action="store_true", help="skip the CA reanalysis measurement")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--batch-count", type=int, default=16, help="variants of --mode batched-only")
    p.add_argument("--batch-max-iter", type=int, default=12, help="iterations of --mode batched-only")
    p.add_argument("--mode", default="full", choices=["full", "solve-only", "batched-only"],
                   help="solve-only: assemble, a short training, one LEARNED, one MIXED and one "
                        "plain solve, nothing else (a short launch list for profilers); batched-only: "
                        "--batch-count variants of the batched workload, one MIXED batched solve capped "
                        "at --batch-max-iter iterations (a small case for a kernel profile)")
    return p.parse_args()


def shape_of(s):
    nx, ny, nz = (int(v) for v in s.lower().split("x"))
    return nx, ny, nz


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks --

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []
        self.t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_id}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------ batched reanalysis --

# Algorithmic bytes per (DOF, load case) of one batched iteration, vectors
# only (each array counted once per phase).  MIXED: A 36 (z FP32, p_old,
# q_old read; p, q written), B 56 (u, p, q, r read; u, r, b32, x32 written),
# residual 12, restriction 4, prolongation 8, post-smoothing 24.  PCG64: A 40
# (z, p_old, q_old read; p, q written), B 56 (u, p, q, r read; u, r, z
# written).
BATCH_VEC_BYTES_MIXED = 36 + 56 + 12 + 4 + 8 + 24
BATCH_VEC_BYTES_PCG64 = 40 + 56


def run_batched(ob, mg, local, hbm, steps=2, count=64, nrhs=16, rtol=1e-8, dist=None):
    """The batched reanalysis workload: `count` SIMP variants n x 20 x 20 (n ~
    U{20..60}), `nrhs` load cases each, solved by one persistent kernel per
    rank.  With several ranks the variants are partitioned (longest first onto
    the least-loaded rank); ranks exchange only timings and statistics."""
    from openfea_b200.multirank import gather_by_variant, max_over_ranks, partition_variants
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    all_variants = mg.design_variants(count=count, nrhs=nrhs)
    mine = partition_variants([3 * m.nd * nrhs for m, _ in all_variants], world)[rank]
    variants = [all_variants[i] for i in mine]
    ctxs, loads, meshes = [], [], []
    for m, F in variants:
        c = ob.Context(local)
        fm = c.upload_mesh(m)
        c.assemble_pattern()
        c.assemble_linear()
        ctxs.append(c)
        meshes.append((m, fm))
        loads.append(np.stack([mg.to_free(F[j], fm) for j in range(nrhs)]))
    sizes = gather_by_variant({i: (c.n, c.nnz) for i, c in zip(mine, ctxs)}, dist)
    n_tot = sum(v[0] for v in sizes.values())      # all ranks' variants
    nnz_tot = sum(v[1] for v in sizes.values())
    b = ob.Batch(ctxs, nrhs)
    b.set_rhs(loads)
    out = {}
    for meth, vec_b in (("GPU_PCG", BATCH_VEC_BYTES_PCG64), ("GPU_MIXED", BATCH_VEC_BYTES_MIXED)):
        b.solve_resident(meth, rtol=rtol)  # warm-up (tunes on first use, cached on disk)
        runs = [b.solve_resident(meth, rtol=rtol) for _ in range(steps if meth == "GPU_MIXED" else 1)]
        st = runs[-1]
        assert all(s_["status"] == 0 and s_["rel_residual"] <= rtol for s_ in st), st
        sec = max_over_ranks(min(r[0]["seconds"] for r in runs), dist)
        st = list(gather_by_variant(dict(zip(mine, st)), dist).values())
        iters = max(s_["iterations"] for s_ in st)
        # matrix bytes per iteration: FP64 BSELL once (+ BF16 twice for MIXED), 76/9 resp. 22/9 B per nnz
        mat = 76 * nnz_tot / 9 + (2 * 22 * nnz_tot / 9 if meth == "GPU_MIXED" else 0)
        per_iter = mat + vec_b * n_tot * nrhs
        out[meth] = {"seconds": sec, "iterations_max": iters,
                     "iterations_min": min(s_["iterations"] for s_ in st),
                     "worst_rel_residual": max(s_["rel_residual"] for s_ in st),
                     "solves_per_s": count * nrhs / sec, "tuning": b.tuning(meth),
                     "bytes_per_iteration": per_iter, "achieved_gbs": per_iter * iters / sec / 1e9,
                     "frac_of_hbm": per_iter * iters / sec / 1e9 / (hbm * world)}
    u_dev = b.solution()  # of the MIXED solve (the last one)
    # end to end through the one-call C ABI with host buffers (create, upload, solve, download)
    t0 = time.perf_counter()
    U, st = ob.solve_batched(ctxs, loads, method="GPU_MIXED", rtol=rtol)
    e2e = max_over_ranks(time.perf_counter() - t0, dist)
    diff = max_over_ranks(max(float(np.linalg.norm(a - c) / max(np.linalg.norm(c), 1e-300))
                              for a, c in zip(U, u_dev)), dist)
    b.close()
    for c in ctxs:
        c.close()
    mixed = out["GPU_MIXED"]
    return {
        "workload": (f"{count} C3D8 SIMP variants n x 20 x 20 (n ~ U{{20..60}}, rho ~ U[0.1,1], E = 210 GPa rho^3), "
                     f"{nrhs} random load cases each on the x=L face, rtol {rtol:g}; one persistent cooperative "
                     f"kernel per solve, graph-launched"),
        "n_dof_total": n_tot, "nnz_total": nnz_tot, "load_cases": count * nrhs,
        "ranks": world, "scaling": "strong (the variants are partitioned over the ranks)",
        "value": mixed["seconds"], "unit": "s per batch (all load cases of all variants)",
        "mixed": mixed, "plain_pcg64": out["GPU_PCG"],
        "speedup_vs_plain_pcg64": out["GPU_PCG"]["seconds"] / mixed["seconds"],
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes": int(8 * n_tot * nrhs), "d2h_bytes": int(8 * n_tot * nrhs),
                "max_rel_diff_vs_resident": diff},
    }


# ------------------------- learned preconditioner on a SIMP density field --

def run_learned_simp(ob, mg, local, shape, rtol=1e-8, steps=2):
    """The learned-preconditioner configuration: the cantilever mesh with a
    SIMP density field (rho ~ U[0.1, 1] per element, 3x3x3 box filter, E =
    210 GPa rho^3).  The stage is trained on the plain-PCG residuals of one
    seeded density sample (2,000 samples) and applied, unchanged, to another
    density sample; plain PCG64 and MIXED are timed on the same test matrix."""
    nx, ny, nz = shape

    def make(seed):
        m, ff = mg.cantilever_large(nx, ny, nz)
        m.E = 210e9 * mg.simp_density((nx, ny, nz), seed, smooth=True) ** 3
        c = ob.Context(local)
        fm = c.upload_mesh(m)
        c.assemble_pattern()
        c.assemble_linear()
        return c, mg.to_free(ff, fm)

    ctr, _ = make(11)
    cte, f = make(12)
    t0 = time.perf_counter()
    train = ctr.learned_train(None, sample_iters=2000, sample_every=1, steps=400, batch=16, lr=1e-3, seed=1234)
    train["wall_s"] = time.perf_counter() - t0
    weights = ctr.learned_weights()
    cte.set_learned_weights(weights)

    errs = {}
    shape_s = f"{nx}x{ny}x{nz}"

    def timed(method, reps):
        out = []
        for _ in range(reps):
            cte.precond_reset()
            u, st = cte.solve(f, method=method, rtol=rtol)
            assert st["status"] == 0 and st["rel_residual"] <= rtol, st
            out.append(st)
        errs[method] = oracle_error(u, "simp", shape_s)
        return min(out, key=lambda s_: s_["seconds"])

    plain = timed("GPU_PCG", 2)  # best of two: the first solve on a context also pays first-use costs
    mixed = timed("GPU_MIXED", steps + 1)
    learned = timed("GPU_LEARNED", steps + 1)
    ctr.close()
    cte.close()
    return {
        "workload": (f"C3D8 cantilever {nx}x{ny}x{nz}, SIMP density (rho ~ U[0.1,1], 3x3x3 box filter, seed 12), "
                     f"E = 210 GPa rho^3; stage trained on density seed 11 (2,000 plain-PCG residual samples); "
                     f"rel. residual {rtol:g}; set-up included"),
        "learned_s": learned["seconds"], "learned_iterations": learned["iterations"],
        "learned_rejected": learned["rejected_learned"], "learned_setup_s": learned["setup_seconds"],
        "mixed_s": mixed["seconds"], "mixed_iterations": mixed["iterations"],
        "plain_pcg64_s": plain["seconds"], "plain_pcg64_iterations": plain["iterations"],
        "speedup_learned_vs_plain": plain["seconds"] / learned["seconds"],
        "gain_learned_vs_mixed": mixed["seconds"] / learned["seconds"],
        "error_vs_oracle": errs,
        "training": train,
    }, weights


def run_ca(ob, mg, local, shape, n_basis=4, rtol=1e-6):
    """The CA reanalysis at full size: the cantilever and a modified model
    whose cavity (x in [0.3, 0.5] L, y and z in the middle half) is softened
    to 1e-3 E (SPD, so the modified model also has an exact solution to
    compare with).  CA from n_basis vectors (basis solves with K0 by MIXED)
    against a full MIXED solve of the modified model.  The basis solves stop
    at rtol: CA's own approximation error (about 1e-4 here) dominates any
    tighter basis."""
    nx, ny, nz = shape
    m0, ffull = mg.cantilever_large(nx, ny, nz)
    ex = (np.arange(m0.ne) // (ny * nz)) / nx
    ey = (np.arange(m0.ne) // nz % ny) / ny
    ez = (np.arange(m0.ne) % nz) / nz
    cav = (ex >= 0.3) & (ex < 0.5) & (ey >= 0.25) & (ey < 0.75) & (ez >= 0.25) & (ez < 0.75)
    E1 = np.full(m0.ne, m0.E0)
    E1[cav] = 1e-3 * m0.E0
    ctxs = []
    for E in (None, E1):
        c = ob.Context(local)
        m = mg.Mesh(m0.xyz, m0.topo, m0.etype, m0.fix, E, m0.E0, m0.nu)
        fm = c.upload_mesh(m)
        c.assemble_pattern()
        c.assemble_linear()
        ctxs.append(c)
    base, mod = ctxs
    f = mg.to_free(ffull, fm)
    u0, st0 = base.solve(f, method="GPU_MIXED", rtol=1e-10)
    runs = [ob.ca_reanalysis(base, mod, f, u0, n_basis=n_basis, method="GPU_MIXED", rtol=rtol) for _ in range(3)]
    u, cs = min(runs, key=lambda r: r[1]["seconds"])
    full = []
    for _ in range(3):
        mod.precond_reset()
        full.append(mod.solve(f, method="GPU_MIXED", rtol=1e-8))
    uex, stx = min(full, key=lambda r: r[1]["seconds"])
    base.close()
    mod.close()
    return {
        "workload": (f"C3D8 cantilever {nx}x{ny}x{nz}; modified model: a cavity of {int(cav.sum())} elements "
                     f"softened to 1e-3 E; CA with {n_basis} basis vectors (basis solves with K0 by GPU_MIXED "
                     f"to {rtol:g}), u0 given"),
        "ca_s": cs["seconds"], "basis_used": cs["basis_used"], "basis_solve_iterations": cs["solve_iterations"],
        "ca_rel_residual": cs["rel_residual"],
        "ca_rel_error_vs_full_solve": float(np.linalg.norm(u - uex) / np.linalg.norm(uex)),
        "u0_rel_error_vs_full_solve": float(np.linalg.norm(u0 - uex) / np.linalg.norm(uex)),
        "full_mixed_solve_s": stx["seconds"], "full_mixed_iterations": stx["iterations"],
        "note": "wall time of the one ofea_ca_reanalysis call (host buffers); the full solve is device time",
    }


# --------------------------------------------------------- reference (CPU) --

def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_model(shape):
    """The workload built by the reference's own code (oracle/_ref): set_BCs,
    then build_CSR + fill_CSR_sparse_mat timed in full."""
    from oracle.oracle import Reference
    from openfea_b200 import meshgen as mg
    m, ffull = mg.cantilever_large(*shape)
    fm = mg.free_map(m.nd, m.fix)
    rm = Reference().model(m)
    t0 = time.perf_counter()
    rm.assemble()
    wall = time.perf_counter() - t0
    t = rm.times()
    return rm, mg.to_free(ffull, fm), {"build_csr_s": t["build_csr"], "fill_s": t["fill"], "wall_s": wall}


def reference_cg_iterations(shape):
    """The iteration count of the reference K's Eigen CG + IC solve to 1e-8,
    measured by a full run of the same solver when the fixture was made
    (tests/golden/make_scale_golden.py), or None."""
    path = os.path.join(ROOT, "tests", "golden", "scale_cantilever_200x50x50.npz")
    if tuple(shape) != (200, 50, 50) or not os.path.exists(path):
        return None
    return int(np.load(path)["iterations_1e8"])


def cpu_baseline_sample(shape, rtol, threads):
    """A bounded sample (about 10 s) of the reference's solve of the workload:
    the 80 x 20 x 20 block of the same cantilever family (105,840 DOF),
    assembled by the reference's build_CSR + fill_CSR_sparse_mat and solved in
    full by Eigen CG + IC (the solver of the `--impl reference` measurement),
    then scaled to the full K: IC set-up and per-iteration time by the
    non-zero ratio, times the full K's iteration count measured by a full run
    of the same solver."""
    n_full_it = reference_cg_iterations(shape)
    if n_full_it is None:
        return None
    rm, f, asm = reference_model((80, 20, 20))
    u, st = rm.cg_ic(f, rtol=rtol, threads=threads)
    nx, ny, nz = shape
    ratio = block_nnz(nx, ny, nz) / block_nnz(80, 20, 20)
    solve = st["setup_s"] * ratio + st["cg_s"] / st["iterations"] * ratio * n_full_it
    return {
        "value": solve, "cores": threads,
        "sample": (f"reference K of the 80x20x20 block (build_CSR + fill_CSR_sparse_mat, {asm['wall_s']:.1f} s) "
                   f"solved by vendored Eigen CG + IncompleteCholesky to {rtol:g} on {threads} threads "
                   f"({st['iterations']} iterations, IC {st['setup_s']:.2f} s, CG {st['cg_s']:.2f} s), scaled "
                   f"to the {nx}x{ny}x{nz} K by its non-zero ratio ({ratio:.1f}) and its "
                   f"{n_full_it} iterations measured by a full run"),
    }


def block_nnz(nx, ny, nz):
    """3x3 blocks of K of the cantilever nx x ny x nz clamped at x = 0: every
    free node couples with the free nodes of its 3x3x3 neighbourhood; along
    an axis of m nodes that is 3m - 2 pairs (x: the nx free nodes)."""
    return (3 * nx - 2) * (3 * (ny + 1) - 2) * (3 * (nz + 1) - 2)


def run_reference(args):
    """The reference's CPU path on this workload, measured at full size: the
    reference builds and assembles K (build_CSR + fill_CSR_sparse_mat, timed
    in full), then its K is solved to the same relative residual by the
    vendored Eigen 3.4.0 ConjugateGradient + IncompleteCholesky (FP64, all
    host threads for the SpMV; SuperLU, the reference's own solver, takes
    about a day at this size and MKL Pardiso, its default, is not installed).
    That full solve (IC set-up + CG) is `value`, measured once before the
    steps; each warm-up and timed step is then a bounded sample, 10 CG
    iterations with the same IC factor on the same K, and `ms_per_step` is
    that sample's time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.oracle import Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libofea_ref.so is not built"}))
        return 0
    shape = shape_of(args.shape)
    threads = host_threads()
    t_start = time.perf_counter()
    rm, f, asm = reference_model(shape)
    u, full = rm.cg_ic(f, rtol=args.rtol, threads=threads)
    solve_s = full["setup_s"] + full["cg_s"]
    samples = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        _, st = rm.cg_ic_run(f, rtol=1e-30, max_iter=10)
        if i >= args.warmup:
            samples.append((time.perf_counter() - t0, st))
    step_s = statistics.mean(t for t, _ in samples)
    per_iter = statistics.mean(st["cg_s"] / st["iterations"] for _, st in samples)
    line = {
        "impl": "reference", "metric": METRIC, "value": solve_s, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": (f"C3D8 cantilever {args.shape} (h=5 mm), {rm.n} DOF, E=210 GPa, nu=0.3, "
                                f"clamped x=0, 1 MPa end traction; the reference-assembled K solved to FP64 "
                                f"rel. residual {args.rtol:g}"),
                   "n_dof": rm.n},
        "cpu_baseline": {"value": solve_s, "unit": "s", "cores": threads, "kind": "reference",
                         "sample": (f"value: one full solve of the reference-assembled K by vendored Eigen CG + "
                                    f"IncompleteCholesky (natural ordering) on {threads} threads, "
                                    f"{full['iterations']} iterations; steps: 10 CG iterations each")},
        "e2e": {"value": solve_s, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "detail": {"ic_setup_s": full["setup_s"], "cg_s": full["cg_s"], "iterations": full["iterations"],
                   "rel_residual": full["rel_residual"], "cg_s_per_iteration_in_steps": per_iter,
                   "assembly": asm, "analysis_s": asm["wall_s"] + solve_s, "host_threads": threads,
                   "run_wall_s": time.perf_counter() - t_start,
                   "superlu": "not run at this size (about n^2.7: a day or more)",
                   "pardiso": "unavailable on this box (MKL not installed)"},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- ours --

def oracle_error(u, name, shape, oracle_dir=os.path.join(ROOT, "tests", "golden")):
    """Relative L2 error of a solution (torch or numpy, free DOFs) against the
    committed oracle of the workload: the reference-assembled K solved by
    Eigen CG + IC to a relative residual near 1e-12, kept on a sub-grid of
    nodes (tests/golden/make_scale_golden.py).  None where no oracle exists."""
    path = os.path.join(oracle_dir, f"scale_{name}_{shape}.npz")
    if not os.path.exists(path):
        return None
    g = np.load(path)
    idx = g["idx"].astype(np.int64)
    uu = u.detach().cpu().numpy()[idx] if hasattr(u, "detach") else np.asarray(u)[idx]
    ref = g["u_sub"]
    return {"rel_l2_subgrid": float(np.linalg.norm(uu - ref) / np.linalg.norm(ref)),
            "oracle": "reference K + Eigen CG/IC to %.1e" % float(g["rel_residual"])}


def run_ours(args):
    import torch
    import openfea_b200 as ob
    from openfea_b200 import meshgen as mg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.mode == "batched-only":
        variants = mg.design_variants(count=args.batch_count, nrhs=16)
        ctxs, loads = [], []
        for m, F in variants:
            c = ob.Context(local)
            fm = c.upload_mesh(m)
            c.assemble_pattern()
            c.assemble_linear()
            ctxs.append(c)
            loads.append(np.stack([mg.to_free(F[j], fm) for j in range(F.shape[0])]))
        b = ob.Batch(ctxs, 16)
        b.set_rhs(loads)
        tune = b.tuning("GPU_MIXED")
        st = b.solve_resident("GPU_MIXED", rtol=args.rtol, max_iter=args.batch_max_iter, raise_on_error=False)
        if rank == 0:
            print(json.dumps({"mode": "batched-only", "variants": args.batch_count,
                              "n_dof_total": sum(c.n for c in ctxs), "tuning": tune,
                              "seconds": st[0]["seconds"], "iterations": st[0]["iterations"]}), flush=True)
        b.close()
        for c in ctxs:
            c.close()
        if dist:
            dist.destroy_process_group()
        return 0

    nx, ny, nz = shape_of(args.shape)
    mesh, ffull = mg.cantilever_large(nx, ny, nz)
    fm = mg.free_map(mesh.nd, mesh.fix)
    f = mg.to_free(ffull, fm)

    stream = torch.cuda.Stream()
    ctx = ob.Context(local)
    ctx.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    ctx.upload_mesh(mesh, fm)
    n, nnz = ctx.assemble_pattern()
    ctx.assemble_linear()
    setup_s = time.perf_counter() - t0

    def time_assembly(reps=3):
        """Device time of one FP64 assembly (integration, gather, block-Jacobi
        inverse, BSELL fill) on the context's stream, best of reps."""
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.assemble_linear()
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        return best * 1e-3
    asm_s = time_assembly()
    ne = int(mesh.ne)
    # reference-form integration flops (dense B^T D B at 8 Gauss points) and the
    # algorithmic HBM bytes of an assembly: K values written once, coordinates,
    # connectivity and E read once, and a 4-byte slot index per scalar
    # contribution (576 per C3D8)
    asm_flops = 69120.0 * ne
    asm_bytes = 8.0 * nnz + 24.0 * mesh.nd + 4.0 * 8 * ne + 8.0 * ne + 4.0 * 576 * ne
    assembly = {"seconds": asm_s, "dof_per_s": n / asm_s, "elements": ne,
                "reference_form_gflops": asm_flops / asm_s / 1e9,
                "algorithmic_bytes": asm_bytes, "achieved_gbs": asm_bytes / asm_s / 1e9,
                "note": "device time of assemble_linear: integration + gather + block-Jacobi + BSELL fill"}

    f_dev = torch.from_numpy(f).to(f"cuda:{local}")
    u_dev = torch.zeros_like(f_dev)
    torch.cuda.synchronize()

    def solve(method, fresh=True):
        # every step pays the preconditioner set-up for its K, as one linear
        # analysis does (assemble once, solve once)
        if fresh:
            ctx.precond_reset()
        rc, st = ctx.solve_device(f_dev.data_ptr(), u_dev.data_ptr(), method=method, rtol=args.rtol)
        if rc != 0:
            raise RuntimeError(f"{method} solve failed: {st}")
        return st

    if args.mode == "solve-only":
        # a short launch list for profilers: a brief training (20 steps), then
        # one LEARNED, one MIXED and one plain solve
        ctx.learned_train(None, sample_iters=200, sample_every=4, steps=20, batch=16)
        ctx.set_setup_trace(True)
        st_l = solve("GPU_LEARNED")
        ph_l = ctx.setup_phase_times()
        st_m = solve("GPU_MIXED")
        ph_m = ctx.setup_phase_times()
        ctx.set_setup_trace(False)
        st_p = solve("GPU_PCG")
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"mode": "solve-only", "shape": args.shape, "n": n, "nnz": nnz,
                              "learned": st_l, "mixed": st_m, "plain": st_p,
                              "setup_phases_ms": {"GPU_LEARNED": ph_l, "GPU_MIXED": ph_m}}), flush=True)
        ctx.close()
        if dist:
            dist.destroy_process_group()
        return 0

    # the learned stage: trained once on plain-PCG residuals of a seeded random load
    t_tr = time.perf_counter()
    train = ctx.learned_train(None, sample_iters=4000, sample_every=1, steps=800, batch=16, lr=1e-3, seed=1234)
    train["wall_s"] = time.perf_counter() - t_tr
    weights = ctx.learned_weights()

    for _ in range(args.warmup):
        solve("GPU_LEARNED")
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    gpu_uuid = None
    try:
        gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
        if not gpu_uuid.startswith("GPU-"):
            gpu_uuid = "GPU-" + gpu_uuid
    except Exception:
        gpu_uuid = str(local)
    with ClockSampler(gpu_uuid) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
        for _ in range(args.steps):
            stats.append(solve("GPU_LEARNED"))
        with torch.cuda.stream(stream):
            ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    total_ms = max_over_ranks(ev0.elapsed_time(ev1))
    sec = total_ms / 1e3 / args.steps
    for st in stats:
        assert st["status"] == 0 and st["rel_residual"] <= args.rtol, st
    u_learned = u_dev.clone()
    oracle_err = {"GPU_LEARNED": oracle_error(u_learned, "cantilever", args.shape)}

    # the same solver without the learned stage (same K, f, set-up included)
    stm = [solve("GPU_MIXED") for _ in range(2)]
    mixed_s = max_over_ranks(min(s_["seconds"] for s_ in stm))
    oracle_err["GPU_MIXED"] = oracle_error(u_dev, "cantilever", args.shape)

    # the plain FP64 PCG the metric compares against (same workload, outside the timed steps)
    st64 = solve("GPU_PCG")
    st64b = solve("GPU_PCG")
    plain_s = max_over_ranks(min(st64["seconds"], st64b["seconds"]))
    oracle_err["GPU_PCG"] = oracle_error(u_dev, "cantilever", args.shape)
    err_vs_plain = float(torch.linalg.norm(u_learned - u_dev) / torch.linalg.norm(u_dev))

    # the set-up's phases (CUDA events on the context stream), one traced
    # solve of each preconditioned method after the timed region
    ctx.set_setup_trace(True)
    solve("GPU_LEARNED")
    setup_phases = {"GPU_LEARNED": ctx.setup_phase_times()}
    solve("GPU_MIXED")
    setup_phases["GPU_MIXED"] = ctx.setup_phase_times()
    ctx.set_setup_trace(False)

    # roofline of the dominant kernels (CUDA events on the launching stream)
    solve("GPU_MIXED")
    hbm, peak_kind = peaks()
    msM, byM = ctx.profile_kernels("GPU_MIXED", reps=30)
    solve("GPU_PCG")
    msP, byP = ctx.profile_kernels("GPU_PCG", reps=30)
    gbsA = byM[0] / (msM[0] * 1e-3) / 1e9
    gbs32 = byM[1] / (msM[1] * 1e-3) / 1e9
    gbs64 = byP[0] / (msP[0] * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(f"k_fcg_A/{args.shape}")
        except Exception:
            traffic = None

    # end to end through the C ABI with host buffers
    e2e, phases = [], []
    h2d = mesh.xyz.nbytes + mesh.nd * 4 + mesh.ne * (8 * 4 + 4) + f.nbytes
    d2h = n * 8
    for i in range(args.e2e_steps + 1):
        barrier()
        t0 = time.perf_counter()
        c2 = ob.Context(local)
        c2.upload_mesh(mesh, fm)
        t1 = time.perf_counter()
        c2.assemble_pattern()
        t2 = time.perf_counter()
        c2.assemble_linear()
        c2.set_learned_weights(weights)
        t3 = time.perf_counter()
        u_host, st = c2.solve(f, method="GPU_LEARNED", rtol=args.rtol)
        t4 = time.perf_counter()
        c2.close()
        if i > 0:
            e2e.append(max_over_ranks(t4 - t0))
            phases.append({"context_upload_s": t1 - t0, "pattern_s": t2 - t1, "assembly_s": t3 - t2,
                           "solve_s": t4 - t3, "solve_device_s": st["seconds"],
                           "precond_setup_s": st["setup_seconds"]})
        assert st["status"] == 0
    e2e_s = statistics.mean(e2e) if e2e else None
    batched = None
    if not args.no_batched:
        batched = run_batched(ob, mg, local, hbm, dist=dist)
    learned_simp = transfer = None
    if not args.no_simp:
        learned_simp, simp_weights = run_learned_simp(ob, mg, local, (nx, ny, nz), rtol=args.rtol)
        # the headline workload with a stage trained on another matrix (the
        # SIMP density sample's), not on the benchmark's own K
        ctx.set_learned_weights(simp_weights)
        stt = [solve("GPU_LEARNED") for _ in range(3)]
        bt = min(stt, key=lambda s_: s_["seconds"])
        assert bt["status"] == 0 and bt["rel_residual"] <= args.rtol, bt
        transfer = {"weights": "trained on the SIMP density sample (seed 11) of the same mesh, not on this K",
                    "seconds": bt["seconds"], "iterations": bt["iterations"],
                    "rejected_learned": bt["rejected_learned"], "gain_vs_mixed": mixed_s / bt["seconds"],
                    "error_vs_oracle": oracle_error(u_dev, "cantilever", args.shape)}
        ctx.set_learned_weights(weights)
    ca = None
    if not args.no_ca:
        ca = run_ca(ob, mg, local, (nx, ny, nz))

    line = {
        "metric": METRIC, "value": sec, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {
            "workload": (f"C3D8 cantilever {args.shape} (h=5 mm), {n} DOF, nnz {nnz}, E=210 GPa, "
                         f"nu=0.3, clamped x=0, 1 MPa end traction; FP64 flexible PCG with the FP32 "
                         f"two-level V-cycle preconditioner and the learned coarse stage, to FP64 rel. "
                         f"residual {args.rtol:g}"),
            "n_dof": n, "nnz": nnz, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (FP64 K ~1 GB and BF16 K ~0.25 GB streamed per SpMV)",
        },
        "roofline": {"bound": "hbm", "kernel": "k_fcg_A (FP64 BSELL SpMV + p update + p.q)",
                     "achieved": gbsA, "peak": hbm, "unit": "GB/s", "frac": gbsA / hbm,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "bytes_per_launch": byM[0], "ms_per_launch": msM[0]},
        "spmv32_smoother": {"kernel": "k_fcg_post (BSELL SpMV with BF16 K and FP32 arithmetic + block-Jacobi + dots)",
                            "achieved_gbs": gbs32, "frac": gbs32 / hbm, "bytes_per_launch": byM[1],
                            "ms_per_launch": msM[1]},
        "spmv64_plain": {"kernel": "k_pcg64_A (FP64 BSELL SpMV, plain PCG)", "achieved_gbs": gbs64,
                         "frac": gbs64 / hbm, "bytes_per_launch": byP[0], "ms_per_launch": msP[0]},
        "solver": {"method": "GPU_LEARNED", "iterations": stats[-1]["iterations"],
                   "refinements": stats[-1]["refinements"], "rejected_learned": stats[-1]["rejected_learned"],
                   "rel_residual": stats[-1]["rel_residual"], "plain_pcg64_s": plain_s,
                   "plain_pcg64_iterations": st64["iterations"],
                   "speedup_vs_plain": plain_s / sec, "rel_diff_vs_plain": err_vs_plain,
                   "error_vs_oracle": oracle_err,
                   "mixed_without_learned_s": mixed_s, "mixed_without_learned_iterations": stm[-1]["iterations"],
                   "learned_gain_vs_mixed": mixed_s / sec,
                   "learned_training": train,
                   "learned_with_transferred_weights": transfer,
                   "precond_setup_s": stats[-1]["setup_seconds"],
                   "setup_phases_ms": setup_phases,
                   "mesh_pattern_assembly_s": setup_s},
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "phases": phases[-1] if phases else None},
        "clocks": clk.summary(),
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
        "assembly": assembly,
        "batched": batched,
        "learned_simp": learned_simp,
        "ca_reanalysis": ca,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        try:
            r = cpu_baseline_sample((nx, ny, nz), args.rtol, threads)
            if r is None:
                raise RuntimeError(f"no measured iteration count for the {args.shape} reference solve")
            line["cpu_baseline"] = {"value": r["value"], "unit": "s", "cores": r["cores"], "kind": "reference",
                                    "sample": r["sample"]}
        except Exception as e:  # the reference build is absent
            line["cpu_baseline"] = {"value": None, "unit": "s", "cores": threads, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
