"""openfea_b200: OpenFEA's implicit-static hot path on one B200 (sm_100a).

The product is the C ABI in include/ofea_gpu.h / include/ofea_host.h,
implemented by libofea_gpu.so (hand-written CUDA kernels + C++ host I/O).
This module binds it with ctypes for Python callers and tests, and mirrors the
reference's entry points (``AssambleStiffness.build_CSR`` /
``fill_CSR_sparse_mat``, ``solution_api``) with GPU solver names.

There is no CPU fallback: when the library or a GPU is missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libofea_gpu.so")

OFEA_OK = 0
STATUS = {
    0: "OFEA_OK", -1: "OFEA_ERR_INVALID_ARG", -2: "OFEA_ERR_CUDA", -3: "OFEA_ERR_OOM",
    -4: "OFEA_ERR_NOT_CONVERGED", -5: "OFEA_ERR_TIMEOUT", -6: "OFEA_ERR_STATE",
    -7: "OFEA_ERR_CAPACITY", -8: "OFEA_ERR_BREAKDOWN", -9: "OFEA_ERR_NO_DEVICE",
    -10: "OFEA_ERR_IO", -11: "OFEA_ERR_UNKNOWN_SOLVER", -12: "OFEA_ERR_REJECTED",
}
SOLVERS = {"GPU_PCG": 0, "GPU_MIXED": 1, "GPU_LEARNED": 2}

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_LL = ctypes.c_longlong


class OfeaError(RuntimeError):
    def __init__(self, code, what, msg=""):
        self.code = code
        super().__init__(f"{what}: {STATUS.get(code, code)} {msg}".strip())


class SolveOpts(ctypes.Structure):
    _fields_ = [("method", _I), ("rtol", _D), ("max_iter", _I), ("time_budget_s", _D),
                ("check_every", _I), ("ru_delta", _D), ("use_graph", _I)]


class SolveStats(ctypes.Structure):
    _fields_ = [("status", _I), ("iterations", _I), ("refinements", _I), ("rel_residual", _D),
                ("seconds", _D), ("setup_seconds", _D), ("rejected_learned", _I),
                ("kernel_launches", _LL)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CaStats(ctypes.Structure):
    _fields_ = [("status", _I), ("basis_requested", _I), ("basis_used", _I), ("solve_iterations", _I),
                ("rel_residual", _D), ("seconds", _D)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LearnOpts(ctypes.Structure):
    _fields_ = [("sample_iters", _I), ("sample_every", _I), ("steps", _I), ("batch", _I),
                ("lr", ctypes.c_float), ("seed", ctypes.c_uint), ("reset", _I)]


class LearnStats(ctypes.Structure):
    _fields_ = [("samples", _I), ("steps", _I), ("loss_first", _D), ("loss_last", _D), ("seconds", _D)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    """Load libofea_gpu.so (built by ``python -m openfea_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is not built: run python -m openfea_b200.build")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "ofea_version": (ctypes.c_char_p, []),
        "ofea_status_string": (ctypes.c_char_p, [_I]),
        "ofea_last_error": (ctypes.c_char_p, []),
        "ofea_solve_opts_default": (None, [_P]),
        "ofea_ctx_create": (_I, [ctypes.POINTER(_P), _I]),
        "ofea_ctx_destroy": (_I, [_P]),
        "ofea_ctx_set_stream": (_I, [_P, _P]),
        "ofea_mesh_upload": (_I, [_P, _I, _P, _I, _P, _P, _P, _D, _D, _P]),
        "ofea_mesh_set_modulus": (_I, [_P, _P, _D]),
        "ofea_assemble_pattern": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_LL)]),
        "ofea_assemble_linear": (_I, [_P]),
        "ofea_assemble_nl": (_I, [_P, _P, _P]),
        "ofea_get_csr": (_I, [_P, _P, _P, _P]),
        "ofea_matrix_upload_csc": (_I, [_P, _I, _P, _P, _I, _P, _P, _P]),
        "ofea_tc_matmul": (_I, [_I, _I, _I, _I, _P, _P, _P]),
        "ofea_get_element_matrices": (_I, [_P, _I, _I, _P]),
        "ofea_spmv": (_I, [_P, _P, _P]),
        "ofea_solve": (_I, [_P, _P, _P, _I, _P, _P]),
        "ofea_solve_device": (_I, [_P, _P, _P, _P, _P]),
        "ofea_inp_read": (_I, [ctypes.c_char_p, ctypes.POINTER(_P)]),
        "ofea_ca_info_read": (_I, [ctypes.c_char_p, ctypes.POINTER(_I), ctypes.POINTER(_I), _P, _P, _P, _P, _P]),
        "ofea_ca_reanalysis": (_I, [_P, _P, _P, _P, _I, _P, _P, _P]),
        "ofea_model_free": (None, [_P]),
        "ofea_model_sizes": (_I, [_P, _P, _P, _P, _P]),
        "ofea_model_arrays": (_I, [_P, _P, _P, _P, _P, _P]),
        "ofea_model_material": (_I, [_P, _P, _P, _P, _P]),
        "ofea_model_cload": (_I, [_P, _P, _P]),
        "ofea_build_free_index": (_I, [_I, _I, _P, _P, _P]),
        "ofea_build_single_load": (_I, [_I, _P, _I, _P, _I, _D, _P]),
        "ofea_full_displacement": (_I, [_I, _P, _P, _P]),
        "ofea_write_vtk": (_I, [ctypes.c_char_p, _I, _P, _I, _P, _P, _P, _D]),
        "ofea_write_vtk_stress": (_I, [ctypes.c_char_p, _I, _P, _I, _P, _P, _P, _D, _P]),
        "ofea_stress": (_I, [_P, _P, _I, _P, _P]),
        "ofea_profile_solver_kernels": (_I, [_P, _I, _I, _P, _P]),
        "ofea_set_setup_trace": (_I, [_P, _I]),
        "ofea_setup_phase_times": (_I, [_P, _P, _I, ctypes.POINTER(_I), ctypes.c_char_p, _I]),
        "ofea_precond_reset": (_I, [_P]),
        "ofea_set_coarse_nodes": (_I, [_P, _I]),
        "ofea_set_coarse_solver": (_I, [_P, _I]),
        "ofea_coarse_apply": (_I, [_P, _P, _P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
        "ofea_set_assembly_path": (_I, [_P, _I]),
        "ofea_get_assembly_path": (_I, [_P, ctypes.POINTER(ctypes.c_int)]),
        "ofea_trim_device_memory": (_I, []),
        "ofea_learn_opts_default": (None, [_P]),
        "ofea_batch_create": (_I, [ctypes.POINTER(_P), _P, _I, _I]),
        "ofea_batch_destroy": (_I, [_P]),
        "ofea_batch_set_rhs": (_I, [_P, _P]),
        "ofea_batch_solve_resident": (_I, [_P, _P, _P]),
        "ofea_batch_get_solution": (_I, [_P, _P]),
        "ofea_batch_solve": (_I, [_P, _P, _P, _P, _P]),
        "ofea_batch_tuning": (_I, [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I),
                                   ctypes.POINTER(_D)]),
        "ofea_batch_set_trace": (_I, [_P, _I]),
        "ofea_batch_phase_times": (_I, [_P, _P, _I, ctypes.POINTER(_I)]),
        "ofea_solve_batched": (_I, [_P, _I, _P, _P, _I, _P, _P]),
        "ofea_check_barrier_timeout": (_I, [_P, _I, ctypes.POINTER(_I)]),
        "ofea_learned_train": (_I, [_P, _P, _P, _P]),
        "ofea_learned_get_weights": (_I, [_P, _P, ctypes.POINTER(_LL)]),
        "ofea_learned_set_weights": (_I, [_P, _P, _LL]),
        "ofea_learned_save": (_I, [_P, ctypes.c_char_p]),
        "ofea_learned_load": (_I, [_P, ctypes.c_char_p]),
        "ofea_learned_level": (_I, [_P, ctypes.POINTER(_I), _P, _P, _P]),
        "ofea_learned_gradient": (_I, [_P, _P, _I, ctypes.POINTER(_D), _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _check(rc, what):
    if rc != OFEA_OK:
        raise OfeaError(rc, what, lib().ofea_last_error().decode(errors="replace"))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def trim_device_memory():
    """Return the library's cached device memory to the driver."""
    _check(lib().ofea_trim_device_memory(), "ofea_trim_device_memory")


class Batch:
    """Many assembled variants (Contexts on one GPU) x up to 32 load cases each,
    solved together by the persistent batched solver (ofea_batch_* in
    include/ofea_gpu.h).  Load cases are given per variant as an array of
    shape (nrhs, n_v)."""

    def __init__(self, contexts, nrhs):
        self.contexts = list(contexts)
        self.nrhs = int(nrhs)
        self.h = _P()
        arr = (_P * len(self.contexts))(*[c.h for c in self.contexts])
        _check(lib().ofea_batch_create(ctypes.byref(self.h), arr, len(self.contexts), self.nrhs),
               "ofea_batch_create")

    def close(self):
        if self.h:
            lib().ofea_batch_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_rhs(self, loads):
        self._f = [np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(self.nrhs, c.n))
                   for F, c in zip(loads, self.contexts)]
        ptrs = (_P * len(self._f))(*[F.ctypes.data for F in self._f])
        _check(lib().ofea_batch_set_rhs(self.h, ptrs), "ofea_batch_set_rhs")

    def solve_resident(self, method="GPU_MIXED", rtol=1e-8, raise_on_error=True, **kw):
        o = solve_opts(method, rtol, **kw)
        stats = (SolveStats * len(self.contexts))()
        rc = lib().ofea_batch_solve_resident(self.h, ctypes.byref(o), stats)
        if rc != OFEA_OK and raise_on_error:
            _check(rc, "ofea_batch_solve_resident")
        return [s_.as_dict() for s_ in stats]

    def solution(self):
        U = [np.zeros((self.nrhs, c.n)) for c in self.contexts]
        ptrs = (_P * len(U))(*[u.ctypes.data for u in U])
        _check(lib().ofea_batch_get_solution(self.h, ptrs), "ofea_batch_get_solution")
        return U

    def solve(self, loads, method="GPU_MIXED", rtol=1e-8, **kw):
        self.set_rhs(loads)
        st = self.solve_resident(method, rtol, **kw)
        return self.solution(), st

    def tuning(self, method="GPU_MIXED"):
        r, t, c, ms = _I(), _I(), _I(), _D()
        _check(lib().ofea_batch_tuning(self.h, SOLVERS[method], ctypes.byref(r), ctypes.byref(t), ctypes.byref(c),
                                       ctypes.byref(ms)), "ofea_batch_tuning")
        return {"rhs_per_lane": r.value, "threads": t.value, "ctas_per_sm": c.value, "ms_per_iteration": ms.value}

    def set_trace(self, max_phases):
        """Record the device clock after each grid barrier of later solves
        (up to max_phases barriers per launch; 0 turns it off)."""
        _check(lib().ofea_batch_set_trace(self.h, int(max_phases)), "ofea_batch_set_trace")

    def phase_times(self):
        """Milliseconds between consecutive barriers of the last traced launch."""
        n = _I()
        _check(lib().ofea_batch_phase_times(self.h, None, 0, ctypes.byref(n)), "ofea_batch_phase_times")
        out = np.zeros(n.value)
        _check(lib().ofea_batch_phase_times(self.h, out.ctypes.data, n.value, ctypes.byref(n)),
               "ofea_batch_phase_times")
        return out


def solve_batched(contexts, loads, method="GPU_MIXED", rtol=1e-8, **kw):
    """One-call batched solve through ofea_solve_batched: loads[v] has shape
    (nrhs, n_v); returns the solutions in the same shapes and per-variant stats."""
    nrhs = int(np.asarray(loads[0]).shape[0])
    F = [np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(nrhs, c.n)) for x, c in zip(loads, contexts)]
    U = [np.zeros_like(x) for x in F]
    ctx = (_P * len(contexts))(*[c.h for c in contexts])
    fp = (_P * len(F))(*[x.ctypes.data for x in F])
    up = (_P * len(U))(*[x.ctypes.data for x in U])
    o = solve_opts(method, rtol, **kw)
    stats = (SolveStats * len(contexts))()
    _check(lib().ofea_solve_batched(ctx, len(contexts), fp, up, nrhs, ctypes.byref(o), stats), "ofea_solve_batched")
    return U, [s_.as_dict() for s_ in stats]


def tc_matmul(A, B, device=0):
    """D = A B^T on the tensor cores (BF16 operands, FP32 accumulation), the
    product the learned stage's dense layers use (ofea_tc_matmul)."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    M, K = A.shape
    N, K2 = B.shape
    assert K == K2
    D = np.zeros((M, N), dtype=np.float32)
    _check(lib().ofea_tc_matmul(device, M, N, K, _ptr(A), _ptr(B), _ptr(D)), "ofea_tc_matmul")
    return D


def check_barrier_timeout(ctx, limit_ms=20):
    """The batched solver's grid barrier given a CTA that never arrives: returns
    1 if it opened (it must not), 0 when every wait ran out as designed."""
    r = _I(-1)
    _check(lib().ofea_check_barrier_timeout(ctx.h, int(limit_ms), ctypes.byref(r)), "ofea_check_barrier_timeout")
    return r.value


def solve_opts(method="GPU_PCG", rtol=1e-8, max_iter=100000, time_budget_s=0.0, check_every=0,
               ru_delta=0.1, use_graph=True) -> SolveOpts:
    o = SolveOpts()
    lib().ofea_solve_opts_default(ctypes.byref(o))
    o.method = SOLVERS[method] if isinstance(method, str) else int(method)
    o.rtol, o.max_iter, o.time_budget_s = rtol, max_iter, time_budget_s
    o.check_every, o.ru_delta, o.use_graph = check_every, ru_delta, int(bool(use_graph))
    return o


class Context:
    """One GPU context: mesh, pattern, K and solver state resident on the device."""

    def __init__(self, device=0):
        self.h = _P()
        _check(lib().ofea_ctx_create(ctypes.byref(self.h), device), "ofea_ctx_create")
        self.n = 0
        self.nnz = 0

    def close(self):
        if self.h:
            lib().ofea_ctx_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        _check(lib().ofea_ctx_set_stream(self.h, _P(stream_handle)), "ofea_ctx_set_stream")

    def upload(self, xyz, topo, etype, free_map, E0, nu, E_elem=None):
        xyz, topo, etype, fm = _f64(xyz), _i32(topo), _i32(etype), _i32(free_map)
        E = _f64(E_elem) if E_elem is not None else None
        self._keep = (xyz, topo, etype, fm, E)
        _check(lib().ofea_mesh_upload(self.h, xyz.shape[0], _ptr(xyz), topo.shape[0], _ptr(topo),
                                      _ptr(etype), _ptr(E), E0, nu, _ptr(fm)), "ofea_mesh_upload")
        self.nd, self.ne = int(xyz.shape[0]), int(topo.shape[0])

    def upload_mesh(self, mesh, free_map=None):
        fm = free_map if free_map is not None else build_free_index(mesh.nd, mesh.fix)
        self.upload(mesh.xyz, mesh.topo, mesh.etype, fm, mesh.E0, mesh.nu, mesh.E)
        return fm

    def upload_csc(self, xyz, free_map, col_ptr, row_idx, val):
        """K as the reference's assembled CSC arrays (col_idx_, row_idx_,
        nz_val_) with the model's coordinates and free numbering; replaces
        any mesh (ofea_matrix_upload_csc)."""
        xyz, fm = _f64(xyz), _i32(free_map)
        cp, ri, v = _i32(col_ptr), _i32(row_idx), _f64(val)
        n = cp.size - 1
        _check(lib().ofea_matrix_upload_csc(self.h, xyz.shape[0], _ptr(xyz), _ptr(fm), n, _ptr(cp), _ptr(ri),
                                            _ptr(v)), "ofea_matrix_upload_csc")
        self.nd, self.ne = int(xyz.shape[0]), 0
        self.n, self.nnz = n, int(cp[-1])

    def set_modulus(self, E_elem, E0):
        E = _f64(E_elem) if E_elem is not None else None
        _check(lib().ofea_mesh_set_modulus(self.h, _ptr(E), E0), "ofea_mesh_set_modulus")

    def assemble_pattern(self):
        n, nnz = _I(), _LL()
        _check(lib().ofea_assemble_pattern(self.h, ctypes.byref(n), ctypes.byref(nnz)), "ofea_assemble_pattern")
        self.n, self.nnz = n.value, nnz.value
        return self.n, self.nnz

    def assemble_linear(self):
        _check(lib().ofea_assemble_linear(self.h), "ofea_assemble_linear")

    def assemble_nl(self, u):
        u = _f64(u)
        fint = np.zeros(self.n)
        _check(lib().ofea_assemble_nl(self.h, _ptr(u), _ptr(fint)), "ofea_assemble_nl")
        return fint

    def stress(self, u, mode="reference"):
        """Stress recovery (ofea_stress): per element (ne, 7) in caller order and
        per node (7, nd): xx yy zz xy yz xz von Mises.  mode "reference" gives
        the reference's numbers (C3D4: engineering strain B u; C3D8: zero),
        "cauchy" the Cauchy stress D B u."""
        u = _f64(u)
        elem = np.zeros((self.ne, 7))
        node = np.zeros((7, self.nd))
        m = {"reference": 0, "cauchy": 1}[mode]
        _check(lib().ofea_stress(self.h, _ptr(u), m, _ptr(elem), _ptr(node)), "ofea_stress")
        return elem, node

    def get_csr(self):
        rp = np.zeros(self.n + 1, dtype=np.int32)
        col = np.zeros(self.nnz, dtype=np.int32)
        val = np.zeros(self.nnz)
        _check(lib().ofea_get_csr(self.h, _ptr(rp), _ptr(col), _ptr(val)), "ofea_get_csr")
        return rp, col, val

    def element_matrices(self, first, count, npe):
        m = 3 * npe
        K = np.zeros((count, m, m))
        _check(lib().ofea_get_element_matrices(self.h, first, count, _ptr(K)), "ofea_get_element_matrices")
        return K

    def spmv(self, x):
        x = _f64(x)
        y = np.zeros(self.n)
        _check(lib().ofea_spmv(self.h, _ptr(x), _ptr(y)), "ofea_spmv")
        return y

    def solve(self, f, method="GPU_PCG", rtol=1e-8, raise_on_error=True, **kw):
        F = _f64(f)
        nrhs = 1 if F.ndim == 1 else F.shape[1]
        Fc = np.asfortranarray(F.reshape(self.n, nrhs))
        U = np.zeros((self.n, nrhs), order="F")
        stats = (SolveStats * nrhs)()
        o = solve_opts(method, rtol, **kw)
        rc = lib().ofea_solve(self.h, Fc.ctypes.data_as(_P), U.ctypes.data_as(_P), nrhs,
                              ctypes.byref(o), stats)
        if rc != OFEA_OK and raise_on_error:
            _check(rc, "ofea_solve")
        st = [s.as_dict() for s in stats]
        return (U[:, 0] if F.ndim == 1 else U), (st[0] if F.ndim == 1 else st)

    def set_coarse_nodes(self, nodes):
        """Target free nodes per coarse aggregate (default 1000)."""
        _check(lib().ofea_set_coarse_nodes(self.h, int(nodes)), "ofea_set_coarse_nodes")

    def set_coarse_solver(self, method):
        """0: block LDL^T factor of the banded coarse matrix where its band
        allows (default); 1: dense Gauss-Jordan inverse."""
        _check(lib().ofea_set_coarse_solver(self.h, int(method)), "ofea_set_coarse_solver")

    def coarse_apply(self, c=None):
        """y = E^-1 c by the current coarse solve (FP32 arithmetic); with c
        None, (m, factored) only."""
        m, fac = ctypes.c_int(0), ctypes.c_int(0)
        _check(lib().ofea_coarse_apply(self.h, None, None, ctypes.byref(m), ctypes.byref(fac)), "ofea_coarse_apply")
        if c is None:
            return m.value, bool(fac.value)
        c = np.ascontiguousarray(c, dtype=np.float64)
        if c.shape != (m.value,):
            raise ValueError(f"coarse vector must have {m.value} values")
        y = np.zeros(m.value)
        _check(lib().ofea_coarse_apply(self.h, _ptr(c), _ptr(y), None, None), "ofea_coarse_apply")
        return y

    def set_assembly_path(self, path):
        """0: one-pass C3D8 assembly where the mesh allows it (default); 1: two-pass."""
        _check(lib().ofea_set_assembly_path(self.h, int(path)), "ofea_set_assembly_path")

    def assembly_path(self):
        """0 if K came from the one-pass C3D8 assembly, 1 if from the two-pass one (or a CSC upload)."""
        v = ctypes.c_int(-1)
        _check(lib().ofea_get_assembly_path(self.h, ctypes.byref(v)), "ofea_get_assembly_path")
        return v.value

    def precond_reset(self):
        """Rebuild the preconditioner at the next solve (as after a new assembly)."""
        _check(lib().ofea_precond_reset(self.h), "ofea_precond_reset")

    def profile_kernels(self, method="GPU_MIXED", reps=20):
        """Average ms and algorithmic bytes per launch of the solver's A and B
        kernels (CUDA events on the context stream)."""
        ms = np.zeros(2)
        by = np.zeros(2)
        m = SOLVERS[method] if isinstance(method, str) else int(method)
        _check(lib().ofea_profile_solver_kernels(self.h, m, reps, _ptr(ms), _ptr(by)),
               "ofea_profile_solver_kernels")
        return ms, by

    def set_setup_trace(self, on=True):
        """Record the preconditioner set-up's phase boundaries (CUDA events)
        on the next MIXED / LEARNED solves."""
        _check(lib().ofea_set_setup_trace(self.h, int(bool(on))), "ofea_set_setup_trace")

    def setup_phase_times(self):
        """{phase: device ms} of the last traced set-up, in order."""
        n = ctypes.c_int(0)
        _check(lib().ofea_setup_phase_times(self.h, None, 0, ctypes.byref(n), None, 0), "ofea_setup_phase_times")
        ms = np.zeros(max(n.value, 1))
        buf = ctypes.create_string_buffer(64 * max(n.value, 1) + 1)
        _check(lib().ofea_setup_phase_times(self.h, _ptr(ms), n.value, ctypes.byref(n), buf, len(buf)),
               "ofea_setup_phase_times")
        names = buf.value.decode().split(",") if n.value else []
        return dict(zip(names, ms[:n.value].tolist()))

    # ---- learned coarse-correction stage
    def learned_train(self, f=None, sample_iters=600, sample_every=4, steps=400, batch=16, lr=1e-3,
                      seed=1234, reset=False):
        o = LearnOpts()
        lib().ofea_learn_opts_default(ctypes.byref(o))
        o.sample_iters, o.sample_every, o.steps, o.batch = sample_iters, sample_every, steps, batch
        o.lr, o.seed, o.reset = lr, seed, int(bool(reset))
        st = LearnStats()
        fa = _f64(f) if f is not None else None
        _check(lib().ofea_learned_train(self.h, _ptr(fa), ctypes.byref(o), ctypes.byref(st)),
               "ofea_learned_train")
        return st.as_dict()

    def learned_weights(self):
        n = _LL()
        _check(lib().ofea_learned_get_weights(self.h, None, ctypes.byref(n)), "ofea_learned_get_weights")
        w = np.zeros(n.value, dtype=np.float32)
        _check(lib().ofea_learned_get_weights(self.h, _ptr(w), ctypes.byref(n)), "ofea_learned_get_weights")
        return w

    def set_learned_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().ofea_learned_set_weights(self.h, _ptr(w), w.size), "ofea_learned_set_weights")

    def learned_save(self, path):
        _check(lib().ofea_learned_save(self.h, str(path).encode()), "ofea_learned_save")

    def learned_load(self, path):
        _check(lib().ofea_learned_load(self.h, str(path).encode()), "ofea_learned_load")

    def learned_level(self):
        na = _I()
        _check(lib().ofea_learned_level(self.h, ctypes.byref(na), None, None, None), "ofea_learned_level")
        nbr = np.zeros((na.value, 27), dtype=np.int32)
        E = np.zeros((na.value, 27, 6, 6), dtype=np.float32)
        feat = np.zeros((na.value, 8), dtype=np.float32)
        _check(lib().ofea_learned_level(self.h, ctypes.byref(na), _ptr(nbr), _ptr(E), _ptr(feat)),
               "ofea_learned_level")
        return nbr, E, feat

    def learned_gradient(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = _LL()
        _check(lib().ofea_learned_get_weights(self.h, None, ctypes.byref(n)), "ofea_learned_get_weights")
        g = np.zeros(n.value, dtype=np.float32)
        loss = _D()
        _check(lib().ofea_learned_gradient(self.h, _ptr(x), x.shape[0], ctypes.byref(loss), _ptr(g)),
               "ofea_learned_gradient")
        return loss.value, g

    def solve_device(self, f_ptr, u_ptr, method="GPU_PCG", rtol=1e-8, **kw):
        o = solve_opts(method, rtol, **kw)
        st = SolveStats()
        rc = lib().ofea_solve_device(self.h, _P(f_ptr), _P(u_ptr), ctypes.byref(o), ctypes.byref(st))
        return rc, st.as_dict()


# --------------------------------------------------------------- host I/O --

def inp_read(path):
    """ReadInfo (src/data2cae.cpp) through the C ABI; returns a dict of arrays."""
    L = lib()
    m = _P()
    _check(L.ofea_inp_read(str(path).encode(), ctypes.byref(m)), "ofea_inp_read")
    try:
        nd, ne, nfix, nload = _I(), _I(), _I(), _I()
        L.ofea_model_sizes(m, ctypes.byref(nd), ctypes.byref(ne), ctypes.byref(nfix), ctypes.byref(nload))
        xyz = np.zeros((nd.value, 3))
        topo = np.zeros((ne.value, 8), dtype=np.int32)
        et = np.zeros(ne.value, dtype=np.int32)
        fix = np.zeros(nfix.value, dtype=np.int32)
        load = np.zeros(nload.value, dtype=np.int32)
        L.ofea_model_arrays(m, _ptr(xyz), _ptr(topo), _ptr(et), _ptr(fix), _ptr(load))
        E, nu, rho, has = _D(), _D(), _D(), _I()
        L.ofea_model_material(m, ctypes.byref(E), ctypes.byref(nu), ctypes.byref(rho), ctypes.byref(has))
        dof, val = _I(), _D()
        L.ofea_model_cload(m, ctypes.byref(dof), ctypes.byref(val))
        return dict(xyz=xyz, topo=topo, etype=et, fix=fix, load_set=load, E=E.value, nu=nu.value,
                    density=rho.value, has_elastic=bool(has.value), load_dof=dof.value,
                    load_value=val.value)
    finally:
        L.ofea_model_free(m)


def ca_info_read(path):
    """The CA change file (ReadInfo::CA_read_change, src/data2cae.cpp:520-661):
    modified coordinates of every original node, the changed elements (kind 0
    deleted, 1 moved, 2 added; etype; 0-based topology, -1 padded) and the
    original-to-modified node map (-1: removed)."""
    L = lib()
    nd, nc = _I(), _I()
    _check(L.ofea_ca_info_read(str(path).encode(), ctypes.byref(nd), ctypes.byref(nc), None, None, None, None, None),
           "ofea_ca_info_read")
    xyz = np.zeros((nd.value, 3))
    kind = np.zeros(nc.value, dtype=np.int32)
    et = np.zeros(nc.value, dtype=np.int32)
    topo = np.zeros((nc.value, 8), dtype=np.int32)
    nmap = np.zeros(nd.value, dtype=np.int32)
    _check(L.ofea_ca_info_read(str(path).encode(), ctypes.byref(nd), ctypes.byref(nc), _ptr(xyz), _ptr(kind),
                               _ptr(et), _ptr(topo), _ptr(nmap)), "ofea_ca_info_read")
    return dict(xyz=xyz, kind=kind, etype=et, topo=topo, node_map=nmap)


def ca_reanalysis(base, modified, f, u0=None, n_basis=4, method="GPU_PCG", rtol=1e-10, **kw):
    """Combined-approximations reanalysis (ofea_ca_reanalysis): the CA
    solution of the modified model from n_basis basis vectors built with the
    base model's K.  Returns (u, stats)."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    u = np.zeros(base.n)
    u0p = None
    if u0 is not None:
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        u0p = u0.ctypes.data
    o = solve_opts(method, rtol, **kw)
    st = CaStats()
    _check(lib().ofea_ca_reanalysis(base.h, modified.h, f.ctypes.data, u0p, int(n_basis), ctypes.byref(o),
                                    u.ctypes.data, ctypes.byref(st)), "ofea_ca_reanalysis")
    return u, st.as_dict()


def build_free_index(nd, fix):
    fix = _i32(fix)
    fm = np.zeros(nd, dtype=np.int32)
    nf = _I()
    _check(lib().ofea_build_free_index(nd, fix.size, _ptr(fix), _ptr(fm), ctypes.byref(nf)),
           "ofea_build_free_index")
    return fm


def build_single_load(nd, free_map, load_set, dof, value):
    fm, ls = _i32(free_map), _i32(load_set)
    f = np.zeros(3 * int((fm >= 0).sum()))
    _check(lib().ofea_build_single_load(nd, _ptr(fm), ls.size, _ptr(ls), dof, value, _ptr(f)),
           "ofea_build_single_load")
    return f


def full_displacement(nd, free_map, u):
    out = np.zeros(3 * nd)
    _check(lib().ofea_full_displacement(nd, _ptr(_i32(free_map)), _ptr(_f64(u)), _ptr(out)),
           "ofea_full_displacement")
    return out


def write_vtk(path, xyz, topo, etype, u_full, scale=1.0, node_stress=None):
    """export_dis_2_vtk (src/data2vtk.cpp:47-264); node_stress (7, nd) adds the
    S_xx .. S_Mises fields (ofea_write_vtk_stress)."""
    xyz, topo, et, uf = _f64(xyz), _i32(topo), _i32(etype), _f64(u_full)
    if node_stress is None:
        _check(lib().ofea_write_vtk(str(path).encode(), xyz.shape[0], _ptr(xyz), topo.shape[0], _ptr(topo),
                                    _ptr(et), _ptr(uf), scale), "ofea_write_vtk")
    else:
        ns = _f64(node_stress)
        _check(lib().ofea_write_vtk_stress(str(path).encode(), xyz.shape[0], _ptr(xyz), topo.shape[0], _ptr(topo),
                                           _ptr(et), _ptr(uf), scale, _ptr(ns)), "ofea_write_vtk_stress")


# ------------------------------------------- reference-named entry points --

@dataclass
class DataManagement:
    """The fields of data_management (src/include/data_management.h:48-62)
    that the assembly and solve entry points read and write."""
    nd_: int
    ne_: int
    coords_: np.ndarray          # nd x 3
    node_topos_: np.ndarray      # ne x 8, 1-based
    ele_list_idx_: np.ndarray    # 0 C3D4, 1 C3D8
    dis_bc_set_: np.ndarray      # 1-based fixed nodes
    young_modulus: float
    poisson_ratio: float
    E_elem: np.ndarray | None = None
    resort_free_nodes_: np.ndarray | None = None
    single_load_vec_: np.ndarray | None = None
    single_dis_vec_: np.ndarray | None = None


class AssambleStiffness:
    """assamble_stiffness (src/include/assemble.h:35-72) with K on the GPU."""

    def __init__(self, device=0):
        self.ctx = Context(device)
        self.num_nz_val_ = 0

    def build_CSR(self, data: DataManagement):
        if data.resort_free_nodes_ is None:
            data.resort_free_nodes_ = build_free_index(data.nd_, data.dis_bc_set_)
        self.ctx.upload(data.coords_, data.node_topos_, data.ele_list_idx_, data.resort_free_nodes_,
                        data.young_modulus, data.poisson_ratio, data.E_elem)
        n, nnz = self.ctx.assemble_pattern()
        self.num_nz_val_ = nnz
        return n, nnz

    def fill_CSR_sparse_mat(self, data: DataManagement):
        self.ctx.assemble_linear()

    def csr(self):
        return self.ctx.get_csr()


def solution_api(item_ass: AssambleStiffness, data: DataManagement, solver_type: str, rtol=1e-8):
    """solution_api (src/linear_solution.cpp:17-64) with the GPU solvers:
    "GPU_PCG" (FP64), "GPU_MIXED" or "GPU_LEARNED" (after learned_train).  Returns False for an unknown solver
    string, as the reference does; raises on solver failure (the reference
    exits)."""
    if solver_type not in ("GPU_PCG", "GPU_MIXED", "GPU_LEARNED"):
        return False
    u, st = item_ass.ctx.solve(data.single_load_vec_, method=solver_type, rtol=rtol)
    data.single_dis_vec_ = u
    item_ass.last_stats = st
    return True
