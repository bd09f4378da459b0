"""ctypes access to the oracle libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, where it is the checker, never the product.

* ``Oracle`` wraps liboracle.so, the C restatement (ofea_oracle.c).
* ``Reference`` wraps _ref/libofea_ref.so, the reference's own hot-path code
  compiled from its sources by this directory's Makefile; absent where the
  reference tree was never available to build it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_LL = ctypes.c_longlong


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    def __init__(self, path=None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle oracle)")
        L = ctypes.CDLL(path)
        L.orc_build_free_index.restype = _I
        L.orc_build_free_index.argtypes = [_I, _I, _P, _P]
        for nm in ("orc_c3d8_ke", "orc_c3d4_ke"):
            getattr(L, nm).restype = _D
            getattr(L, nm).argtypes = [_P, _D, _D, _P]
        for nm in ("orc_c3d8_nl", "orc_c3d4_nl"):
            getattr(L, nm).restype = None
            getattr(L, nm).argtypes = [_P, _P, _D, _D, _P, _P]
        L.orc_pattern_count.restype = _LL
        L.orc_pattern_count.argtypes = [_I, _I, _P, _P, _P, _I, _P]
        L.orc_pattern_fill.argtypes = [_I, _I, _P, _P, _P, _I, _P, _P]
        L.orc_fill.argtypes = [_I, _P, _I, _P, _P, _P, _P, _D, _D, _P, _P, _P]
        L.orc_nl_fill.argtypes = [_I, _P, _I, _P, _P, _P, _P, _D, _D, _P, _P, _P, _P, _P]
        L.orc_spmv.argtypes = [_I, _P, _P, _P, _P, _P]
        L.orc_pcg.restype = _I
        L.orc_pcg.argtypes = [_I, _P, _P, _P, _P, _P, _D, _I, _P, _P]
        L.orc_full_displacement.argtypes = [_I, _P, _P, _P]
        self.L = L

    def free_index(self, nd, fix):
        fix = _i32(fix)
        fm = np.zeros(nd, dtype=np.int32)
        nf = self.L.orc_build_free_index(nd, fix.size, _ptr(fix), _ptr(fm))
        if nf < 0:
            raise ValueError("invalid fixed-node set")
        return fm

    def element_ke(self, etype, coords, E, nu):
        X = _f64(coords)
        npe = 8 if etype == 1 else 4
        K = np.zeros((3 * npe, 3 * npe))
        fn = self.L.orc_c3d8_ke if etype == 1 else self.L.orc_c3d4_ke
        det = fn(_ptr(X), E, nu, _ptr(K))
        return K, det

    def element_nl(self, etype, coords, u_el, E, nu):
        X, U = _f64(coords), _f64(u_el)
        npe = 8 if etype == 1 else 4
        K = np.zeros((3 * npe, 3 * npe))
        f = np.zeros(3 * npe)
        fn = self.L.orc_c3d8_nl if etype == 1 else self.L.orc_c3d4_nl
        fn(_ptr(X), _ptr(U), E, nu, _ptr(K), _ptr(f))
        return K, f

    def pattern(self, mesh, fm):
        topo, et = _i32(mesh.topo), _i32(mesh.etype)
        n = 3 * int((fm >= 0).sum())
        cp = np.zeros(n + 1, dtype=np.int32)
        nnz = self.L.orc_pattern_count(mesh.nd, mesh.ne, _ptr(topo), _ptr(et), _ptr(fm), n, _ptr(cp))
        ri = np.zeros(nnz, dtype=np.int32)
        self.L.orc_pattern_fill(mesh.nd, mesh.ne, _ptr(topo), _ptr(et), _ptr(fm), n, _ptr(cp), _ptr(ri))
        return cp, ri

    def assemble(self, mesh, fm):
        """Pattern + fill; returns (col_ptr, row_idx, val) in the reference's CSC layout."""
        cp, ri = self.pattern(mesh, fm)
        val = np.zeros(ri.size)
        xyz, topo, et = _f64(mesh.xyz), _i32(mesh.topo), _i32(mesh.etype)
        E = _f64(mesh.E) if mesh.E is not None else None
        self.L.orc_fill(mesh.nd, _ptr(xyz), mesh.ne, _ptr(topo), _ptr(et), _ptr(fm), _ptr(E),
                        mesh.E0, mesh.nu, _ptr(cp), _ptr(ri), _ptr(val))
        return cp, ri, val

    def nl_assemble(self, mesh, fm, cp, ri, u):
        val = np.zeros(ri.size)
        fint = np.zeros(cp.size - 1)
        xyz, topo, et, u = _f64(mesh.xyz), _i32(mesh.topo), _i32(mesh.etype), _f64(u)
        E = _f64(mesh.E) if mesh.E is not None else None
        self.L.orc_nl_fill(mesh.nd, _ptr(xyz), mesh.ne, _ptr(topo), _ptr(et), _ptr(fm), _ptr(E),
                           mesh.E0, mesh.nu, _ptr(u), _ptr(cp), _ptr(ri), _ptr(val), _ptr(fint))
        return val, fint

    def spmv(self, cp, ri, val, x):
        y = np.zeros(cp.size - 1)
        x = _f64(x)
        self.L.orc_spmv(cp.size - 1, _ptr(cp), _ptr(ri), _ptr(val), _ptr(x), _ptr(y))
        return y

    def pcg(self, cp, ri, val, f, rtol=1e-12, max_iter=200000):
        f = _f64(f)
        u = np.zeros(f.size)
        it, rr = _I(0), _D(0.0)
        st = self.L.orc_pcg(f.size, _ptr(cp), _ptr(ri), _ptr(val), _ptr(f), _ptr(u), rtol,
                            max_iter, ctypes.byref(it), ctypes.byref(rr))
        return u, st, it.value, rr.value


class Reference:
    """The reference's own code (oracle/_ref/libofea_ref.so)."""

    PATH = os.path.join(HERE, "_ref", "libofea_ref.so")

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def __init__(self):
        if not self.available():
            raise FileNotFoundError(f"{self.PATH} not built (make -C oracle ref)")
        L = ctypes.CDLL(self.PATH)
        L.ref_model_create.restype = _P
        L.ref_model_create.argtypes = [_I, _P, _I, _P, _P, _P, _D, _D, _I, _P]
        L.ref_model_from_inp.restype = _P
        L.ref_model_from_inp.argtypes = [ctypes.c_char_p, _I, _D, _D]
        L.ref_model_destroy.argtypes = [_P]
        L.ref_model_sizes.argtypes = [_P, _P, _P, _P]
        L.ref_model_mesh.argtypes = [_P, _P, _P, _P, _P, _P, _P]
        L.ref_model_set_load.argtypes = [_P, _P]
        L.ref_model_assemble.restype = _LL
        L.ref_model_assemble.argtypes = [_P]
        L.ref_model_get_csc.argtypes = [_P, _P, _P, _P]
        L.ref_model_solve.restype = _I
        L.ref_model_solve.argtypes = [_P, _P]
        L.ref_model_full_displacement.argtypes = [_P, _P]
        L.ref_model_times.argtypes = [_P, _P]
        L.ref_model_nl_assemble.restype = _LL
        L.ref_model_nl_assemble.argtypes = [_P, _P, _P]
        L.ref_model_nl_get_csc.argtypes = [_P, _P, _P, _P]
        L.ref_model_nl_solve.restype = _I
        L.ref_model_nl_solve.argtypes = [_P, _P, _P]
        L.ref_model_solve_multi.restype = _I
        L.ref_model_solve_multi.argtypes = [_P, _I, _P, _P]
        L.ref_model_cg_ic_setup.restype = _D
        L.ref_model_cg_ic_setup.argtypes = [_P, _I]
        L.ref_model_cg_ic_run.restype = _I
        L.ref_model_cg_ic_run.argtypes = [_P, _P, _P, _D, _I, _P]
        L.ref_element_ke.argtypes = [_I, _P, _D, _D, _P]
        L.ref_element_nl.argtypes = [_I, _P, _P, _D, _D, _P, _P]
        self.L = L

    def element_ke(self, etype, coords, E, nu):
        X = _f64(coords)
        npe = 8 if etype == 1 else 4
        K = np.zeros((3 * npe, 3 * npe))
        self.L.ref_element_ke(etype, _ptr(X), E, nu, _ptr(K))
        return K

    def element_nl(self, etype, coords, u_el, E, nu):
        X, U = _f64(coords), _f64(u_el)
        npe = 8 if etype == 1 else 4
        K = np.zeros((3 * npe, 3 * npe))
        f = np.zeros(3 * npe)
        self.L.ref_element_nl(etype, _ptr(X), _ptr(U), E, nu, _ptr(K), _ptr(f))
        return K, f

    def model(self, mesh):
        return RefModel(self, mesh=mesh)

    def model_from_inp(self, path, E=None, nu=None):
        return RefModel(self, inp=path, E=E, nu=nu)


class RefModel:
    def __init__(self, ref, mesh=None, inp=None, E=None, nu=None):
        self.r = ref
        L = ref.L
        if mesh is not None:
            xyz, topo, et, fix = _f64(mesh.xyz), _i32(mesh.topo), _i32(mesh.etype), _i32(mesh.fix)
            Ee = _f64(mesh.E) if mesh.E is not None else None
            self.h = L.ref_model_create(mesh.nd, _ptr(xyz), mesh.ne, _ptr(topo), _ptr(et), _ptr(Ee),
                                        mesh.E0, mesh.nu, fix.size, _ptr(fix))
        else:
            ov = 1 if E is not None else 0
            self.h = L.ref_model_from_inp(inp.encode(), ov, E or 0.0, nu or 0.0)
        nd, ne, n = _I(), _I(), _I()
        L.ref_model_sizes(self.h, ctypes.byref(nd), ctypes.byref(ne), ctypes.byref(n))
        self.nd, self.ne, self.n = nd.value, ne.value, n.value

    def __del__(self):
        try:
            self.r.L.ref_model_destroy(self.h)
        except Exception:
            pass

    def mesh_arrays(self):
        xyz = np.zeros((self.nd, 3))
        topo = np.zeros((self.ne, 8), dtype=np.int32)
        et = np.zeros(self.ne, dtype=np.int32)
        fm = np.zeros(self.nd, dtype=np.int32)
        f = np.zeros(self.n)
        Enu = np.zeros(2)
        self.r.L.ref_model_mesh(self.h, _ptr(xyz), _ptr(topo), _ptr(et), _ptr(fm), _ptr(f), _ptr(Enu))
        return dict(xyz=xyz, topo=topo, etype=et, free_map=fm, f=f, E=Enu[0], nu=Enu[1])

    def set_load(self, f):
        f = _f64(f)
        assert f.size == self.n
        self.r.L.ref_model_set_load(self.h, _ptr(f))

    def assemble(self):
        nnz = self.r.L.ref_model_assemble(self.h)
        cp = np.zeros(self.n + 1, dtype=np.int32)
        ri = np.zeros(nnz, dtype=np.int32)
        val = np.zeros(nnz)
        self.r.L.ref_model_get_csc(self.h, _ptr(cp), _ptr(ri), _ptr(val))
        return cp, ri, val

    def solve(self):
        u = np.zeros(self.n)
        st = self.r.L.ref_model_solve(self.h, _ptr(u))
        if st != 0:
            raise RuntimeError("reference solve failed")
        return u

    def solve_multi(self, F):
        """Load cases F (nrhs, n) on one factor: solution_api("SuperLU_class")
        for the first, superlu_solution_next for the rest."""
        F = np.ascontiguousarray(np.atleast_2d(F), dtype=np.float64)
        assert F.shape[1] == self.n
        U = np.zeros_like(F)
        if self.r.L.ref_model_solve_multi(self.h, F.shape[0], _ptr(F), _ptr(U)) != 0:
            raise RuntimeError("reference SuperLU_class solve failed")
        return U

    def cg_ic_setup(self, threads=1):
        """Vendored Eigen IncompleteCholesky of the reference-assembled K
        (call assemble() first); returns the set-up seconds."""
        t = self.r.L.ref_model_cg_ic_setup(self.h, threads)
        if t < 0:
            raise RuntimeError(f"Eigen IC set-up failed ({t})")
        return t

    def cg_ic_run(self, f, rtol=1e-10, max_iter=100000, u0=None):
        """One Eigen ConjugateGradient solve (FP64) with the IC factor of
        cg_ic_setup, started from u0 (zero)."""
        f = _f64(f)
        u = np.zeros(self.n) if u0 is None else _f64(u0).copy()
        out = np.zeros(4)
        if self.r.L.ref_model_cg_ic_run(self.h, _ptr(f), _ptr(u), rtol, max_iter, _ptr(out)) != 0:
            raise RuntimeError("Eigen CG: no IC set-up")
        return u, dict(iterations=int(out[0]), est_rel_residual=out[1], rel_residual=out[2], cg_s=out[3])

    def cg_ic(self, f, rtol=1e-10, max_iter=100000, threads=1, u0=None):
        """IC set-up + one CG solve; the stats carry both times."""
        t = self.cg_ic_setup(threads)
        u, st = self.cg_ic_run(f, rtol, max_iter, u0)
        st.update(setup_s=t, threads=threads, ordering="natural")
        return u, st

    def full_displacement(self):
        uf = np.zeros(3 * self.nd)
        self.r.L.ref_model_full_displacement(self.h, _ptr(uf))
        return uf

    def times(self):
        t = np.zeros(3)
        self.r.L.ref_model_times(self.h, _ptr(t))
        return dict(build_csr=t[0], fill=t[1], solve=t[2])

    def nl_assemble(self, u):
        fint = np.zeros(self.n)
        u = _f64(u)
        nnz = self.r.L.ref_model_nl_assemble(self.h, _ptr(u), _ptr(fint))
        cp = np.zeros(self.n + 1, dtype=np.int32)
        ri = np.zeros(nnz, dtype=np.int32)
        val = np.zeros(nnz)
        self.r.L.ref_model_nl_get_csc(self.h, _ptr(cp), _ptr(ri), _ptr(val))
        return cp, ri, val, fint

    def nl_solve(self, b):
        b = _f64(b)
        x = np.zeros(self.n)
        self.r.L.ref_model_nl_solve(self.h, _ptr(b), _ptr(x))
        return x
