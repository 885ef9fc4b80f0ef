"""ctypes wrapper of the CPU oracle (oracle/oracle.cpp) -- test infrastructure.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline /
reference arm import this module, and only to check or time the product; the
product (``dendro_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")

OCT_DTYPE = np.dtype([("x", "<u4"), ("y", "<u4"), ("z", "<u4"), ("lf", "<u4")])


def build(force: bool = False) -> str:
    """Compile oracle.cpp into liboracle.so beside it (g++ -O2 -fopenmp)."""
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", src, "-o", _SO])
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        P = C.c_void_p
        i64p = C.POINTER(C.c_int64)
        L.orc_points2octree.argtypes = [P, C.c_int64, C.c_uint32, C.c_uint32, C.POINTER(P), i64p]
        L.orc_balance.argtypes = [P, C.c_int64, C.c_uint32, C.POINTER(P), i64p]
        L.orc_coarsen.argtypes = [P, C.c_int64, C.c_uint32, C.POINTER(P), i64p]
        L.orc_is_sorted_linear.argtypes = [P, C.c_int64]
        L.orc_free.argtypes = [P]
        L.orc_mesh_create.argtypes = [P, C.c_int64, C.c_uint32, C.POINTER(C.c_int)]
        L.orc_mesh_create.restype = P
        L.orc_mesh_destroy.argtypes = [P]
        L.orc_mesh_sizes.argtypes = [P, i64p, i64p, i64p]
        L.orc_mesh_export.argtypes = [P] * 9
        L.orc_matvec.argtypes = [P, P, P, P]
        L.orc_matvec_elems.argtypes = [P, P, P, P, P, C.c_int64]
        L.orc_diagonal.argtypes = [P, P, P]
        L.orc_load_vector.argtypes = [P, P, P]
        L.orc_rhs_table.argtypes = [P]
        L.orc_elasticity_matvec.argtypes = [P, C.c_double, C.c_double, P, P, P]
        L.orc_stencils.argtypes = [P, P, P]
        L.orc_hanging_T.argtypes = [C.c_uint32, C.c_uint32, P]
        L.orc_prolongation.argtypes = [P, P, C.POINTER(P), C.POINTER(P), C.POINTER(P), i64p]
        L.orc_coarse_coef.argtypes = [P, P, P, P]
        L.orc_damg_create.argtypes = [P, C.c_int64, C.c_uint32, C.c_int, P, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]
        L.orc_damg_create.restype = P
        L.orc_damg_create_dof.argtypes = [P, C.c_int64, C.c_uint32, C.c_int, P, C.c_int, C.c_double, C.c_double,
                                          C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_damg_create_dof.restype = P
        L.orc_damg_destroy.argtypes = [P]
        L.orc_damg_level_sizes.argtypes = [P, P, P]
        L.orc_damg_level_mesh.argtypes = [P, C.c_int]
        L.orc_damg_level_mesh.restype = P
        L.orc_damg_vcycle.argtypes = [P, P, P]
        L.orc_damg_pcg.argtypes = [P, P, P, C.c_double, C.c_int, P]
        L.orc_damg_set_coarse_op.argtypes = [P, C.c_int]
        L.orc_damg_level_apply.argtypes = [P, C.c_int, P, P]
        L.orc_type1_stencils.argtypes = [P, P]
        L.orc_jacobian3.argtypes = [P, P, P, P, P]
        L.orc_dirichlet_matvec.argtypes = [P, C.c_int, P, P, P]
        L.orc_dirichlet_diagonal.argtypes = [P, C.c_int, P, P]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _take_octs(p, n):
    out = np.empty(n.value, OCT_DTYPE)
    if n.value:
        C.memmove(out.ctypes.data, p.value, n.value * 16)
    lib().orc_free(p)
    return out


def points2octree(pts: np.ndarray, max_depth: int, max_num_pts: int = 1) -> np.ndarray:
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    p, n = C.c_void_p(), C.c_int64()
    rc = lib().orc_points2octree(_ptr(pts), len(pts), max_depth, max_num_pts, C.byref(p), C.byref(n))
    if rc:
        raise ValueError("oracle points2octree failed: %d" % rc)
    return _take_octs(p, n)


def balance(octs: np.ndarray, max_depth: int) -> np.ndarray:
    octs = np.ascontiguousarray(octs, OCT_DTYPE)
    p, n = C.c_void_p(), C.c_int64()
    lib().orc_balance(_ptr(octs), len(octs), max_depth, C.byref(p), C.byref(n))
    return _take_octs(p, n)


def coarsen(octs: np.ndarray, max_depth: int) -> np.ndarray:
    octs = np.ascontiguousarray(octs, OCT_DTYPE)
    p, n = C.c_void_p(), C.c_int64()
    lib().orc_coarsen(_ptr(octs), len(octs), max_depth, C.byref(p), C.byref(n))
    return _take_octs(p, n)


def is_sorted_linear(octs: np.ndarray) -> bool:
    octs = np.ascontiguousarray(octs, OCT_DTYPE)
    return bool(lib().orc_is_sorted_linear(_ptr(octs), len(octs)))


class Mesh:
    """Oracle mesh of one level (embedded octree, boundary pseudo-octants, DA maps)."""

    def __init__(self, octs: np.ndarray, max_depth: int, handle=None, owner=None):
        self._owner = owner
        if handle is None:
            octs = np.ascontiguousarray(octs, OCT_DTYPE)
            st = C.c_int()
            handle = lib().orc_mesh_create(_ptr(octs), len(octs), max_depth, C.byref(st))
            if not handle:
                raise ValueError("oracle mesh build failed: %d" % st.value)
        self.h = handle
        E, N, no = C.c_int64(), C.c_int64(), C.c_int64()
        lib().orc_mesh_sizes(self.h, C.byref(E), C.byref(N), C.byref(no))
        self.E, self.N, self.n_oct = E.value, N.value, no.value
        self.nlist = np.empty((self.E, 8), np.uint32)
        self.hmask = np.empty(self.E, np.uint8)
        self.cnum = np.empty(self.E, np.uint8)
        self.etype = np.empty(self.E, np.uint8)
        self.elev = np.empty(self.E, np.uint8)
        self.node_xyz = np.empty((self.N, 3), np.uint32)
        self.node_bdy = np.empty(self.N, np.uint8)
        self.octs = np.empty(self.n_oct, OCT_DTYPE)
        lib().orc_mesh_export(self.h, *[_ptr(a) for a in (self.nlist, self.hmask, self.cnum, self.etype,
                                                         self.elev, self.node_xyz, self.node_bdy,
                                                         self.octs)])

    def __del__(self):
        if getattr(self, "h", None) and self._owner is None and _lib is not None:
            _lib.orc_mesh_destroy(self.h)
            self.h = None

    def matvec(self, x, coef=None):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.N, np.float64)
        c = None if coef is None else np.ascontiguousarray(coef, np.float64)
        lib().orc_matvec(self.h, _ptr(c), _ptr(x), _ptr(y))
        return y

    def matvec_elems(self, x, elems, coef=None):
        """The matvec's sum over the listed elements only (global node ids)."""
        x = np.ascontiguousarray(x, np.float64)
        e = np.ascontiguousarray(elems, np.int64)
        y = np.zeros(self.N, np.float64)
        c = None if coef is None else np.ascontiguousarray(coef, np.float64)
        lib().orc_matvec_elems(self.h, _ptr(c), _ptr(x), _ptr(y), _ptr(e), len(e))
        return y

    def load_vector(self, force):
        """ComputeRHS_omgNeumann (omgNeumann.C:749-785): force per element (at its centre) -> b."""
        f = np.ascontiguousarray(force, np.float64)
        b = np.empty(self.N, np.float64)
        lib().orc_load_vector(self.h, _ptr(f), _ptr(b))
        return b

    def diagonal(self, coef=None):
        d = np.empty(self.N, np.float64)
        c = None if coef is None else np.ascontiguousarray(coef, np.float64)
        lib().orc_diagonal(self.h, _ptr(c), _ptr(d))
        return d

    def dirichlet_matvec(self, x, bdy, mass: bool):
        """DirichletLaplacianMatMult (mass False) / DirichletJacobianMatMult."""
        x = np.ascontiguousarray(x, np.float64)
        b = np.ascontiguousarray(bdy, np.uint8)
        y = np.empty_like(x)
        lib().orc_dirichlet_matvec(self.h, int(mass), _ptr(b), _ptr(x), _ptr(y))
        return y

    def dirichlet_diagonal(self, bdy, mass: bool):
        b = np.ascontiguousarray(bdy, np.uint8)
        d = np.empty(self.N)
        lib().orc_dirichlet_diagonal(self.h, int(mass), _ptr(b), _ptr(d))
        return d

    def elasticity_matvec(self, x, mu, lam, bdy=None):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(3 * self.N, np.float64)
        b = np.ascontiguousarray(self.node_bdy if bdy is None else bdy, np.uint8)
        lib().orc_elasticity_matvec(self.h, mu, lam, _ptr(b), _ptr(x), _ptr(y))
        return y


def stencils():
    L = np.empty((8, 18, 8, 8))
    M = np.empty((8, 18, 8, 8))
    G = np.empty((8, 18, 24, 24))
    lib().orc_stencils(_ptr(L), _ptr(M), _ptr(G))
    return L, M, G


def type1_stencils():
    """The oracle's type-1 tables (L1, M1), each [8][18][8][8][8]:
    [coarse child number][element type][fine child][i][j]."""
    L = np.empty((8, 18, 8, 8, 8))
    M = np.empty((8, 18, 8, 8, 8))
    lib().orc_type1_stencils(_ptr(L), _ptr(M))
    return L, M


def jacobian3(fine: Mesh, fine_coef, coarse: Mesh, x):
    """Jacobian3MatMult (examples/src/backend/omgJac.C:2235): the coarse mesh's
    operator from the fine mesh's coefficients (a, b per element)."""
    fc = np.ascontiguousarray(fine_coef, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty_like(x)
    if lib().orc_jacobian3(fine.h, _ptr(fc), coarse.h, _ptr(x), _ptr(y)):
        raise ValueError("coarse element without fine elements")
    return y


def prolongation(fine: Mesh, coarse: Mesh):
    """CSR (ptr, col, val) of P: fine nodes x coarse nodes."""
    p, c, v, nnz = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_int64()
    rc = lib().orc_prolongation(fine.h, coarse.h, C.byref(p), C.byref(c), C.byref(v), C.byref(nnz))
    if rc:
        raise ValueError("oracle prolongation failed: %d" % rc)
    ptr = np.empty(fine.N + 1, np.int64)
    col = np.empty(nnz.value, np.uint32)
    val = np.empty(nnz.value, np.float64)
    C.memmove(ptr.ctypes.data, p.value, 8 * (fine.N + 1))
    C.memmove(col.ctypes.data, c.value, 4 * nnz.value)
    C.memmove(val.ctypes.data, v.value, 8 * nnz.value)
    for q in (p, c, v):
        lib().orc_free(q)
    return ptr, col, val


def rhs_table() -> np.ndarray:
    """RHSType2Stencil [childNum][elemType][vertex] as the oracle derives it (T^T 1)."""
    out = np.empty((8, 18, 8))
    lib().orc_rhs_table(_ptr(out))
    return out


def coarse_coef(fine: Mesh, fine_coef, coarse: Mesh):
    out = np.empty(2 * coarse.E)
    fc = np.ascontiguousarray(fine_coef, np.float64)
    rc = lib().orc_coarse_coef(fine.h, _ptr(fc), coarse.h, _ptr(out))
    if rc:
        raise ValueError("coarse coefficient mapping failed")
    return out


class DAMG:
    """Oracle multigrid hierarchy + FP64 PCG/V(2,2) solver."""

    def __init__(self, finest: np.ndarray, max_depth: int, nlevels: int, coef=None, dof: int = 1,
                 mu: float = 1.0, lam: float = 1.0):
        """dof 3: linear elasticity (mu, lam) on every level, each level's
        boundary nodes Dirichlet, as the reference's elasticity driver."""
        finest = np.ascontiguousarray(finest, OCT_DTYPE)
        st, nl = C.c_int(), C.c_int()
        c = None if coef is None else np.ascontiguousarray(coef, np.float64)
        self.dof = int(dof)
        self.h = lib().orc_damg_create_dof(_ptr(finest), len(finest), max_depth, nlevels, _ptr(c), self.dof,
                                           float(mu), float(lam), C.byref(st), C.byref(nl))
        if not self.h:
            raise ValueError("oracle DAMG create failed: %d" % st.value)
        self.nlevels = nl.value
        E = np.empty(self.nlevels, np.int64)
        N = np.empty(self.nlevels, np.int64)
        lib().orc_damg_level_sizes(self.h, _ptr(E), _ptr(N))
        self.E, self.N = E, N

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_damg_destroy(self.h)
            self.h = None

    def level_mesh(self, l: int) -> Mesh:
        return Mesh(None, 0, handle=lib().orc_damg_level_mesh(self.h, l), owner=self)

    def set_coarse_op(self, op: int):
        """1: Jacobian3 below the finest level (J), Jacobi diagonal from the
        level's own averaged coefficients (B); 0: type 2 throughout."""
        if lib().orc_damg_set_coarse_op(self.h, op):
            raise ValueError("coarsest operator not positive definite")

    def level_apply(self, l: int, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        lib().orc_damg_level_apply(self.h, l, _ptr(x), _ptr(y))
        return y

    def vcycle(self, b):
        b = np.ascontiguousarray(b, np.float64)
        x = np.empty_like(b)
        lib().orc_damg_vcycle(self.h, _ptr(b), _ptr(x))
        return x

    def pcg(self, b, rtol=1e-8, maxit=200):
        b = np.ascontiguousarray(b, np.float64)
        x = np.empty_like(b)
        hist = np.zeros(maxit + 1)
        it = lib().orc_damg_pcg(self.h, _ptr(b), _ptr(x), rtol, maxit, _ptr(hist))
        n = abs(it)
        return x, it, hist[: n + 1]


def partition_weighted(weights, nranks: int) -> np.ndarray:
    """par::partitionW (include/par/parUtils.txx:1011-1177) for a list held by
    one rank, as item ranges: rank r receives items first[r] .. first[r+1]-1.
    The rule (parUtils.txx:1130-1150): with the inclusive weight scan s, the
    total W, avgLoad = W // P and extra = W % P, an item goes to rank 0 when
    s == 0, to (s - 1) // (avgLoad + 1) while s <= extra * (avgLoad + 1), else
    to (s - 1 - extra) // avgLoad; with avgLoad == 0 all items go to rank 0
    (parUtils.txx:1175-1176)."""
    w = [int(v) for v in weights]
    cnt = [0] * nranks
    total = sum(w)
    avg, extra = total // nranks, total % nranks
    if avg == 0:
        cnt[0] = len(w)
    else:
        s = 0
        for v in w:
            s += v
            if s == 0:
                r = 0
            elif s <= extra * (avg + 1):
                r = (s - 1) // (avg + 1)
            else:
                r = (s - 1 - extra) // avg
            cnt[r] += 1
    return np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
