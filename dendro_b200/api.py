"""Python classes over the C ABI, named after the reference's interfaces.

Arrays may be numpy (host) or torch CUDA tensors (device); the operators take
device tensors for the resident path and host arrays for the end-to-end path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import OCT_DTYPE, DamgConfig, SolveReport, check, lib, ptr


def _is_device(a) -> bool:
    return not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)


class Octree:
    """Device-resident sorted linear octree (a vector<ot::TreeNode>)."""

    def __init__(self, handle):
        self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().dg_octree_destroy(self.h)
            self.h = None

    def __len__(self):
        return int(lib().dg_octree_size(self.h))

    @property
    def maxDepth(self) -> int:
        return int(lib().dg_octree_max_depth(self.h))

    def to_numpy(self) -> np.ndarray:
        out = np.empty(len(self), OCT_DTYPE)
        check(lib().dg_octree_export(self.h, ptr(out)), "octree_export")
        return out

    @classmethod
    def from_octants(cls, octs, maxDepth: int) -> "Octree":
        h = C.c_void_p()
        if _is_device(octs):
            check(lib().dg_octree_from_octants(ptr(octs), octs.numel() // 4, 1, maxDepth, C.byref(h)),
                  "octree_from_octants")
        else:
            a = np.ascontiguousarray(octs, OCT_DTYPE)
            check(lib().dg_octree_from_octants(ptr(a), len(a), 0, maxDepth, C.byref(h)), "octree_from_octants")
        return cls(h)


def points2Octree(pts, maxDepth: int, maxNumPts: int = 1) -> Octree:
    """ot::points2Octree (src/oct/Construct.C:727): points in [0,1)^3 -> octree."""
    h = C.c_void_p()
    if _is_device(pts):
        n = pts.numel() // 3
        check(lib().dg_points2octree(ptr(pts), n, 1, maxDepth, maxNumPts, C.byref(h)), "points2octree")
    else:
        a = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        check(lib().dg_points2octree(ptr(a), len(a), 0, maxDepth, maxNumPts, C.byref(h)), "points2octree")
    return Octree(h)


def writePtsToFile(path, pts) -> None:
    """ot::writePtsToFile (src/oct/OctFunctions.C:370): uint32 count + xyz FP64."""
    a = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    check(lib().dg_write_pts(os.fsencode(path), ptr(a), len(a)), "write_pts")


def readPtsFromFile(path) -> np.ndarray:
    """ot::readPtsFromFile (src/oct/OctFunctions.C:313): the points, [n, 3]."""
    n = C.c_int64()
    check(lib().dg_read_pts(os.fsencode(path), None, 0, C.byref(n)), "read_pts")
    out = np.empty((n.value, 3))
    check(lib().dg_read_pts(os.fsencode(path), ptr(out), n.value, C.byref(n)), "read_pts")
    return out


def writeDataPtsToFile(path, pts, vals) -> None:
    """ot::writeDataPtsToFile (src/oct/OctFunctions.C:387): count, xyz, one value per point."""
    a = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    v = np.ascontiguousarray(vals, np.float64).reshape(-1)
    if len(v) != len(a):
        raise ValueError("one value per point")
    check(lib().dg_write_data_pts(os.fsencode(path), ptr(a), ptr(v), len(a)), "write_data_pts")


def readDataPtsFromFile(path):
    """ot::readDataPtsFromFile (src/oct/OctFunctions.C:343): (points [n, 3], values [n])."""
    n = C.c_int64()
    check(lib().dg_read_data_pts(os.fsencode(path), None, None, 0, C.byref(n)), "read_data_pts")
    pts, vals = np.empty((n.value, 3)), np.empty(n.value)
    check(lib().dg_read_data_pts(os.fsencode(path), ptr(pts), ptr(vals), n.value, C.byref(n)), "read_data_pts")
    return pts, vals


def writeNodesToFile(path, octree: Octree) -> None:
    """ot::writeNodesToFile (src/oct/OctFunctions.C:424): the .ot text format."""
    check(lib().dg_octree_write(octree.h, os.fsencode(path)), "octree_write")


def readNodesFromFile(path) -> Octree:
    """ot::readNodesFromFile (src/oct/OctFunctions.C:403): an .ot file as an octree on the GPU."""
    h = C.c_void_p()
    check(lib().dg_octree_read(os.fsencode(path), C.byref(h)), "octree_read")
    return Octree(h)


def balanceOctree(octree: Octree) -> Octree:
    """ot::balanceOctree with incCorner = true (src/oct/Balance.C:31)."""
    h = C.c_void_p()
    check(lib().dg_balance_octree(octree.h, C.byref(h)), "balance_octree")
    return Octree(h)


def coarsenOctree(octree: Octree) -> Octree:
    """ot::coarsenOctree (src/oct/Coarsen.C:53-104)."""
    h = C.c_void_p()
    check(lib().dg_coarsen_octree(octree.h, C.byref(h)), "coarsen_octree")
    return Octree(h)


class DA:
    """ot::DA: the mesh of a balanced octree, resident on the GPU."""

    def __init__(self, octree: Octree = None, handle=None, owner=None):
        self._owner = owner
        if handle is None:
            h = C.c_void_p()
            check(lib().dg_da_create(octree.h, C.byref(h)), "da_create")
            handle = h
        self.h = handle if isinstance(handle, C.c_void_p) else C.c_void_p(handle)
        E, N, P = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().dg_da_sizes(self.h, C.byref(E), C.byref(N), C.byref(P)), "da_sizes")
        self.E, self.N, self.P = E.value, N.value, P.value
        self.maxDepth = int(lib().dg_da_max_depth(self.h))  # embedded depth
        self.octets = int(lib().dg_da_octets(self.h))  # parent octants with leaf children

    @classmethod
    def from_maps(cls, max_depth, nlist, level, cnum, hmask, node_xyz, elem_xyz) -> "DA":
        arrs = [np.ascontiguousarray(a, dt) for a, dt in
                ((nlist, np.uint32), (level, np.uint8), (cnum, np.uint8), (hmask, np.uint8),
                 (node_xyz, np.uint32), (elem_xyz, np.uint32))]
        h = C.c_void_p()
        check(lib().dg_da_create_from_maps(len(arrs[1]), len(arrs[4]), max_depth, *[ptr(a) for a in arrs],
                                           C.byref(h)), "da_create_from_maps")
        return cls(handle=h)

    def __del__(self):
        if getattr(self, "h", None) is not None and self._owner is None and self.h.value:
            lib().dg_da_destroy(self.h)
            self.h = None

    def getElementSize(self) -> int:
        return self.E

    def getNodeSize(self) -> int:
        """Nodes including the positive-boundary nodes (getNodeSize + getBoundaryNodeSize)."""
        return self.N

    def export(self) -> dict:
        E, N = self.E, self.N
        out = dict(nlist=np.empty((E, 8), np.uint32), hmask=np.empty(E, np.uint8), cnum=np.empty(E, np.uint8),
                   etype=np.empty(E, np.uint8), level=np.empty(E, np.uint8),
                   node_xyz=np.empty((N, 3), np.uint32), elem_xyz=np.empty((E, 3), np.uint32),
                   node_bdy=np.empty(N, np.uint8))
        check(lib().dg_da_export(self.h, *[ptr(out[k]) for k in ("nlist", "hmask", "cnum", "etype", "level",
                                                                  "node_xyz", "elem_xyz", "node_bdy")]),
              "da_export")
        return out

    def loadVector(self, force, b=None):
        """ComputeRHS_omgNeumann (omgNeumann.C:749-785): the force sampled at the element
        centres (elementCenters order) -> the load vector b [N].  Device tensors stay on
        the device; numpy arrays go through host copies."""
        if _is_device(force):
            import torch
            if b is None:
                b = torch.empty(self.N, dtype=torch.float64, device=force.device)
            check(lib().dg_da_load_vector(self.h, ptr(force), ptr(b), 1), "da_load_vector")
            return b
        f = np.ascontiguousarray(force, np.float64)
        out = np.empty(self.N, np.float64)
        check(lib().dg_da_load_vector(self.h, ptr(f), ptr(out), 0), "da_load_vector")
        return out

    def compressMaps(self, quotient_bits: int = 16) -> int:
        """Build the compressed element map (the DA's compressLut option); returns its bytes.
        The operator's autotuner then also times the element kernel that reads it."""
        check(lib().dg_da_compress_maps(self.h, int(quotient_bits)), "da_compress_maps")
        return self.compressedMapBytes()[0]

    def compressedMapBytes(self):
        """(bytes of the compressed map or 0, tiles stored with 32-bit quotients)."""
        w = C.c_int64()
        b = int(lib().dg_da_compressed_map_bytes(self.h, C.byref(w)))
        return b, w.value

    def decompressMaps(self) -> np.ndarray:
        """The element map [E, 8] decoded from the compressed form on the GPU."""
        out = np.empty((self.E, 8), np.uint32)
        check(lib().dg_da_decompress_maps(self.h, ptr(out)), "da_decompress_maps")
        return out

    def elementCenters(self) -> np.ndarray:
        """CalculateCenters (examples/src/backend/omgNeumann.C:788-820), [E, 3] in [0,1]."""
        c = np.empty((self.E, 3))
        check(lib().dg_da_element_centers(self.h, ptr(c)), "element_centers")
        return c

    def dumpMesh(self, prefix: str) -> None:
        """The files of examples/src/drivers/dumpMesh.C for one rank:
        <prefix>_NL_0_1.out, <prefix>_EL_0_1.out, <prefix>_M_0_1.out."""
        check(lib().dg_da_dump_mesh(self.h, os.fsencode(prefix)), "da_dump_mesh")


class _Mat:
    def __init__(self, da: DA, h):
        self.da = da
        self.h = h
        self.n = int(lib().dg_mat_size(self.h))

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().dg_mat_destroy(self.h)
            self.h = None

    def mult(self, x, y=None, stream=None):
        """y = A x.  Device tensors run on `stream` (a torch stream or None);
        host numpy arrays go through the copy-in / copy-out entry point."""
        if _is_device(x):
            import torch
            if y is None:
                y = torch.empty_like(x)
            s = None if stream is None else C.c_void_p(stream.cuda_stream)
            if x.dtype == torch.float64:
                check(lib().dg_mat_mult(self.h, ptr(x), ptr(y), s), "mat_mult")
            elif x.dtype == torch.float32:
                check(lib().dg_mat_mult_f32(self.h, ptr(x), ptr(y), s), "mat_mult_f32")
            else:
                raise TypeError("x must be float64 or float32")
            return y
        xa = np.ascontiguousarray(x, np.float64)
        ya = np.empty(self.n) if y is None else y
        check(lib().dg_mat_mult_host(self.h, ptr(xa), ptr(ya)), "mat_mult_host")
        return ya

    def mult_add(self, x, y, stream=None):
        """y += A x (FP64 or FP32 device tensors, scalar operator)."""
        import torch
        s = None if stream is None else C.c_void_p(stream.cuda_stream)
        if x.dtype == torch.float32:
            check(lib().dg_mat_mult_add_f32(self.h, ptr(x), ptr(y), s), "mat_mult_add_f32")
        else:
            check(lib().dg_mat_mult_add(self.h, ptr(x), ptr(y), s), "mat_mult_add")
        return y

    def mult_multi(self, X, Y=None, split: int = 3, stream=None):
        """Y = A X for the columns of X, a CUDA float32 tensor [N, nrhs]
        (nrhs a multiple of 16), on the tensor cores (split 3: FP32-level
        accuracy from three TF32 products; 1: one TF32 product; 5 and 4: the
        same two precisions with tcgen05 and tensor-memory accumulators on
        pairs of element parents, nrhs a multiple of 64), or with split 0 in
        the octet form on the CUDA cores (exact FP32 products; nrhs a multiple
        of 32)."""
        import torch
        if not (X.is_cuda and X.dtype == torch.float32 and X.dim() == 2 and X.is_contiguous()):
            raise TypeError("X must be a contiguous CUDA float32 tensor [N, nrhs]")
        if Y is None:
            Y = torch.empty_like(X)
        s = None if stream is None else C.c_void_p(stream.cuda_stream)
        check(lib().dg_mat_mult_multi(self.h, ptr(X), ptr(Y), X.shape[1], split, s), "mat_mult_multi")
        return Y

    def kernel_name(self, prec: int = 0) -> str:
        """Launch shape the autotuner chose for this mesh (after the first mult)."""
        return lib().dg_mat_kernel_name(self.h, prec).decode()

    @staticmethod
    def kernel_count() -> int:
        """Number of operator launch shapes the autotuner chooses from."""
        return lib().dg_mat_kernel_count()

    def set_kernel(self, variant: int, prec: int = 0) -> None:
        """Fix the operator launch shape for this mesh and precision (no timing)."""
        check(lib().dg_mat_set_kernel(self.h, prec, variant), "dg_mat_set_kernel")

    def getDiagonal(self, d=None, stream=None):
        import torch
        if d is None:
            d = torch.empty(self.n, dtype=torch.float64, device="cuda")
        s = None if stream is None else C.c_void_p(stream.cuda_stream)
        check(lib().dg_mat_get_diagonal(self.h, ptr(d), s), "mat_get_diagonal")
        return d


class Jacobian2(_Mat):
    """-div(a grad u) + b u (CreateJacobian2 / Jacobian2MatMult,
    examples/src/backend/omgNeumann.C:533,643); coef = [a0, b0, a1, b1, ...]
    per element, or None for a = b = 1."""

    def __init__(self, da: DA, coef=None):
        h = C.c_void_p()
        c = None if coef is None else np.ascontiguousarray(coef, np.float64).reshape(-1)
        if c is not None and len(c) != 2 * da.E:
            raise ValueError("coef must hold 2 values per element")
        check(lib().dg_mat_create_lapmass(da.h, ptr(c), C.byref(h)), "mat_create_lapmass")
        super().__init__(da, h)


class Elasticity(_Mat):
    """3-dof linear elasticity (ElasticityMatMult, examples/src/backend/elasticityJac.C:212)."""

    def __init__(self, da: DA, mu: float, lam: float, dirichlet=None):
        h = C.c_void_p()
        d = None if dirichlet is None else np.ascontiguousarray(dirichlet, np.uint8)
        check(lib().dg_mat_create_elasticity(da.h, mu, lam, ptr(d), C.byref(h)), "mat_create_elasticity")
        super().__init__(da, h)


class DirichletLaplacian(_Mat):
    """CreateDirichletLaplacian / DirichletLaplacianMatMult (examples/src/backend/
    omgJac.C:61, 859): h/2 L with unit coefficients, Dirichlet rows identity and
    columns dropped; dirichlet [N] defaults to the domain-boundary nodes."""

    _mass = 0

    def __init__(self, da: DA, dirichlet=None):
        h = C.c_void_p()
        d = None if dirichlet is None else np.ascontiguousarray(dirichlet, np.uint8)
        check(lib().dg_mat_create_dirichlet(da.h, self._mass, ptr(d), C.byref(h)), "mat_create_dirichlet")
        super().__init__(da, h)


class DirichletJacobian(DirichletLaplacian):
    """CreateDirichletJacobian / DirichletJacobianMatMult (omgJac.C:166, 957):
    h/2 L + h^3/8 M with unit coefficients, Dirichlet rows and columns as above."""

    _mass = 1


class DAMG:
    """ot::DAMG: level hierarchy + V-cycle preconditioned CG on the GPU."""

    def __init__(self, finest, nlevels: int = 30, nu_pre: int = 2, nu_post: int = 2,
                 omega: float = 2.0 / 3.0, rtol: float = 1e-8, maxit: int = 200, inner_prec: int = 0,
                 use_graph: bool = False, coarse_op: int = 0, dof: int = 1, mu: float = 1.0, lam: float = 1.0):
        """`finest` is one balanced Octree, or a list of them for the batched
        form (independent meshes solved together, one launch per kernel).
        coarse_op 1: operators below the finest level from the next finer
        level's coefficients (Jacobian3) instead of the level's averaged ones.
        dof 3 (DAMGCreateAndSetDA's dof): linear elasticity with Lame
        parameters mu, lam on every level, each level's boundary nodes
        Dirichlet (examples/src/drivers/newElasSolver.C); vectors are
        node-major [N][3]."""
        cfg = DamgConfig()
        lib().dg_damg_default_config(C.byref(cfg))
        cfg.nlevels, cfg.nu_pre, cfg.nu_post, cfg.omega = nlevels, nu_pre, nu_post, omega
        cfg.rtol, cfg.maxit, cfg.inner_prec, cfg.use_graph = rtol, maxit, inner_prec, int(use_graph)
        cfg.coarse_op = int(coarse_op)
        cfg.dof, cfg.mu, cfg.lambda_ = int(dof), float(mu), float(lam)
        self.dof = int(dof)
        h = C.c_void_p()
        if isinstance(finest, (list, tuple)):
            arr = (C.c_void_p * len(finest))(*[t.h.value for t in finest])
            check(lib().dg_damg_create_batch(arr, len(finest), C.byref(cfg), C.byref(h)), "damg_create_batch")
        else:
            check(lib().dg_damg_create(finest.h, C.byref(cfg), C.byref(h)), "damg_create")
        self.h = h
        self.count = int(lib().dg_damg_batch_count(self.h))
        self.nlevels = int(lib().dg_damg_levels(self.h))
        E = np.empty(self.nlevels, np.int64)
        N = np.empty(self.nlevels, np.int64)
        check(lib().dg_damg_level_sizes(self.h, ptr(E), ptr(N)), "damg_level_sizes")
        self.E, self.N = E, N

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().dg_damg_destroy(self.h)
            self.h = None

    def batch_offsets(self, level: int = 0):
        """(element offsets, node offsets) of each mesh on a level, count + 1 entries."""
        eo = np.empty(self.count + 1, np.int64)
        no = np.empty(self.count + 1, np.int64)
        check(lib().dg_damg_batch_offsets(self.h, level, ptr(eo), ptr(no)), "damg_batch_offsets")
        return eo, no

    def setTolerances(self, rtol: float, maxit: int = 200) -> None:
        """KSPSetTolerances: relative residual target and iteration limit."""
        check(lib().dg_damg_set_tolerances(self.h, rtol, maxit), "damg_set_tolerances")

    def level_da(self, l: int) -> DA:
        return DA(handle=lib().dg_damg_level_da(self.h, l), owner=self)

    def setKSP(self, coef=None):
        """DAMGSetKSP with the Jacobian2 operator (include/omg/omg.h:488)."""
        c = None if coef is None else np.ascontiguousarray(coef, np.float64).reshape(-1)
        check(lib().dg_damg_set_lapmass(self.h, ptr(c)), "damg_set_lapmass")

    def solve(self, b, x=None, allow_unconverged: bool = False):
        """DAMGSolve (include/omg/omg.h:492): returns (x, report dict)."""
        rep = SolveReport()
        if _is_device(b):
            import torch
            x = torch.empty_like(b) if x is None else x
            st = lib().dg_damg_solve(self.h, ptr(b), ptr(x), 1, C.byref(rep))
        else:
            ba = np.ascontiguousarray(b, np.float64)
            x = np.empty_like(ba) if x is None else x
            st = lib().dg_damg_solve(self.h, ptr(ba), ptr(x), 0, C.byref(rep))
        if not (allow_unconverged and st == 4):
            check(st, "damg_solve")
        return x, dict(iterations=rep.iterations, converged=bool(rep.converged), rel_residual=rep.rel_residual,
                       solve_ms=rep.solve_ms, smoother_fallbacks=rep.smoother_fallbacks)

    def solve_multi(self, B, X=None, allow_unconverged: bool = False):
        """Many right-hand sides at once: B [N, nrhs] FP64 (nrhs 32, 64, 128 or
        256; CUDA tensor or numpy), one flexible PCG per column around one
        V-cycle per iteration for all columns.  Returns (X, report dict)."""
        rep = SolveReport()
        R = int(B.shape[1])
        if _is_device(B):
            import torch
            B = B.contiguous()
            X = torch.empty_like(B) if X is None else X
            st = lib().dg_damg_solve_multi(self.h, ptr(B), ptr(X), R, 1, C.byref(rep))
        else:
            Ba = np.ascontiguousarray(B, np.float64)
            X = np.empty_like(Ba) if X is None else X
            st = lib().dg_damg_solve_multi(self.h, ptr(Ba), ptr(X), R, 0, C.byref(rep))
        if not (allow_unconverged and st == 4):
            check(st, "damg_solve_multi")
        return X, dict(iterations=rep.iterations, converged=bool(rep.converged), rel_residual=rep.rel_residual,
                       solve_ms=rep.solve_ms)

    def setSmoother(self, mlp=None, sweeps: int = 2, fallback_ratio: float = 0.7):
        """Finest-level post-smoother: a learned MLP (dendro_b200.learned.MLP)
        or None for damped Jacobi; needs the FP32 inner V-cycle (inner_prec=1)."""
        self._mlp = mlp  # keep the network alive while the hierarchy uses it
        check(lib().dg_damg_set_smoother(self.h, None if mlp is None else mlp.h, sweeps, fallback_ratio),
              "damg_set_smoother")

    def prolong(self, level: int, xc: np.ndarray, xf: np.ndarray) -> np.ndarray:
        xc = np.ascontiguousarray(xc, np.float64)
        xf = np.ascontiguousarray(xf, np.float64).copy()
        check(lib().dg_damg_prolong(self.h, level, ptr(xc), ptr(xf), 0), "damg_prolong")
        return xf

    def levelApply(self, level: int, x):
        """y = J x on one level (0 = finest), host numpy or device tensor."""
        if _is_device(x):
            import torch
            y = torch.empty_like(x)
            check(lib().dg_damg_level_apply(self.h, level, ptr(x), ptr(y), 1), "damg_level_apply")
            return y
        xa = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(xa)
        check(lib().dg_damg_level_apply(self.h, level, ptr(xa), ptr(y), 0), "damg_level_apply")
        return y

    def restrict(self, level: int, rf: np.ndarray) -> np.ndarray:
        rf = np.ascontiguousarray(rf, np.float64)
        rc = np.empty(self.dof * int(self.N[level + 1]))
        check(lib().dg_damg_restrict(self.h, level, ptr(rf), ptr(rc), 0), "damg_restrict")
        return rc


def vecDot(x, y, stream=None) -> float:
    """FP64 inner product of two device vectors (PETSc VecDot stand-in)."""
    import torch
    out = torch.empty(1, dtype=torch.float64, device=x.device)
    s = None if stream is None else C.c_void_p(stream.cuda_stream)
    check(lib().dg_vec_dot(ptr(x), ptr(y), x.numel(), ptr(out), s), "vec_dot")
    return float(out.item())


def deviceCheck(stream=None) -> None:
    """Synchronise `stream` (a torch stream or None) and raise DendroError
    (DG_ETIMEOUT) when a bounded device wait of an operator kernel ran out
    since the last check; the launches concerned produced no valid result."""
    s = None if stream is None else C.c_void_p(stream.cuda_stream)
    check(lib().dg_device_check(s), "device_check")


def setDeviceWaitLimit(cycles: int) -> None:
    """Test hook: clock64 cycles a staged operator kernel waits for its copies
    before giving up (<= 0 restores the default of 2^31 cycles)."""
    check(lib().dg_set_device_wait_limit(int(cycles)), "set_device_wait_limit")
