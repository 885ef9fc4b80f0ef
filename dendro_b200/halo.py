"""One mesh split over several ranks (ot::DA and ot::DAMG with npes > 1), one
process per GPU.

The partition and each rank's exchange plans are built on the host
(libdendro_b200: dg_halo_create, a restatement of par::partitionW and of the
DA's scatter maps; dg_parcsr_create for the multigrid transfers); an exchange
is a pack kernel and one all-to-all through a communicator (``TorchComm``:
torch.distributed, NCCL between GPUs, gloo on the host) per direction:

* ``read_from_ghosts``  owners -> readers, into the ghost slots
  (ReadFromGhostsBegin/End, include/oda/oda.txx:479-560);
* ``write_to_ghosts``   readers -> owners, added to the owned values
  (WriteToGhostsBegin/End, include/oda/oda.txx:566-640).

``HaloJacobian2.mult`` follows Jacobian2MatMult (examples/src/backend/
omgNeumann.C:505-525): the exchange is started, the independent elements
(all vertices owned) are applied while it is in flight, then the dependent
ones are added in place (one launch of y += A x over the local vector).
Local vectors hold the owned nodes first, then the ghosts; after ``mult`` the
owned part of y is complete and its ghost slots are not defined.

A communicator provides ``rank``, ``size``, ``all_to_all_single(out, inp,
out_splits, in_splits, async_op)`` (the torch.distributed signature, returning
a work handle or None), ``all_reduce(t)`` (sum, in place) and
``all_gather_v(t, counts)`` (the ranks' tensors concatenated in rank order).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, ptr
from .api import DA, DAMG, Jacobian2


class TorchComm:
    """torch.distributed as the transport (the default process group, or
    `group`); a single rank when no process group is initialised."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.rank, self.size = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.size = 0, 1

    def all_to_all_single(self, out, inp, out_splits, in_splits, async_op=False):
        import torch.distributed as dist
        if self.size == 1:
            if out.numel():
                out.copy_(inp)
            return None
        return dist.all_to_all_single(out, inp, out_splits, in_splits, group=self.group, async_op=async_op)

    def all_reduce(self, t):
        import torch.distributed as dist
        if self.size > 1:
            dist.all_reduce(t, group=self.group)
        return t

    def all_gather_v(self, t, counts):
        import torch
        import torch.distributed as dist
        if self.size == 1:
            return t
        m = max(int(c) for c in counts)
        buf = torch.zeros(m, dtype=t.dtype, device=t.device)
        buf[: t.numel()] = t
        parts = [torch.empty_like(buf) for _ in range(self.size)]
        dist.all_gather(parts, buf, group=self.group)
        return torch.cat([p[: int(c)] for p, c in zip(parts, counts)])


def partition_weighted(n: int, nranks: int, weights=None) -> np.ndarray:
    """par::partitionW's ranges (include/par/parUtils.txx:1011-1177) for n
    items: rank r gets first[r] .. first[r+1] - 1."""
    first = np.empty(nranks + 1, np.int64)
    w = None if weights is None else np.ascontiguousarray(weights, np.uint32)
    if w is not None and len(w) != n:
        raise ValueError("one weight per item")
    check(lib().dg_partition_weighted(n, ptr(w), nranks, ptr(first)), "partition_weighted")
    return first


def _stream(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def _splits(counts, dof=1):
    return [int(c) * dof for c in counts]


class HaloDA:
    """This rank's part of a mesh partitioned over the ranks of `comm`."""

    def __init__(self, da: DA = None, maps: dict = None, max_depth: int = None, rank: int = None,
                 nranks: int = None, weights=None, comm=None):
        """From a mesh on the GPU (`da`), or from its host maps (`maps` as
        returned by DA.export(), with the octree's `max_depth`: no GPU is
        touched).  rank / nranks default to the communicator's (a TorchComm
        over the default process group when `comm` is None); a part built
        for an explicit rank without a communicator cannot exchange."""
        if comm is None and rank is None:
            comm = TorchComm()
        self.comm = comm
        self.rank = comm.rank if rank is None else int(rank)
        self.nranks = comm.size if nranks is None else int(nranks)
        w = None if weights is None else np.ascontiguousarray(weights, np.uint32).reshape(-1)
        h = C.c_void_p()
        if da is not None:
            if w is not None and len(w) != da.E:
                raise ValueError(f"weights has {len(w)} entries, the mesh has {da.E} elements")
            check(lib().dg_halo_create_from_da(da.h, ptr(w), self.nranks, self.rank, C.byref(h)), "halo_create")
        else:
            m = {k: np.ascontiguousarray(maps[k], dt) for k, dt in
                 (("nlist", np.uint32), ("level", np.uint8), ("cnum", np.uint8), ("hmask", np.uint8),
                  ("node_xyz", np.uint32), ("elem_xyz", np.uint32))}
            E, N = len(m["level"]), len(m["node_xyz"])
            if m["nlist"].size != 8 * E or m["node_xyz"].size != 3 * N or m["elem_xyz"].size != 3 * E:
                raise ValueError("maps: nlist must hold 8 ids per element, node_xyz and elem_xyz 3 coordinates "
                                 "per node / element")
            if len(m["cnum"]) != E or len(m["hmask"]) != E:
                raise ValueError("maps: level, cnum and hmask must have one entry per element")
            if w is not None and len(w) != E:
                raise ValueError(f"weights has {len(w)} entries, the mesh has {E} elements")
            check(lib().dg_halo_create(E, N, max_depth, *[ptr(m[k]) for k in ("nlist", "level", "cnum", "hmask",
                                                                              "node_xyz", "elem_xyz")],
                                       ptr(w), self.nranks, self.rank, C.byref(h)), "halo_create")
        self.h = h
        v = [C.c_int64() for _ in range(5)]
        check(lib().dg_halo_sizes(self.h, *[C.byref(x) for x in v]), "halo_sizes")
        (self.n_owned, self.n_ghost, self.first_owned, n_ind, n_dep) = [x.value for x in v]
        self.n_local = self.n_owned + self.n_ghost
        P = self.nranks
        self.elem_first = np.empty(P + 1, np.int64)
        self.node_first = np.empty(P + 1, np.int64)
        check(lib().dg_halo_ranges(self.h, ptr(self.elem_first), ptr(self.node_first)), "halo_ranges")
        self.send_counts = np.empty(P, np.int64)
        self.recv_counts = np.empty(P, np.int64)
        check(lib().dg_halo_comm(self.h, ptr(self.send_counts), ptr(self.recv_counts), None, None), "halo_comm")
        self.send_idx = np.empty(int(self.send_counts.sum()), np.uint32)
        self.ghosts = np.empty(self.n_ghost, np.uint32)
        check(lib().dg_halo_comm(self.h, None, None, ptr(self.send_idx), ptr(self.ghosts)), "halo_comm")
        self.independent = np.empty(n_ind, np.int64)
        self.ind_nlist = np.empty((n_ind, 8), np.uint32)
        check(lib().dg_halo_part(self.h, 0, ptr(self.independent), ptr(self.ind_nlist)), "halo_part")
        self.dependent = np.empty(n_dep, np.int64)
        self.dep_nlist = np.empty((n_dep, 8), np.uint32)
        check(lib().dg_halo_part(self.h, 1, ptr(self.dependent), ptr(self.dep_nlist)), "halo_part")
        self.da_ind = self.da_dep = None

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().dg_halo_destroy(self.h)
            self.h = None

    def local_to_global(self) -> np.ndarray:
        """Global node id of every local node (owned, then ghosts)."""
        own = np.arange(self.first_owned, self.first_owned + self.n_owned, dtype=np.int64)
        return np.concatenate([own, self.ghosts.astype(np.int64)])

    def local_das(self):
        """The GPU meshes of the independent and the dependent elements (None
        for a part without elements), built on first use."""
        if self.da_ind is None and len(self.independent):
            h = C.c_void_p()
            check(lib().dg_halo_local_da(self.h, 0, C.byref(h)), "halo_local_da")
            self.da_ind = DA(handle=h)
        if self.da_dep is None and len(self.dependent):
            h = C.c_void_p()
            check(lib().dg_halo_local_da(self.h, 1, C.byref(h)), "halo_local_da")
            self.da_dep = DA(handle=h)
        return self.da_ind, self.da_dep

    # ------------------------------------------------------------ vectors ---
    def local_vector(self, owned=None, dof: int = 1, dtype=None):
        """A device vector in local layout (zeros, owned part from `owned`);
        FP64 unless dtype says otherwise (torch.float32 for the FP32 cycle)."""
        import torch
        dt = torch.float64 if dtype is None else dtype
        x = torch.zeros(self.n_local * dof, dtype=dt, device="cuda")
        if owned is not None:
            x[: self.n_owned * dof].copy_(torch.as_tensor(owned, dtype=dt).reshape(-1))
        return x

    # ----------------------------------------------------------- kernels ---
    def pack(self, x_local, send=None, dof: int = 1, stream=None):
        """ReadFromGhostsBegin's send buffer: the owned values each peer reads."""
        import torch
        if send is None:
            send = torch.empty(len(self.send_idx) * dof, dtype=x_local.dtype, device=x_local.device)
        if x_local.dtype == torch.float32:
            check(lib().dg_halo_pack_f32(self.h, ptr(x_local), ptr(send), dof, _stream(stream)), "halo_pack_f32")
        else:
            check(lib().dg_halo_pack(self.h, ptr(x_local), ptr(send), dof, _stream(stream)), "halo_pack")
        return send

    def accumulate(self, recv, y_local, dof: int = 1, stream=None):
        """WriteToGhostsEnd: add the peers' ghost contributions to the owned values."""
        check(lib().dg_halo_accumulate(self.h, ptr(recv), ptr(y_local), dof, _stream(stream)), "halo_accumulate")
        return y_local

    # -------------------------------------------------------- exchanges ---
    def read_from_ghosts(self, x_local, dof: int = 1, async_op: bool = False):
        """Fill x_local's ghost slots from their owners (one all-to-all).
        With async_op the returned work handle (or None) must be waited on
        before the ghost slots are read."""
        if self.comm is None:
            raise RuntimeError("this part was built for an explicit rank without a communicator")
        send = self.pack(x_local, dof=dof)
        return self.comm.all_to_all_single(x_local[self.n_owned * dof:], send, _splits(self.recv_counts, dof),
                                           _splits(self.send_counts, dof), async_op=async_op)

    def write_to_ghosts(self, y_local, dof: int = 1):
        """Send y_local's ghost slots to their owners and add them there."""
        import torch
        if self.comm is None:
            raise RuntimeError("this part was built for an explicit rank without a communicator")
        recv = torch.empty(len(self.send_idx) * dof, dtype=y_local.dtype, device=y_local.device)
        self.comm.all_to_all_single(recv, y_local[self.n_owned * dof:], _splits(self.send_counts, dof),
                                    _splits(self.recv_counts, dof))
        return self.accumulate(recv, y_local, dof=dof)

    def dot(self, x, y, dof: int = 1) -> float:
        """Global inner product over the owned values (VecDot with an FP64
        sum over ranks)."""
        import torch
        n = self.n_owned * dof
        v = torch.dot(x[:n], y[:n]).reshape(1)
        if self.comm is not None:
            self.comm.all_reduce(v)
        elif self.nranks > 1:
            raise RuntimeError("this part was built for an explicit rank without a communicator")
        return float(v.item())


class HaloJacobian2:
    """-div(a grad u) + b u on a partitioned mesh (Jacobian2MatMult over
    the independent, then the dependent elements); coef holds the global
    mesh's per-element (a, b) pairs, or None for a = b = 1."""

    def __init__(self, hda: HaloDA, coef=None):
        self.hda = hda
        da_ind, da_dep = hda.local_das()
        c = None if coef is None else np.ascontiguousarray(coef, np.float64).reshape(-1, 2)
        self.A_ind = None if da_ind is None else Jacobian2(da_ind, None if c is None else c[hda.independent])
        self.A_dep = None if da_dep is None else Jacobian2(da_dep, None if c is None else c[hda.dependent])

    def mult(self, x_local, y_local=None, overlap: bool = True):
        """y = A x on the owned nodes; x_local's ghost slots are refreshed."""
        hda = self.hda
        work = hda.read_from_ghosts(x_local, async_op=overlap) if hda.nranks > 1 else None
        y_local = self._independent(x_local, y_local)
        if work is not None:
            work.wait()
        return self._dependent(x_local, y_local)

    def apply_local(self, x_local, y_local=None):
        """y = A x on the owned nodes from x_local as it is (ghost slots
        already filled): the operator part of mult without the exchange."""
        return self._dependent(x_local, self._independent(x_local, y_local))

    def _independent(self, x_local, y_local):
        import torch
        hda = self.hda
        if y_local is None:
            y_local = torch.zeros_like(x_local)
        y_own = y_local[: hda.n_owned]
        if self.A_ind is not None:
            self.A_ind.mult(x_local[: hda.n_owned], y_own, stream=torch.cuda.current_stream())
        else:
            y_own.zero_()
        return y_local

    def _dependent(self, x_local, y_local):
        import torch
        if self.A_dep is not None:
            self.A_dep.mult_add(x_local, y_local, stream=torch.cuda.current_stream())
        return y_local

    def getDiagonal(self):
        """Diagonal on the owned nodes [n_owned]."""
        import torch
        hda = self.hda
        d = torch.zeros(hda.n_owned, dtype=torch.float64, device="cuda")
        if self.A_ind is not None:
            self.A_ind.getDiagonal(d)
        if self.A_dep is not None:
            d += self.A_dep.getDiagonal()[: hda.n_owned]
        return d


class ParCSR:
    """This rank's rows of a sparse matrix M between two partitioned levels
    (rows owned by row_first, input values owned by col_first): y = M x with
    one exchange of the input values the rows read."""

    def __init__(self, ptr_, col, val, nrows, ncols, row_first, col_first, rank, nranks, comm=None):
        self.comm = comm
        p = np.ascontiguousarray(ptr_, np.uint32)
        c = np.ascontiguousarray(col, np.uint32)
        v = np.ascontiguousarray(val, np.float64)
        rf = np.ascontiguousarray(row_first, np.int64)
        cf = np.ascontiguousarray(col_first, np.int64)
        if len(rf) != nranks + 1 or len(cf) != nranks + 1:
            raise ValueError("row_first and col_first need nranks + 1 entries")
        if len(p) != nrows + 1:
            raise ValueError(f"ptr has {len(p)} entries, expected nrows + 1 = {nrows + 1}")
        if nrows and (len(c) < int(p[-1]) or len(v) < int(p[-1])):
            raise ValueError(f"col / val hold {len(c)} / {len(v)} entries, ptr[-1] = {int(p[-1])}")
        h = C.c_void_p()
        check(lib().dg_parcsr_create(nrows, ncols, ptr(p), ptr(c), ptr(v), ptr(rf), ptr(cf), nranks, rank,
                                     C.byref(h)), "parcsr_create")
        self.h = h
        s = [C.c_int64() for _ in range(4)]
        check(lib().dg_parcsr_sizes(self.h, *[C.byref(x) for x in s]), "parcsr_sizes")
        self.n_rows, self.n_cols_owned, self.n_ghost, self.nnz = [x.value for x in s]
        self.send_counts = np.empty(nranks, np.int64)
        self.recv_counts = np.empty(nranks, np.int64)
        check(lib().dg_parcsr_comm(self.h, ptr(self.send_counts), ptr(self.recv_counts), None, None), "parcsr_comm")
        self.n_send = int(self.send_counts.sum())

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().dg_parcsr_destroy(self.h)
            self.h = None

    def mult(self, x_own, y=None, add: bool = False):
        """y = M x (or y += M x) on the owned rows from the owned input values
        (FP64, or FP32 with the FP32 copy of the entries)."""
        import torch
        dev, dt = x_own.device, x_own.dtype
        f32 = dt == torch.float32
        send = torch.empty(self.n_send, dtype=dt, device=dev)
        check((lib().dg_parcsr_pack_f32 if f32 else lib().dg_parcsr_pack)(self.h, ptr(x_own), ptr(send), _stream()),
              "parcsr_pack")
        ghost = torch.empty(self.n_ghost, dtype=dt, device=dev)
        if self.comm is not None:
            self.comm.all_to_all_single(ghost, send, _splits(self.recv_counts), _splits(self.send_counts))
        elif self.n_ghost or self.n_send:
            raise RuntimeError("these rows read other ranks' values: a communicator is needed")
        if y is None:
            y = torch.empty(self.n_rows, dtype=dt, device=dev)
        apply = lib().dg_parcsr_apply_f32 if f32 else lib().dg_parcsr_apply
        check(apply(self.h, ptr(x_own), ptr(ghost), ptr(y), int(add), _stream()), "parcsr_apply")
        return y


class HaloDAMG:
    """ot::DAMG over a partitioned mesh: every level split over the ranks by
    the weighted partition of its elements, the level operators as
    HaloJacobian2, R and P as ParCSR products with one exchange each, and
    the coarsest level gathered to every rank and solved with the dense
    inverse (PC_KSP_Shell gathers it to one rank, include/omg/omg.h:236-249).
    The V-cycle is the single-GPU one's (damped Jacobi V(nu_pre, nu_post)
    from a zero guess, R of the residual, P added), applied to the ranks'
    owned values; CG as DAMGSolve's (src/omg/omg.C:1121-1169).

    The hierarchy is built whole on every rank (set-up); each rank then keeps
    and applies only its parts.  coarse_op 0 (averaged coefficients) only.

    inner_prec 1 runs the V-cycle in FP32 (operators on the FP32 coefficient
    copies, smoother, transfers and exchanges in FP32, the gathered coarsest
    level solved in FP64) inside an FP64 flexible CG, as the single-GPU
    mixed-precision solver does."""

    def __init__(self, octree, coef=None, comm=None, nlevels: int = 30, nu_pre: int = 2, nu_post: int = 2,
                 omega: float = 2.0 / 3.0, inner_prec: int = 0):
        import torch
        self.inner_prec = int(inner_prec)
        self.comm = TorchComm() if comm is None else comm
        rank, P = self.comm.rank, self.comm.size
        self.m = DAMG(octree, nlevels=nlevels, nu_pre=nu_pre, nu_post=nu_post, omega=omega)
        self.m.setKSP(coef)
        self.nlevels = self.m.nlevels
        self.nu_pre, self.nu_post, self.omega = nu_pre, nu_post, omega
        self.levels = []
        for l in range(self.nlevels):
            da = self.m.level_da(l)
            hda = HaloDA(da, comm=self.comm)
            c = np.empty(2 * da.E)
            check(lib().dg_damg_level_coef(self.m.h, l, ptr(c)), "damg_level_coef")
            A = HaloJacobian2(hda, c) if l + 1 < self.nlevels else None
            dinv = None if A is None else 1.0 / A.getDiagonal()
            dinv32 = None if dinv is None else dinv.float()
            self.levels.append(dict(hda=hda, A=A, dinv=dinv, dinv32=dinv32, N=da.N))
        self.P, self.R = [], []
        for l in range(self.nlevels - 1):
            nf, ncs = int(self.m.N[l]), int(self.m.N[l + 1])
            ff, cf = self.levels[l]["hda"].node_first, self.levels[l + 1]["hda"].node_first
            mats = []
            for which, (nr, nc, rf, colf) in enumerate(((nf, ncs, ff, cf), (ncs, nf, cf, ff))):
                nnz = C.c_int64()
                check(lib().dg_damg_transfer_export(self.m.h, l, which, C.byref(nnz), None, None, None),
                      "damg_transfer_export")
                p_ = np.empty(nr + 1, np.uint32)
                c_ = np.empty(nnz.value, np.uint32)
                v_ = np.empty(nnz.value)
                check(lib().dg_damg_transfer_export(self.m.h, l, which, C.byref(nnz), ptr(p_), ptr(c_), ptr(v_)),
                      "damg_transfer_export")
                mats.append(ParCSR(p_, c_, v_, nr, nc, rf, colf, rank, P, comm=self.comm))
            self.P.append(mats[0])
            self.R.append(mats[1])
        top = self.levels[-1]["hda"]
        self.coarse_counts = np.diff(top.node_first)
        self._xc = torch.empty(int(self.m.N[-1]), dtype=torch.float64, device="cuda")

    @property
    def n_owned(self) -> int:
        return self.levels[0]["hda"].n_owned

    @property
    def first_owned(self) -> int:
        return self.levels[0]["hda"].first_owned

    def _smooth(self, L, x_loc, b):
        import torch
        n = L["hda"].n_owned
        ax = L["A"].mult(x_loc)
        if x_loc.dtype == torch.float32:
            check(lib().dg_vec_jacobi_update_f32(ptr(x_loc), ptr(b), ptr(ax), ptr(L["dinv32"]), self.omega, n,
                                                 _stream()), "vec_jacobi_update_f32")
        else:
            check(lib().dg_vec_jacobi_update(ptr(x_loc), ptr(b), ptr(ax), ptr(L["dinv"]), self.omega, n,
                                             _stream()), "vec_jacobi_update")

    def vcycle(self, b, l: int = 0):
        """z = V(b) on level l from the owned values b [n_owned], in b's
        precision (FP32 b: the FP32 cycle, its coarsest level solved in FP64)."""
        import torch
        L = self.levels[l]
        hda = L["hda"]
        f32 = b.dtype == torch.float32
        if l + 1 == self.nlevels:
            full = self.comm.all_gather_v(b, self.coarse_counts).contiguous()
            if f32:
                full = full.double()
            check(lib().dg_damg_coarse_solve(self.m.h, ptr(full), ptr(self._xc), _stream()), "damg_coarse_solve")
            z = self._xc[hda.first_owned:hda.first_owned + hda.n_owned].clone()
            return z.float() if f32 else z
        n = hda.n_owned
        x_loc = hda.local_vector(dtype=b.dtype)
        if self.nu_pre > 0:
            x_loc[:n].copy_(self.omega * (L["dinv32"] if f32 else L["dinv"]) * b)
            for _ in range(self.nu_pre - 1):
                self._smooth(L, x_loc, b)
            r = b - L["A"].mult(x_loc)[:n]
        else:
            r = b
        rc = self.R[l].mult(r.contiguous())
        xc = self.vcycle(rc, l + 1)
        self.P[l].mult(xc, x_loc[:n], add=True)
        for _ in range(self.nu_post):
            self._smooth(L, x_loc, b)
        return x_loc[:n].clone()

    def solve(self, b_owned, rtol: float = 1e-8, maxit: int = 200):
        """PCG with one V-cycle per iteration on the owned values: returns
        (x_owned, iterations, converged, relative residual)."""
        import torch
        hda = self.levels[0]["hda"]
        A = self.levels[0]["A"]
        n = hda.n_owned
        b = torch.as_tensor(b_owned, dtype=torch.float64, device="cuda").reshape(-1)
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        r = b.clone()
        bnorm = hda.dot(b, b) ** 0.5
        if bnorm == 0:
            return x, 0, True, 0.0
        # the FP32 cycle is not exactly the same linear map from one call to
        # the next (FP32 rounding), so CG takes the flexible (Polak-Ribiere)
        # direction update: beta = z_new . (r_new - r_old) / (z_old . r_old)
        flexible = self.inner_prec == 1
        pre = (lambda v: self.vcycle(v.float()).double()) if flexible else self.vcycle
        z = pre(r)
        p_loc = hda.local_vector()
        p_loc[:n].copy_(z)
        rz = hda.dot(r, z)
        rel = 1.0
        it = 0
        for it in range(1, maxit + 1):
            q = A.mult(p_loc)[:n]
            alpha = rz / hda.dot(p_loc, q)
            x.add_(p_loc[:n], alpha=alpha)
            r_old = r.clone() if flexible else None
            r.add_(q, alpha=-alpha)
            rel = hda.dot(r, r) ** 0.5 / bnorm
            if rel <= rtol:
                return x, it, True, rel
            z = pre(r)
            rz_new = hda.dot(r, z)
            beta = (rz_new - hda.dot(r_old, z)) / rz if flexible else rz_new / rz
            p_loc[:n].mul_(beta).add_(z)
            rz = rz_new
        return x, it, False, rel


def halo_cg(A, b_owned, rtol: float = 1e-8, maxit: int = 1000):
    """Jacobi-preconditioned CG over a partitioned mesh (KSPCG with a
    distributed MatShell and PCJACOBI): returns (x_owned, iterations,
    converged), the stopping test ||r|| <= rtol ||b|| in FP64 over all
    ranks.  A provides hda (a HaloDA), mult(x_local) and getDiagonal();
    vectors live on b_owned's device."""
    import torch
    hda = A.hda
    n = hda.n_owned
    b = torch.as_tensor(b_owned, dtype=torch.float64).reshape(-1)
    dev = b.device
    dinv = 1.0 / A.getDiagonal()
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    r = b.clone()
    p_loc = torch.zeros(hda.n_local, dtype=torch.float64, device=dev)
    z = dinv * r
    p_loc[:n].copy_(z)
    rz = hda.dot(r, z)
    bb = hda.dot(b, b)
    rr = bb
    it = 0
    while it < maxit and rr > (rtol * rtol) * bb:
        q = A.mult(p_loc)[:n]
        alpha = rz / hda.dot(p_loc, q)
        x.add_(p_loc[:n], alpha=alpha)
        r.add_(q, alpha=-alpha)
        z = dinv * r
        rz_new = hda.dot(r, z)
        p_loc[:n].mul_(rz_new / rz).add_(z)
        rz = rz_new
        rr = hda.dot(r, r)
        it += 1
    return x, it, bool(rr <= (rtol * rtol) * bb)
