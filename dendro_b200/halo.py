"""One mesh split over several ranks (ot::DA with npes > 1), one process per GPU.

The partition and each rank's exchange plan are built on the host
(libdendro_b200: dg_halo_create, a restatement of par::partitionW and of the
DA's scatter maps); the exchange is a pack kernel and one all-to-all over
torch.distributed (NCCL between GPUs, gloo on the host) per direction:

* ``read_from_ghosts``  owners -> readers, into the ghost slots
  (ReadFromGhostsBegin/End, include/oda/oda.txx:479-560);
* ``write_to_ghosts``   readers -> owners, added to the owned values
  (WriteToGhostsBegin/End, include/oda/oda.txx:566-640).

``HaloJacobian2.mult`` follows Jacobian2MatMult (examples/src/backend/
omgNeumann.C:505-525): the exchange is started, the independent elements
(all vertices owned) are applied while it is in flight, then the dependent
ones are added in place (one launch of y += A x over the local vector).  Local vectors hold the owned nodes first, then the ghosts; after
``mult`` the owned part of y is complete and its ghost slots are not defined.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib, ptr
from .api import DA, Jacobian2


def partition_weighted(n: int, nranks: int, weights=None) -> np.ndarray:
    """par::partitionW's ranges (include/par/parUtils.txx:1011-1177) for n
    items: rank r gets first[r] .. first[r+1] - 1."""
    first = np.empty(nranks + 1, np.int64)
    w = None if weights is None else np.ascontiguousarray(weights, np.uint32)
    if w is not None and len(w) != n:
        raise ValueError("one weight per item")
    check(lib().dg_partition_weighted(n, ptr(w), nranks, ptr(first)), "partition_weighted")
    return first


def _world(rank, nranks):
    if rank is not None and nranks is not None:
        return int(rank), int(nranks)
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


class HaloDA:
    """This rank's part of a mesh partitioned over `nranks` ranks."""

    def __init__(self, da: DA = None, maps: dict = None, max_depth: int = None, rank: int = None,
                 nranks: int = None, weights=None):
        """From a mesh on the GPU (`da`), or from its host maps (`maps` as
        returned by DA.export(), with the octree's `max_depth`: no GPU is
        touched).  rank / nranks default to the torch.distributed group's."""
        self.rank, self.nranks = _world(rank, nranks)
        w = None if weights is None else np.ascontiguousarray(weights, np.uint32)
        h = C.c_void_p()
        if da is not None:
            check(lib().dg_halo_create_from_da(da.h, ptr(w), self.nranks, self.rank, C.byref(h)), "halo_create")
        else:
            m = {k: np.ascontiguousarray(maps[k], dt) for k, dt in
                 (("nlist", np.uint32), ("level", np.uint8), ("cnum", np.uint8), ("hmask", np.uint8),
                  ("node_xyz", np.uint32), ("elem_xyz", np.uint32))}
            E, N = len(m["level"]), len(m["node_xyz"])
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
    def local_vector(self, owned=None, dof: int = 1):
        """A device vector in local layout (zeros, owned part from `owned`)."""
        import torch
        x = torch.zeros(self.n_local * dof, dtype=torch.float64, device="cuda")
        if owned is not None:
            x[: self.n_owned * dof].copy_(torch.as_tensor(owned, dtype=torch.float64).reshape(-1))
        return x

    def owned(self, x_local, dof: int = 1):
        return x_local[: self.n_owned * dof]

    # ----------------------------------------------------------- kernels ---
    @staticmethod
    def _stream(stream):
        import torch
        s = torch.cuda.current_stream() if stream is None else stream
        return C.c_void_p(s.cuda_stream)

    def pack(self, x_local, send=None, dof: int = 1, stream=None):
        """ReadFromGhostsBegin's send buffer: the owned values each peer reads."""
        import torch
        if send is None:
            send = torch.empty(len(self.send_idx) * dof, dtype=torch.float64, device=x_local.device)
        check(lib().dg_halo_pack(self.h, ptr(x_local), ptr(send), dof, self._stream(stream)), "halo_pack")
        return send

    def accumulate(self, recv, y_local, dof: int = 1, stream=None):
        """WriteToGhostsEnd: add the peers' ghost contributions to the owned values."""
        check(lib().dg_halo_accumulate(self.h, ptr(recv), ptr(y_local), dof, self._stream(stream)),
              "halo_accumulate")
        return y_local

    # -------------------------------------------------------- exchanges ---
    def read_from_ghosts(self, x_local, dof: int = 1, group=None, async_op: bool = False):
        """Fill x_local's ghost slots from their owners (one all-to-all).
        With async_op the returned work handle must be waited on before the
        ghost slots are read."""
        import torch.distributed as dist
        send = self.pack(x_local, dof=dof)
        recv = x_local[self.n_owned * dof:]
        return dist.all_to_all_single(recv, send, output_split_sizes=[int(c) * dof for c in self.recv_counts],
                                      input_split_sizes=[int(c) * dof for c in self.send_counts], group=group,
                                      async_op=async_op)

    def write_to_ghosts(self, y_local, dof: int = 1, group=None):
        """Send y_local's ghost slots to their owners and add them there."""
        import torch
        import torch.distributed as dist
        send = y_local[self.n_owned * dof:]
        recv = torch.empty(len(self.send_idx) * dof, dtype=y_local.dtype, device=y_local.device)
        dist.all_to_all_single(recv, send, output_split_sizes=[int(c) * dof for c in self.send_counts],
                               input_split_sizes=[int(c) * dof for c in self.recv_counts], group=group)
        return self.accumulate(recv, y_local, dof=dof)

    def dot(self, x_local, y_local, group=None, dof: int = 1) -> float:
        """Global inner product over the owned values (VecDot with an FP64
        sum over ranks)."""
        import torch
        import torch.distributed as dist
        n = self.n_owned * dof
        v = torch.dot(x_local[:n], y_local[:n]).reshape(1)
        if self.nranks > 1:
            dist.all_reduce(v, group=group)
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

    def mult(self, x_local, y_local=None, group=None, overlap: bool = True):
        """y = A x on the owned nodes; x_local's ghost slots are refreshed."""
        hda = self.hda
        work = hda.read_from_ghosts(x_local, group=group, async_op=overlap) if hda.nranks > 1 else None
        y_local = self._independent(x_local, y_local)
        if work is not None and overlap:
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


def halo_cg(A, b_owned, rtol: float = 1e-8, maxit: int = 1000, group=None):
    """Jacobi-preconditioned CG over a partitioned mesh (KSPCG with a
    distributed MatShell and PCJACOBI): returns (x_owned, iterations,
    converged), the stopping test ||r|| <= rtol ||b|| in FP64 over all
    ranks.  A provides hda (a HaloDA), mult(x_local, group=) and
    getDiagonal(); vectors live on b_owned's device."""
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
    rz = hda.dot(r, z, group=group)
    bb = hda.dot(b, b, group=group)
    rr = bb
    it = 0
    while it < maxit and rr > (rtol * rtol) * bb:
        q = A.mult(p_loc, group=group)[:n]
        alpha = rz / hda.dot(p_loc, q, group=group)
        x.add_(p_loc[:n], alpha=alpha)
        r.add_(q, alpha=-alpha)
        z = dinv * r
        rz_new = hda.dot(r, z, group=group)
        p_loc[:n].mul_(rz_new / rz).add_(z)
        rz = rz_new
        rr = hda.dot(r, r, group=group)
        it += 1
    return x, it, bool(rr <= (rtol * rtol) * bb)
