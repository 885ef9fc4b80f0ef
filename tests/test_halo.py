"""Partitioned meshes on the host (no GPU): the weighted partition against the
oracle's restatement of par::partitionW, each rank's halo plan built from the
oracle's mesh maps (ownership, local elements, local numbering, exchange
lists), the owned rows of y = A x from the local elements alone (oracle
element loop), and the exchange plan run as an all-to-all over gloo ranks."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.cases import points


def test_partition_matches_partitionW(oracle):
    from dendro_b200.halo import partition_weighted
    rng = np.random.default_rng(11)
    cases = [(np.ones(10, int), 3), (np.ones(3, int), 5), (np.ones(0, int), 2), (np.ones(7, int), 1),
             (np.zeros(6, int), 3), (np.array([0, 0, 5, 1, 1, 9, 0, 2]), 3), (np.array([100, 1, 1, 1]), 3)]
    cases += [(rng.integers(0, 50, int(rng.integers(1, 400))), int(rng.integers(1, 17))) for _ in range(60)]
    for w, P in cases:
        got = partition_weighted(len(w), P, w)
        assert np.array_equal(got, oracle.partition_weighted(w, P)), (w, P)
        if w.sum() >= P:  # equal loads up to one unit plus the heaviest item
            loads = np.add.reduceat(np.append(w, 0), got[:-1])[:P] * (np.diff(got) > 0)
            assert loads.max() <= w.sum() // P + 1 + w.max()
    assert np.array_equal(partition_weighted(10, 4), oracle.partition_weighted(np.ones(10, int), 4))


def oracle_maps(oracle, name):
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    mesh = oracle.Mesh(bal, d)
    maps = dict(nlist=mesh.nlist, level=mesh.elev, cnum=mesh.cnum, hmask=mesh.hmask, node_xyz=mesh.node_xyz,
                elem_xyz=np.stack([bal["x"], bal["y"], bal["z"]], 1))
    return mesh, maps, d


def plans(maps, d, P, weights=None):
    from dendro_b200.halo import HaloDA
    return [HaloDA(maps=maps, max_depth=d, rank=r, nranks=P, weights=weights) for r in range(P)]


@pytest.mark.parametrize("name,P", [("gauss2k_d8", 2), ("gauss20k_d10", 3), ("lognormal20k_d12", 5),
                                    ("uniform8k_d9_m4", 4), ("corner_points_d5", 7)])
def test_halo_plan(oracle, name, P):
    mesh, maps, d = oracle_maps(oracle, name)
    H = plans(maps, d, P)
    nl = mesh.nlist.astype(np.int64)
    nf = H[0].node_first
    assert nf[0] == 0 and nf[-1] == mesh.N and np.all(np.diff(nf) >= 0)
    owner = np.searchsorted(nf, np.arange(mesh.N), side="right") - 1
    eowner = owner[nl]                                     # [E, 8]
    seen = np.zeros(mesh.E, int)
    for r, h in enumerate(H):
        assert np.array_equal(h.node_first, nf) and np.array_equal(h.elem_first, H[0].elem_first)
        assert h.first_owned == nf[r] and h.n_owned == nf[r + 1] - nf[r]
        touches = (eowner == r).any(1)
        local = np.sort(np.concatenate([h.independent, h.dependent]))
        assert np.array_equal(local, np.nonzero(touches)[0])   # every element with an owned vertex
        assert (eowner[h.independent] == r).all()
        assert ((eowner[h.dependent] != r).any(1)).all()
        seen[local] += 1
        l2g = h.local_to_global()
        assert np.all(np.diff(h.ghosts.astype(np.int64)) > 0)
        assert np.array_equal(np.bincount(owner[h.ghosts], minlength=P), h.recv_counts)
        assert h.recv_counts[r] == 0 and h.send_counts[r] == 0
        assert np.array_equal(h.ind_nlist.astype(np.int64) + h.first_owned, nl[h.independent])
        assert np.array_equal(l2g[h.dep_nlist], nl[h.dependent])
        # every local node is owned or read by a dependent element
        used = np.zeros(h.n_local, bool)
        used[: h.n_owned] = True
        used[h.dep_nlist.ravel()] = True
        assert used.all()
    assert (seen >= 1).all()
    # what r sends to q is what q receives from r, in q's ghost order
    for r, h in enumerate(H):
        off = np.concatenate([[0], np.cumsum(h.send_counts)])
        for q, g in enumerate(H):
            sent = h.send_idx[off[q]:off[q + 1]].astype(np.int64) + h.first_owned
            roff = np.concatenate([[0], np.cumsum(g.recv_counts)])
            assert np.array_equal(sent, g.ghosts[roff[r]:roff[r + 1]].astype(np.int64)), (r, q)


@pytest.mark.parametrize("name,P", [("gauss20k_d10", 2), ("lognormal20k_d12", 4)])
def test_local_elements_complete_owned_rows(oracle, name, P):
    """The owned rows of y = A x summed over a rank's local elements only
    equal the whole mesh's, with weights that skew the partition."""
    mesh, maps, d = oracle_maps(oracle, name)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, mesh.N)
    coef = np.stack([np.where(rng.uniform(size=mesh.E) < 0.3, 1e4, 1.0), rng.uniform(0.5, 2, mesh.E)], 1)
    y = mesh.matvec(x, coef.reshape(-1))
    w = rng.integers(1, 9, mesh.E)
    for h in plans(maps, d, P, weights=w):
        local = np.concatenate([h.independent, h.dependent])
        yl = mesh.matvec_elems(x, local, coef.reshape(-1))
        sl = slice(h.first_owned, h.first_owned + h.n_owned)
        assert np.allclose(yl[sl], y[sl], rtol=1e-13, atol=1e-13 * np.abs(y).max())


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _exchange_worker(rank, world, port, name, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle
        from dendro_b200.halo import HaloDA
        mesh, maps, d = oracle_maps(oracle, name)
        h = HaloDA(maps=maps, max_depth=d)            # rank and size from the process group
        xg = np.random.default_rng(9).uniform(-1, 1, mesh.N)
        # owners -> readers (ReadFromGhosts): the pack is the send_idx gather
        x = torch.zeros(h.n_local, dtype=torch.float64)
        x[:h.n_owned] = torch.from_numpy(xg[h.first_owned:h.first_owned + h.n_owned])
        send = x[torch.from_numpy(h.send_idx.astype(np.int64))]
        dist.all_to_all_single(x[h.n_owned:], send, [int(c) for c in h.recv_counts],
                               [int(c) for c in h.send_counts])
        ok_read = bool(np.array_equal(x.numpy(), xg[h.local_to_global()]))
        # readers -> owners (WriteToGhosts): every ghost slot sends 1, owners add
        y = torch.zeros(h.n_local, dtype=torch.float64)
        y[h.n_owned:] = 1.0
        recv = torch.empty(len(h.send_idx), dtype=torch.float64)
        dist.all_to_all_single(recv, y[h.n_owned:], [int(c) for c in h.send_counts],
                               [int(c) for c in h.recv_counts])
        readers = np.zeros(h.n_owned)
        np.add.at(readers, h.send_idx.astype(np.int64), recv.numpy())
        # every owned node is read by the ranks that hold it as a ghost
        holders = np.zeros(mesh.N)
        for q in range(world):
            if q != rank:
                g = HaloDA(maps=maps, max_depth=d, rank=q, nranks=world)
                holders[g.ghosts.astype(np.int64)] += 1
        ok_write = bool(np.array_equal(readers, holders[h.first_owned:h.first_owned + h.n_owned]))
        out[rank] = (ok_read, ok_write, int(h.n_ghost), int(sum(h.send_counts)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_over_gloo(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, "gauss20k_d10", out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    assert all(res[r][0] and res[r][1] for r in range(world)), res
    assert all(res[r][2] > 0 and res[r][3] > 0 for r in range(world))


class _OracleLocalOp:
    """Stand-in for HaloJacobian2 on the host: the exchange over gloo from the
    halo plan, the owned rows from the oracle's element loop over the rank's
    local elements."""

    def __init__(self, h, mesh, coef):
        self.hda, self.mesh, self.coef = h, mesh, coef
        self.local = np.concatenate([h.independent, h.dependent])
        self.l2g = h.local_to_global()
        self.own = slice(h.first_owned, h.first_owned + h.n_owned)

    def mult(self, x_local, group=None):
        import torch
        import torch.distributed as dist
        h = self.hda
        send = x_local[torch.from_numpy(h.send_idx.astype(np.int64))]
        dist.all_to_all_single(x_local[h.n_owned:], send, [int(c) for c in h.recv_counts],
                               [int(c) for c in h.send_counts])
        xg = np.zeros(self.mesh.N)
        xg[self.l2g] = x_local.numpy()
        y = torch.zeros_like(x_local)
        y[:h.n_owned] = torch.from_numpy(self.mesh.matvec_elems(xg, self.local, self.coef)[self.own])
        return y

    def getDiagonal(self):
        import torch
        return torch.from_numpy(self.mesh.diagonal(self.coef)[self.own].copy())


def _cg_worker(rank, world, port, name, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle
        from dendro_b200.halo import HaloDA, halo_cg
        mesh, maps, d = oracle_maps(oracle, name)
        h = HaloDA(maps=maps, max_depth=d)
        coef = np.tile([1.0, 1.0], mesh.E)
        b = np.random.default_rng(4).uniform(-1, 1, mesh.N)
        x, it, conv = halo_cg(_OracleLocalOp(h, mesh, coef), torch.from_numpy(b[h.first_owned:h.first_owned + h.n_owned]),
                              rtol=1e-8, maxit=2000)
        out[rank] = (h.first_owned, x.numpy(), it, conv)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _jacobi_cg(A, d, b, rtol, maxit):
    x = np.zeros_like(b)
    r = b.copy()
    z = r / d
    p = z.copy()
    rz, bb = r @ z, b @ b
    it = 0
    while it < maxit and r @ r > rtol * rtol * bb:
        q = A(p)
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        z = r / d
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
        it += 1
    return x, it


def test_jacobi_cg_over_gloo_ranks(oracle):
    """halo_cg's distributed steps (local layout, exchanges, FP64 dot sums over
    ranks) solve the whole mesh's system like one process does."""
    world, name = 2, "gauss2k_d8"
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_cg_worker, args=(r, world, port, name, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        res = dict(out)
    mesh, _, _ = oracle_maps(oracle, name)
    x = np.concatenate([res[r][1] for r in range(world)])
    assert res[0][2] == res[1][2] and res[0][3] and res[1][3]
    b = np.random.default_rng(4).uniform(-1, 1, mesh.N)
    assert np.linalg.norm(mesh.matvec(x) - b) <= 1.01e-8 * np.linalg.norm(b)
    _, it_ref = _jacobi_cg(mesh.matvec, mesh.diagonal(), b, 1e-8, 2000)
    assert abs(res[0][2] - it_ref) <= 1


def test_parcsr_plan(oracle):
    """The exchange plan of a row-partitioned sparse matrix: ghosts are the
    columns a rank's rows read that it does not own, and what r sends to q is
    what q receives from r, in q's ghost order."""
    from dendro_b200.halo import ParCSR, partition_weighted
    rng = np.random.default_rng(17)
    nrows, ncols, P = 700, 400, 4
    nnz_row = rng.integers(0, 9, nrows)
    ptr_ = np.concatenate([[0], np.cumsum(nnz_row)]).astype(np.uint32)
    col = np.concatenate([np.sort(rng.choice(ncols, k, replace=False)) for k in nnz_row]).astype(np.uint32)
    val = rng.uniform(-1, 1, len(col))
    rf, cf = partition_weighted(nrows, P), partition_weighted(ncols, P, rng.integers(1, 5, ncols))
    mats = [ParCSR(ptr_, col, val, nrows, ncols, rf, cf, r, P) for r in range(P)]
    owner = np.searchsorted(cf, np.arange(ncols), side="right") - 1
    from dendro_b200._lib import lib, ptr
    ghosts, sends = [], []
    for r, pc in enumerate(mats):
        assert pc.n_rows == rf[r + 1] - rf[r] and pc.n_cols_owned == cf[r + 1] - cf[r]
        assert pc.nnz == ptr_[rf[r + 1]] - ptr_[rf[r]]
        g = np.empty(pc.n_ghost, np.uint32)
        s = np.empty(pc.n_send, np.uint32)
        assert lib().dg_parcsr_comm(pc.h, None, None, ptr(s), ptr(g)) == 0
        cols = col[ptr_[rf[r]]:ptr_[rf[r + 1]]]
        assert np.array_equal(g, np.unique(cols[owner[cols] != r]))
        assert np.array_equal(np.bincount(owner[g], minlength=P), pc.recv_counts)
        ghosts.append(g)
        sends.append(s)
    for r, pc in enumerate(mats):
        off = np.concatenate([[0], np.cumsum(pc.send_counts)])
        for q, qc in enumerate(mats):
            roff = np.concatenate([[0], np.cumsum(qc.recv_counts)])
            assert np.array_equal(sends[r][off[q]:off[q + 1]].astype(np.int64) + cf[r],
                                  ghosts[q][roff[r]:roff[r + 1]].astype(np.int64))


def _comm_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from dendro_b200.halo import TorchComm
        c = TorchComm()
        counts = [3, 0, 5][:world]
        t = torch.arange(counts[rank], dtype=torch.float64) + 10 * rank
        g = c.all_gather_v(t, counts)
        s = c.all_reduce(torch.tensor([1.0 + rank], dtype=torch.float64))
        out[rank] = (c.rank, c.size, g.tolist(), float(s.item()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_torch_comm_over_gloo():
    """The communicator's uneven gather and sum over gloo ranks."""
    world = 3
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_comm_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        assert res[r][:2] == (r, world)
        assert res[r][2] == [0.0, 1.0, 2.0, 20.0, 21.0, 22.0, 23.0, 24.0]
        assert res[r][3] == 6.0


def test_halo_and_parcsr_reject_bad_input(oracle):
    """Bad ranks, node ids out of Morton order, ranges that do not cover the
    rows, columns out of range: DG_EINVAL with no GPU touched."""
    from dendro_b200._lib import DendroError
    from dendro_b200.halo import HaloDA, ParCSR
    mesh, maps, d = oracle_maps(oracle, "gauss2k_d8")
    with pytest.raises(DendroError):
        HaloDA(maps=maps, max_depth=d, rank=3, nranks=3)
    with pytest.raises(DendroError):
        HaloDA(maps=maps, max_depth=d, rank=-1, nranks=2)
    bad = dict(maps)
    bad["node_xyz"] = maps["node_xyz"][::-1].copy()          # anchors out of Morton order
    with pytest.raises(DendroError):
        HaloDA(maps=bad, max_depth=d, rank=0, nranks=2)
    bad = dict(maps)
    bad["nlist"] = maps["nlist"].copy()
    bad["nlist"][5, 3] = mesh.N                              # node id out of range
    with pytest.raises(DendroError):
        HaloDA(maps=bad, max_depth=d, rank=0, nranks=2)
    ptr_ = np.array([0, 2, 3], np.uint32)
    col = np.array([0, 3, 1], np.uint32)
    val = np.ones(3)
    with pytest.raises(DendroError):                         # row ranges do not reach the last row
        ParCSR(ptr_, col, val, 2, 4, [0, 1, 1], [0, 2, 4], 0, 2)
    with pytest.raises(DendroError):                         # column 3 beyond 3 columns
        ParCSR(ptr_, col, val, 2, 3, [0, 1, 2], [0, 2, 3], 0, 2)
    with pytest.raises(DendroError):                         # descending column ranges
        ParCSR(ptr_, col, val, 2, 4, [0, 1, 2], [0, 3, 2], 0, 2)
    pc = ParCSR(ptr_, col, val, 2, 4, [0, 1, 2], [0, 2, 4], 1, 2)
    assert (pc.n_rows, pc.n_cols_owned, pc.n_ghost, pc.nnz) == (1, 2, 1, 1)
    # short host arrays are refused before the library reads them
    for bad_args in ((ptr_[:2], col, val, 2, 4, [0, 1, 2], [0, 2, 4], 1, 2),   # ptr shorter than nrows + 1
                     (ptr_, col[:2], val, 2, 4, [0, 1, 2], [0, 2, 4], 1, 2),   # col shorter than ptr[-1]
                     (ptr_, col, val[:1], 2, 4, [0, 1, 2], [0, 2, 4], 1, 2),   # val shorter than ptr[-1]
                     (ptr_, col, val, 2, 4, [0, 2], [0, 2, 4], 1, 2),          # row_first without nranks + 1
                     (ptr_, col, val, 2, 4, [0, 1, 2], [0, 4], 1, 2)):         # col_first without nranks + 1
        with pytest.raises(ValueError):
            ParCSR(*bad_args)
    E = len(maps["level"])
    with pytest.raises(ValueError):                          # one weight short
        HaloDA(maps=maps, max_depth=d, rank=0, nranks=2, weights=np.ones(E - 1, np.uint32))
    for key in ("nlist", "cnum", "hmask", "elem_xyz"):
        bad = dict(maps)
        bad[key] = maps[key][:-1]                            # maps that disagree in length
        with pytest.raises(ValueError):
            HaloDA(maps=bad, max_depth=d, rank=0, nranks=2)


def test_single_rank_defaults(oracle):
    """Without a process group the communicator is one rank: every element is
    independent, nothing is sent, and the collectives pass values through."""
    import torch
    from dendro_b200.halo import HaloDA, TorchComm
    c = TorchComm()
    assert (c.rank, c.size) == (0, 1)
    t = torch.arange(4, dtype=torch.float64)
    out = torch.empty(0, dtype=torch.float64)
    assert c.all_to_all_single(out, torch.empty(0, dtype=torch.float64), [0], [0]) is None
    assert torch.equal(c.all_reduce(t.clone()), t) and torch.equal(c.all_gather_v(t, [4]), t)
    mesh, maps, d = oracle_maps(oracle, "gauss2k_d8")
    h = HaloDA(maps=maps, max_depth=d)
    assert (h.rank, h.nranks, h.n_ghost, len(h.dependent)) == (0, 1, 0, 0)
    assert h.n_owned == mesh.N and len(h.independent) == mesh.E and len(h.send_idx) == 0
