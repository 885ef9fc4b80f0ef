"""Partitioned meshes on one GPU: every rank's part built in one process, the
all-to-all between them done by the test from the product's pack kernel (no
ranks wait on one another).  The owned rows of y = A x and of the diagonal
against the oracle's whole-mesh results, the accumulation kernel against a
sequential host sum, and the distributed operator and Jacobi CG on one rank."""
import numpy as np
import pytest

from dendro_b200 import inputs as I
from tests.cases import points

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def setup(gpu, oracle, name, P, weights=None):
    from dendro_b200.halo import HaloDA
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    da = gpu.DA(gpu.Octree.from_octants(bal, d))
    ref = oracle.Mesh(bal, d)
    H = [HaloDA(da, rank=r, nranks=P, weights=weights) for r in range(P)]
    return da, ref, H


def offsets(counts):
    return np.concatenate([[0], np.cumsum(counts)])


def emulate_read(H, xs):
    """The all-to-all of read_from_ghosts, between the ranks' buffers."""
    import torch
    sends = [h.pack(x) for h, x in zip(H, xs)]
    for r, h in enumerate(H):
        parts = [sends[q][offsets(g.send_counts)[r]:offsets(g.send_counts)[r + 1]] for q, g in enumerate(H)]
        xs[r][h.n_owned:] = torch.cat(parts)


@pytest.mark.parametrize("name,P", [("gauss20k_d10", 2), ("lognormal20k_d12", 4), ("uniform8k_d9_m4", 3),
                                    ("corner_points_d5", 5)])
def test_partitioned_operator_matches_oracle(gpu, oracle, name, P):
    import torch
    from dendro_b200.halo import HaloJacobian2
    da, ref, H = setup(gpu, oracle, name, P)
    coef = I.sphere_coefficients(da.elementCenters())
    x = I.uniform_rhs(ref.N, 21)
    xs = [h.local_vector(x[h.first_owned:h.first_owned + h.n_owned]) for h in H]
    emulate_read(H, xs)
    for h, xl in zip(H, xs):
        assert np.array_equal(xl.cpu().numpy(), x[h.local_to_global()])
    ops = [HaloJacobian2(h, coef) for h in H]
    y = np.concatenate([op.apply_local(xl)[:op.hda.n_owned].cpu().numpy() for op, xl in zip(ops, xs)])
    assert rel(y, ref.matvec(x, coef)) < TOL
    d = np.concatenate([op.getDiagonal().cpu().numpy() for op in ops])
    assert rel(d, ref.diagonal(coef)) < TOL
    # the whole-mesh operator on the GPU gives the same owned rows
    yg = gpu.Jacobian2(da, coef).mult(torch.tensor(x, device="cuda")).cpu().numpy()
    assert rel(y, yg) < TOL


def test_accumulate_matches_sequential_sum(gpu, oracle):
    """write_to_ghosts' accumulation: y[send_idx[k]] += recv[k] in order."""
    import torch
    _, _, H = setup(gpu, oracle, "lognormal20k_d12", 3)
    rng = np.random.default_rng(5)
    ys = [torch.tensor(rng.uniform(-1, 1, h.n_local), device="cuda") for h in H]
    ghost = [y[h.n_owned:].clone() for h, y in zip(H, ys)]
    for r, h in enumerate(H):
        recv = torch.cat([ghost[q][offsets(g.recv_counts)[r]:offsets(g.recv_counts)[r + 1]]
                          for q, g in enumerate(H)])
        expect = ys[r].cpu().numpy().copy()
        np.add.at(expect, h.send_idx.astype(np.int64), recv.cpu().numpy())
        got = h.accumulate(recv, ys[r]).cpu().numpy()
        assert np.array_equal(got, expect)


@pytest.mark.parametrize("name,P", [("lognormal20k_d12", 4), ("gauss20k_d10", 2)])
def test_partitioned_every_launch_shape(gpu, oracle, name, P):
    """Each operator kernel, fixed in turn, on the independent and dependent
    element subsets of every part: octets there lack children that the
    other subset (or another rank) holds, while their hanging points still
    fold onto those children's corners."""
    from dendro_b200.halo import HaloJacobian2
    da, ref, H = setup(gpu, oracle, name, P)
    coef = I.sphere_coefficients(da.elementCenters())
    x = I.uniform_rhs(ref.N, 21)
    xs = [h.local_vector(x[h.first_owned:h.first_owned + h.n_owned]) for h in H]
    emulate_read(H, xs)
    ops = [HaloJacobian2(h, coef) for h in H]
    y_ref = ref.matvec(x, coef)
    mats = [A for op in ops for A in (op.A_ind, op.A_dep) if A is not None]
    for v in range(mats[0].kernel_count()):
        for A in mats:
            A.set_kernel(v, 0)
        y = np.concatenate([op.apply_local(xl)[:op.hda.n_owned].cpu().numpy() for op, xl in zip(ops, xs)])
        assert rel(y, y_ref) < TOL, (v, mats[0].kernel_name(0))


def test_weighted_partition_and_one_rank_cg(gpu, oracle):
    import torch
    from dendro_b200.halo import HaloDA, HaloJacobian2, halo_cg
    # element weights skew the ranges; the owned rows stay exact
    pts, d, m = points("gauss20k_d10")
    E = len(oracle.balance(oracle.points2octree(pts, d, m), d))
    w = np.where(np.arange(E) < E // 4, 9, 1).astype(np.uint32)
    da, ref, H = setup(gpu, oracle, "gauss20k_d10", 3, weights=w)
    assert not np.array_equal(H[0].elem_first, HaloDA(da, rank=0, nranks=3).elem_first)
    x = I.uniform_rhs(ref.N, 2)
    xs = [h.local_vector(x[h.first_owned:h.first_owned + h.n_owned]) for h in H]
    emulate_read(H, xs)
    y = np.concatenate([HaloJacobian2(h).apply_local(xl)[:h.n_owned].cpu().numpy() for h, xl in zip(H, xs)])
    assert rel(y, ref.matvec(x)) < TOL
    # one rank: every element independent, mult without an exchange, CG to 1e-8
    h1 = HaloDA(da, rank=0, nranks=1)
    assert h1.n_ghost == 0 and len(h1.dependent) == 0 and len(h1.independent) == da.E
    A = HaloJacobian2(h1)
    b = I.uniform_rhs(ref.N, 3)
    xs1, it, conv = halo_cg(A, torch.tensor(b, device="cuda"), rtol=1e-8, maxit=3000)
    assert conv and it > 0
    assert np.linalg.norm(ref.matvec(xs1.cpu().numpy()) - b) <= 1.01e-8 * np.linalg.norm(b)


def test_mult_add(gpu, oracle):
    """y += A x (the dependent elements' launch) against y + (A x)."""
    import torch
    pts, d, m = points("lognormal20k_d12")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    da = gpu.DA(gpu.Octree.from_octants(bal, d))
    coef = I.sphere_coefficients(da.elementCenters())
    A = gpu.Jacobian2(da, coef)
    x = torch.tensor(I.uniform_rhs(da.N, 4), device="cuda")
    y0 = torch.tensor(I.uniform_rhs(da.N, 5), device="cuda")
    y = A.mult_add(x, y0.clone())
    expect = y0.cpu().numpy() + oracle.Mesh(bal, d).matvec(x.cpu().numpy(), coef)
    assert rel(y.cpu().numpy(), expect) < TOL
    with pytest.raises(gpu.DendroError):
        gpu.Elasticity(da, 0.4, 0.6).mult_add(torch.zeros(3 * da.N, dtype=torch.float64, device="cuda"),
                                              torch.zeros(3 * da.N, dtype=torch.float64, device="cuda"))



def test_operator_and_cg_over_thread_ranks(gpu, oracle):
    """mult with its exchange and Jacobi CG, the ranks run as threads on the
    one GPU (exchanges and sums through the host)."""
    import torch
    from dendro_b200.halo import HaloDA, HaloJacobian2, halo_cg
    from tests.threadcomm import ThreadComm, run_ranks
    P = 3
    pts, d, m = points("gauss20k_d10")
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    da = gpu.DA(gpu.Octree.from_octants(bal, d))
    ref = oracle.Mesh(bal, d)
    coef = I.sphere_coefficients(da.elementCenters())
    tc = ThreadComm(P)
    H = [HaloDA(da, comm=tc.rank_comm(r)) for r in range(P)]
    ops = [HaloJacobian2(h, coef) for h in H]
    ops1 = [HaloJacobian2(h) for h in H]
    x = I.uniform_rhs(ref.N, 31)
    b = I.uniform_rhs(ref.N, 32)

    def body(r):
        h = H[r]
        own = slice(h.first_owned, h.first_owned + h.n_owned)
        y = ops[r].mult(h.local_vector(x[own]))[:h.n_owned].cpu().numpy()
        y2 = ops[r].mult(h.local_vector(x[own]), overlap=False)[:h.n_owned].cpu().numpy()
        # WriteToGhosts: every ghost slot holds 1, the owners add what they receive
        w = h.local_vector()
        w[h.n_owned:] = 1.0
        readers = h.write_to_ghosts(w)[:h.n_owned].cpu().numpy()
        xs, it, conv = halo_cg(ops1[r], torch.tensor(b[own], device="cuda"), rtol=1e-8, maxit=3000)
        return y, y2, xs.cpu().numpy(), it, conv, readers

    res = run_ranks(P, body)
    holders = np.zeros(ref.N)
    for h in H:
        holders[h.ghosts.astype(np.int64)] += 1
    assert np.array_equal(np.concatenate([t[5] for t in res]), holders) and holders.max() > 0
    y_ref = ref.matvec(x, coef)
    assert rel(np.concatenate([t[0] for t in res]), y_ref) < TOL
    assert rel(np.concatenate([t[1] for t in res]), y_ref) < TOL
    assert len({t[3] for t in res}) == 1 and all(t[4] for t in res)
    xs = np.concatenate([t[2] for t in res])
    assert np.linalg.norm(ref.matvec(xs) - b) <= 1.01e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("name,P", [("gauss20k_d10", 2), ("lognormal20k_d12", 3)])
def test_damg_over_thread_ranks(gpu, oracle, name, P):
    """The partitioned V-cycle against the single-GPU V-cycle on the same
    hierarchy, and the partitioned PCG's iterations and residual."""
    import torch
    from dendro_b200.halo import HaloDAMG
    from dendro_b200.learned import vcycle
    from tests.threadcomm import ThreadComm, run_ranks
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    octree = gpu.Octree.from_octants(bal, d)
    coef = I.sphere_coefficients(gpu.DA(octree).elementCenters())
    single = gpu.DAMG(octree)
    single.setKSP(coef)
    b = I.uniform_rhs(int(single.N[0]), 41)
    z_ref = vcycle(single, torch.tensor(b, device="cuda")).cpu().numpy()
    _, rep = single.solve(b)
    tc = ThreadComm(P)
    M = [HaloDAMG(octree, coef, comm=tc.rank_comm(r)) for r in range(P)]
    assert all(mm.nlevels == single.nlevels for mm in M)

    def body(r):
        own = slice(M[r].first_owned, M[r].first_owned + M[r].n_owned)
        bo = torch.tensor(b[own], device="cuda")
        z = M[r].vcycle(bo).cpu().numpy()
        x, it, conv, rr = M[r].solve(bo, rtol=1e-8)
        return z, x.cpu().numpy(), it, conv

    res = run_ranks(P, body)
    assert rel(np.concatenate([t[0] for t in res]), z_ref) < 1e-10
    its = {t[2] for t in res}
    assert len(its) == 1 and all(t[3] for t in res)
    assert abs(its.pop() - rep["iterations"]) <= 1
    x = np.concatenate([t[1] for t in res])
    fine = oracle.Mesh(bal, d)
    assert np.linalg.norm(fine.matvec(x, coef) - b) <= 1.01e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("name,P", [("gauss20k_d10", 2), ("lognormal20k_d12", 3)])
def test_damg_fp32_over_thread_ranks(gpu, oracle, name, P):
    """The partitioned FP32 inner V-cycle against the single-GPU FP32 and FP64
    V-cycles (FP32 tolerance, 2e-5), and its FP64 flexible PCG against the
    single-GPU mixed-precision solve (iterations +-1, FP64 residual)."""
    import torch
    from dendro_b200.halo import HaloDAMG
    from dendro_b200.learned import vcycle
    from tests.threadcomm import ThreadComm, run_ranks
    pts, d, m = points(name)
    bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    octree = gpu.Octree.from_octants(bal, d)
    coef = I.sphere_coefficients(gpu.DA(octree).elementCenters())
    single64 = gpu.DAMG(octree)
    single64.setKSP(coef)
    single32 = gpu.DAMG(octree, inner_prec=1)
    single32.setKSP(coef)
    b = I.uniform_rhs(int(single64.N[0]), 43)
    bd = torch.tensor(b, device="cuda")
    z64 = vcycle(single64, bd).cpu().numpy()
    z32 = vcycle(single32, bd).cpu().numpy()
    _, rep = single32.solve(b)
    tc = ThreadComm(P)
    M = [HaloDAMG(octree, coef, comm=tc.rank_comm(r), inner_prec=1) for r in range(P)]

    def body(r):
        own = slice(M[r].first_owned, M[r].first_owned + M[r].n_owned)
        bo = torch.tensor(b[own], device="cuda")
        z = M[r].vcycle(bo.float())
        assert z.dtype == torch.float32
        x, it, conv, rr = M[r].solve(bo, rtol=1e-8)
        return z.double().cpu().numpy(), x.cpu().numpy(), it, conv

    res = run_ranks(P, body)
    z = np.concatenate([t[0] for t in res])
    assert rel(z, z32) < 2e-5 and rel(z, z64) < 2e-5
    its = {t[2] for t in res}
    assert len(its) == 1 and all(t[3] for t in res)
    assert abs(its.pop() - rep["iterations"]) <= 1
    x = np.concatenate([t[1] for t in res])
    fine = oracle.Mesh(bal, d)
    assert np.linalg.norm(fine.matvec(x, coef) - b) <= 1.01e-8 * np.linalg.norm(b)


@pytest.mark.parametrize("name,P", [("root", 2), ("corner_points_d5", 4)])
def test_more_ranks_than_work(gpu, oracle, name, P):
    """Ranks that own no nodes (the one-element mesh over 2 ranks; a
    15-element mesh over 4, where one rank's elements anchor no node) still
    take part in every exchange; the partitioned V-cycle and PCG match the
    single-GPU ones."""
    import torch
    from dendro_b200.halo import HaloDAMG
    from dendro_b200.learned import vcycle
    from tests.threadcomm import ThreadComm, run_ranks
    if name == "root":
        d = 6
        bal = oracle.points2octree(np.zeros((0, 3)), d, 1)
    else:
        pts, d, m = points(name)
        bal = oracle.balance(oracle.points2octree(pts, d, m), d)
    octree = gpu.Octree.from_octants(bal, d)
    single = gpu.DAMG(octree)
    single.setKSP()
    b = I.uniform_rhs(int(single.N[0]), 51)
    z_ref = vcycle(single, torch.tensor(b, device="cuda")).cpu().numpy()
    tc = ThreadComm(P)
    M = [HaloDAMG(octree, comm=tc.rank_comm(r)) for r in range(P)]
    assert min(mm.n_owned for mm in M) == 0

    def body(r):
        own = slice(M[r].first_owned, M[r].first_owned + M[r].n_owned)
        bo = torch.tensor(b[own], device="cuda")
        z = M[r].vcycle(bo).cpu().numpy()
        x, it, conv, _ = M[r].solve(bo, rtol=1e-8)
        return z, x.cpu().numpy(), it, conv

    res = run_ranks(P, body)
    assert rel(np.concatenate([t[0] for t in res]), z_ref) < 1e-10
    assert all(t[3] for t in res)
    x = np.concatenate([t[1] for t in res])
    fine = oracle.Mesh(bal, d)
    assert np.linalg.norm(fine.matvec(x) - b) <= 1.01e-8 * np.linalg.norm(b)
