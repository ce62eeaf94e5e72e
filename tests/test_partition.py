"""The row-partitioned product on the CPU (gloo, world sizes 2 and 3): the
reference's MPI scheme (cuts by stored words at leaf row starts,
m_HACApK_base.f90:511-581; owned row segments all-gathered per product,
HACApK_SOLVER.c:106-251, after the rows a rank's leaves reach below its
range are added in by their owners) with the oracle as every rank's local
product.  The
same plumbing runs an engine per GPU over NCCL; that form is not run here
(one GPU per call on this pool)."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build():
    sys.path.insert(0, os.path.join(ROOT, "hacapk-magma_b200"))
    sys.path.insert(0, ROOT)
    from hacapk_b200 import configs
    return configs.c1(3)


def test_row_cuts_assign_every_leaf_once(build_libs):
    from conftest import sphere
    from hacapk_b200 import partition
    H = sphere(4)
    total = sum(partition.leaf_words(H.leaf(ip)) for ip in range(H.nlf))
    starts = {H.leaf(ip).nstrtl - 1 for ip in range(H.nlf)}
    for nranks in (2, 3, 8):
        cuts = partition.row_cuts(H.st, H.nd, nranks)
        assert cuts[0] == 0 and cuts[-1] == H.nd and all(a < b for a, b in zip(cuts, cuts[1:]))
        assert all(c in starts for c in cuts[1:-1])
        subs = [partition.LeafSubset(H.st, H.nd, cuts[r], cuts[r + 1]) for r in range(nranks)]
        assert sum(s.nlf for s in subs) == H.nlf
        words = [sum(partition.leaf_words(s.st.contents.st_lf[k]) for k in range(s.nlf)) for s in subs]
        assert sum(words) == total
        assert max(words) <= 1.5 * total / nranks


def _rank_main(rank, world, pipelined, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    H, b = _build()
    import torch
    import torch.distributed as dist
    import oracle
    from hacapk_b200 import partition
    dist.init_process_group("gloo")
    mv = partition.RowPartitionedMatvec(
        H.st, H.nd, lambda st, nd: (lambda x: torch.from_numpy(oracle.matvec(st, x.numpy()))))
    x = torch.from_numpy(np.random.default_rng(3).standard_normal(H.nd))
    y = mv(x).numpy()
    solve = partition.bicgstab_pipelined if pipelined else partition.bicgstab
    u, steps, relres = solve(mv, torch.from_numpy(b), tol=1e-8, max_iter=500)
    q.put((rank, y, u.numpy(), steps, relres, mv.subset.nlf, mv.exchange_values))
    dist.destroy_process_group()


@pytest.mark.parametrize("world,pipelined", [(2, False), (3, True)])
def test_partitioned_product_and_solve_gloo(build_libs, world, pipelined):
    """Every rank's combined product equals the oracle's; all ranks hold the
    same solution, reached in a step count within one of the same solver
    over the whole product on one process (the flat solver at world size 2,
    the pipelined one at 3), below 1e-8 in the FP64 residual."""
    import oracle
    import torch
    from hacapk_b200 import partition
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, world, pipelined, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    got = sorted((q.get(timeout=300) for _ in ps), key=lambda t: t[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    H, b = _build()
    x = np.random.default_rng(3).standard_normal(H.nd)
    ref = oracle.matvec(H.st, x)
    for rank, y, u, steps, relres, nlf, sent in got:
        assert 0 < nlf < H.nlf  # each rank holds part of the leaves
        assert np.abs(y - ref).max() <= 1e-13 * np.abs(ref).max()
        # the owned segment plus the spill window, not world full-length vectors
        assert sent < 1.5 * H.nd / world + H.nd / 4, (sent, H.nd)
    # every rank holds the same solution (replicated vectors, same sums)
    assert all(np.array_equal(got[0][2], g[2]) and got[0][3] == g[3] for g in got[1:])
    # against the same solve with the whole product on one process
    solve = partition.bicgstab_pipelined if pipelined else partition.bicgstab
    _, n1, rel1 = solve(lambda v: torch.from_numpy(oracle.matvec(H.st, v.numpy())),
                        torch.from_numpy(b), tol=1e-8, max_iter=500)
    assert abs(got[0][3] - n1) <= 1 and got[0][4] < 1e-8
    rel = np.linalg.norm(b - oracle.matvec(H.st, got[0][2])) / np.linalg.norm(b)
    assert rel < 1.05e-8


@pytest.mark.gpu
def test_rank_subsets_as_engines_on_one_gpu(gpu, build_libs):
    """The GPU side of the partitioned form without the collective: each
    rank's leaf subset as its own engine (engine_product), their products
    summed in rank order, equal the oracle's product."""
    import pytest
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    import oracle
    from hacapk_b200 import configs, partition
    H, _ = configs.c1(4)
    cuts = partition.row_cuts(H.st, H.nd, 3)
    subs = [partition.LeafSubset(H.st, H.nd, cuts[r], cuts[r + 1]) for r in range(3)]
    prods = [partition.engine_product(s.st, H.nd) for s in subs]
    x = np.random.default_rng(8).standard_normal(H.nd)
    xd = torch.from_numpy(x).cuda()
    y = prods[0](xd).clone()
    for pr in prods[1:]:
        y += pr(xd)
    torch.cuda.synchronize()
    ref = oracle.matvec(H.st, x)
    assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()


def test_pipelined_bicgstab_converges_like_the_flat_solver(build_libs):
    """The pipelined solver of HACApK_SOLVER_PIPE.c (two reduction points a
    step) reaches 1e-8 in the FP64 residual within a few steps of the flat
    solver, with and without the reference's diagonal right scaling."""
    import oracle
    import torch
    from hacapk_b200 import partition
    H, b = _build()
    mv = lambda v: torch.from_numpy(oracle.matvec(H.st, v.numpy()))  # noqa: E731
    bt = torch.from_numpy(b)
    _, n_flat, _ = partition.bicgstab(mv, bt, tol=1e-8, max_iter=500)
    for scale in (None, torch.from_numpy(partition.diagonal_scaling(H.st, H.nd))):
        u, n, relres = partition.bicgstab_pipelined(mv, bt, tol=1e-8, max_iter=500, scale=scale)
        true = np.linalg.norm(b - oracle.matvec(H.st, u.numpy())) / np.linalg.norm(b)
        assert relres < 1e-8 and true < 1e-7, (scale is None, relres, true)
        assert abs(n - n_flat) <= max(3, n_flat // 4), (n, n_flat)


def test_solvers_stop_at_a_breakdown():
    """A skew-symmetric operator gives b^T A b = 0: the first denominator of
    both host-side solvers is zero.  They stop there and return the start
    iterate (relres 1) instead of raising; a zero rhs takes no step."""
    import torch
    from hacapk_b200.partition import bicgstab, bicgstab_pipelined
    n = 6
    A = torch.zeros(n, n, dtype=torch.float64)
    for i in range(0, n, 2):
        A[i, i + 1], A[i + 1, i] = 1.0, -1.0
    mv = lambda v: A @ v  # noqa: E731
    b = torch.arange(1.0, n + 1, dtype=torch.float64)
    for solve in (bicgstab, bicgstab_pipelined):
        u, steps, relres = solve(mv, b, tol=1e-8, max_iter=50)
        assert steps == 0 and relres == pytest.approx(1.0) and torch.all(u == 0)
        for tol in (1e-8, 0.0):
            u, steps, relres = solve(mv, torch.zeros(n, dtype=torch.float64), tol=tol)
            assert steps == 0 and relres == 0.0 and torch.all(u == 0)


@pytest.mark.gpu
def test_partitioned_product_and_solve_over_nccl_one_rank(gpu, build_libs):
    """The partitioned form's device path over NCCL on the one GPU a call
    gets: a one-rank NCCL group, the rank's engine (engine_product) on device
    vectors, the owned segment all-gathered through NCCL; the product equals
    the oracle's and the replicated-vector BiCGSTAB over it converges.  (More
    ranks need more GPUs; the exchange itself is covered by the gloo tests.)"""
    import socket
    import torch
    import torch.distributed as dist
    import oracle
    from hacapk_b200 import configs, partition
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        H, b = configs.c1(4)
        mv = partition.RowPartitionedMatvec(H.st, H.nd, partition.engine_product)
        x = np.random.default_rng(9).standard_normal(H.nd)
        y = mv(torch.from_numpy(x).cuda())
        torch.cuda.synchronize()
        ref = oracle.matvec(H.st, x)
        assert np.abs(y.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
        u, steps, relres = partition.bicgstab(mv, torch.from_numpy(b).cuda(), tol=1e-8)
        r = b - oracle.matvec(H.st, u.cpu().numpy())
        assert relres < 1e-8 and np.linalg.norm(r) / np.linalg.norm(b) < 1.05e-8
    finally:
        dist.destroy_process_group()
