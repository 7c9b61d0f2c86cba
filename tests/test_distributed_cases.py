"""Load cases sharded across ranks: the partition and the gather, on CPU ranks over gloo
(world size 2 and 3), with a per-rank solve that needs no GPU (U = 2 F + case-dependent
offset, so a case placed in the wrong column or rank shows)."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from wnfea_b200.distributed import case_range


def test_case_range_partitions():
    for k in (0, 1, 5, 31, 32, 33):
        for world in (1, 2, 3, 8):
            spans = [case_range(k, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == k
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        case_range(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, k, q):
    import torch.distributed as dist

    from wnfea_b200.distributed import solve_c3d10_multi_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 7
        F = np.arange(n * k, dtype=np.float64).reshape(n, k) + 0.5
        seen = []

        def fake(Fl):
            seen.append(Fl.shape[1])
            lo = int(round(Fl[0, 0] - 0.5))  # first case of the slice (F[0, j] = j + 0.5)
            U = 2.0 * Fl + lo
            return U, {"case_iterations": np.arange(Fl.shape[1]) + 10 * rank, "case_rel_res": np.full(Fl.shape[1], 1e-9),
                       "status": -5 if rank == 1 else 0, "solve_seconds": 0.1 * (rank + 1)}

        U, st = solve_c3d10_multi_sharded(None, F, local_solve=fake)
        q.put((rank, U, st, seen))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,k", [(2, 32), (2, 5), (3, 7), (3, 2)])
def test_sharded_gather_on_gloo(world, k):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, k, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n = 7
    F = np.arange(n * k, dtype=np.float64).reshape(n, k) + 0.5
    expect = np.empty_like(F)
    its = np.empty(k, dtype=np.int64)
    for r in range(world):
        lo, hi = case_range(k, world, r)
        expect[:, lo:hi] = 2.0 * F[:, lo:hi] + lo
        its[lo:hi] = np.arange(hi - lo) + 10 * r
    for rank, U, st, seen in res:
        lo, hi = case_range(k, world, rank)
        assert seen == ([hi - lo] if hi > lo else [])
        assert U.shape == (n, k)
        np.testing.assert_array_equal(U, expect)
        np.testing.assert_array_equal(st["case_iterations"], its)
        assert st["rank_cases"] == [b - a for a, b in (case_range(k, world, r) for r in range(world))]
        # rank 1's status is reported when it solved any case
        assert st["status"] == (-5 if case_range(k, world, 1)[1] > case_range(k, world, 1)[0] else 0)
        assert st["solve_seconds"] == pytest.approx(0.1 * max(r + 1 for r in range(world)
                                                               if case_range(k, world, r)[1] > case_range(k, world, r)[0]))


@pytest.mark.gpu
def test_sharded_solve_one_rank_nccl_matches_batched_solve():
    """The real per-rank solve and the NCCL gather (a one-rank CUDA process group): the same
    U and per-case iterations as solve_c3d10_multi."""
    import torch.distributed as dist

    from wnfea_b200.distributed import solve_c3d10_multi_sharded
    from wnfea_b200.mesh import generate_c3d10_ibeam_structured, tip_load_cases
    from wnfea_b200.solid_solver import assemble_c3d10_sparse_3dof, solve_c3d10_multi

    m, _ = generate_c3d10_ibeam_structured(n_slices=8, length=0.1, seed=3)
    K, _, _ = assemble_c3d10_sparse_3dof(m)
    F = tip_load_cases(m.mesh_nodes, n_cases=5, seed=2)
    U_ref, st_ref = solve_c3d10_multi(K, F, rtol=1e-8, precision="mixed_fp32")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        U, st = solve_c3d10_multi_sharded(K, F, rtol=1e-8, precision="mixed_fp32")
    finally:
        dist.destroy_process_group()
    np.testing.assert_array_equal(U, U_ref)
    np.testing.assert_array_equal(st["case_iterations"], st_ref["case_iterations"])
    assert st["status"] == 0 and st["rank_cases"] == [5]
