"""Load cases sharded across ranks, one process per GPU.

The load cases of a multi-RHS solve are independent: each rank takes a contiguous run of the
cases (columns of F), solves them with its own replica of the assembled matrix and the AMG
hierarchy (``solve_c3d10_multi``, no communication during the solve), and the per-rank results
are gathered once at the end with one ``all_gather`` (NCCL for CUDA process groups, gloo on the
CPU).  There is no data-path collective: the matrix, the hierarchy and the solver state never
leave their GPU.
"""

from __future__ import annotations

from typing import Callable

import numpy as np


def case_range(k: int, world: int, rank: int) -> tuple[int, int]:
    """[lo, hi) of the k load cases that rank `rank` of `world` solves: contiguous runs, the
    first k % world ranks one case longer (ranks past k get none)."""
    if world < 1 or not 0 <= rank < world or k < 0:
        raise ValueError(f"bad partition k={k} world={world} rank={rank}")
    base, extra = divmod(k, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _gather_columns(local: np.ndarray, counts: list[int], group, device) -> np.ndarray:
    """(rows, counts[rank]) on every rank -> (rows, sum(counts)) in rank order on every rank."""
    import torch
    import torch.distributed as dist

    rows = local.shape[0]
    width = max(max(counts), 1)
    buf = torch.zeros((width, rows), dtype=torch.float64, device=device)
    if local.shape[1]:
        buf[: local.shape[1]] = torch.from_numpy(np.ascontiguousarray(local.T)).to(device)
    outs = [torch.empty_like(buf) for _ in counts]
    dist.all_gather(outs, buf, group=group)
    cols = [o[:c].cpu().numpy().T for o, c in zip(outs, counts)]
    return np.concatenate(cols, axis=1) if cols else np.zeros((rows, 0))


def solve_c3d10_multi_sharded(K, F: np.ndarray, rtol: float = 1e-8, max_iter: int = 2000,
                              preconditioner: str = "amg", precision: str = "mixed_fp32", amg_params=None,
                              chunk: int = 8, group=None,
                              local_solve: Callable[[np.ndarray], tuple[np.ndarray, dict]] | None = None):
    """``solve_c3d10_multi`` with the load cases split across the ranks of `group` (the default
    process group when None) -> (U, stats) on every rank, U = (n, k) in the original case order.

    Every rank must call it with the same F (the load cases are cheap to replicate) and its own
    K on its own GPU.  stats: ``case_iterations`` / ``case_rel_res`` for all k cases,
    ``status`` = the first nonzero rank status (0 if none), ``rank_cases`` = cases per rank,
    ``solve_seconds`` = the slowest rank's.  ``local_solve`` replaces the per-rank solve
    (F_local -> (U_local, stats)), e.g. to drive the partition and gather without a GPU.
    """
    import torch
    import torch.distributed as dist

    F = np.asarray(F, dtype=np.float64)
    if F.ndim == 1:
        F = F[:, None]
    n, k = F.shape
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    lo, hi = case_range(k, world, rank)
    counts = [b - a for a, b in (case_range(k, world, r) for r in range(world))]
    if local_solve is None:
        from .solid_solver import solve_c3d10_multi

        def local_solve(Fl):
            return solve_c3d10_multi(K, Fl, rtol=rtol, max_iter=max_iter, preconditioner=preconditioner,
                                     precision=precision, amg_params=amg_params, chunk=chunk)
    if hi > lo:
        U_loc, st = local_solve(np.ascontiguousarray(F[:, lo:hi]))
        its = np.asarray(st.get("case_iterations", np.zeros(hi - lo)), dtype=np.float64)
        rel = np.asarray(st.get("case_rel_res", np.zeros(hi - lo)), dtype=np.float64)
        status = float(st.get("status", 0))
        secs = float(st.get("solve_seconds", 0.0))
    else:
        U_loc, its, rel, status, secs = np.zeros((n, 0)), np.zeros(0), np.zeros(0), 0.0, 0.0
    U = _gather_columns(np.asarray(U_loc, dtype=np.float64).reshape(n, hi - lo), counts, group, device)
    per_case = _gather_columns(np.vstack([its, rel]).reshape(2, hi - lo), counts, group, device)
    scal = _gather_columns(np.array([[status], [secs]]), [1] * world, group, device)
    statuses = [int(v) for v in scal[0]]
    stats = {
        "case_iterations": per_case[0].astype(np.int64),
        "case_rel_res": per_case[1],
        "status": next((s for s in statuses if s != 0), 0),
        "rank_status": statuses,
        "rank_cases": counts,
        "solve_seconds": float(scal[1].max()),
    }
    return U, stats
