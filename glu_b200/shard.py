"""Coulomb gauge fixing of one configuration sharded by time slices over the
ranks of a torch.distributed process group (one process per GPU).

The time slices of a Coulomb fix are independent problems (GLU's
Coulomb_FA, src/Gfix/CFACG.c:531-636, fixes them one after the other), so
rank r fixes a contiguous block of slices of its own.  The one exchange is a
boundary: the temporal links of a block's last slice need the gauge field of
the following slice, which the next rank owns; every rank sends the field of
its first slice to the preceding rank (a ring, NCCL point-to-point on GPUs)
and then completes those links.  With one rank the ring closes on itself
and the result is gfix_coulomb's.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np


def slice_blocks(lt: int, world: int, costs=None) -> list[tuple[int, int]]:
    """Contiguous blocks [t0, t1) of the lt slices, one per rank, every block
    holding at least two slices.

    Without costs the blocks hold equal numbers of slices.  With costs (the
    expected cost of each slice, e.g. its volume times the iterations it is
    expected to take: per-slice counts vary severalfold within one
    configuration) the blocks minimise the largest block cost, exactly (a
    linear-partition dynamic programme over the prefix sums)."""
    if world < 1 or lt < 2 * world:
        raise ValueError(f"{lt} time slices cannot give {world} ranks two each")
    if costs is None:
        base, extra = divmod(lt, world)
        out, t0 = [], 0
        for r in range(world):
            n = base + (1 if r < extra else 0)
            out.append((t0, t0 + n))
            t0 += n
        return out
    c = np.asarray(costs, dtype=np.float64)
    if c.shape != (lt,) or not np.all(np.isfinite(c)) or np.any(c < 0):
        raise ValueError("costs must be lt finite, non-negative numbers")
    pre = np.concatenate([[0.0], np.cumsum(c)])
    inf = float("inf")
    # best[r][t]: the least largest block cost of slices [0, t) in r blocks
    best = np.full((world + 1, lt + 1), inf)
    cut = np.zeros((world + 1, lt + 1), dtype=np.int64)
    best[0][0] = 0.0
    for r in range(1, world + 1):
        for t in range(2 * r, lt - 2 * (world - r) + 1):
            s = np.arange(2 * (r - 1), t - 1)  # the last block is [s, t)
            cand = np.maximum(best[r - 1][s], pre[t] - pre[s])
            k = int(np.argmin(cand))
            best[r][t], cut[r][t] = cand[k], s[k]
    out, t = [], lt
    for r in range(world, 0, -1):
        s = int(cut[r][t])
        out.append((s, t))
        t = s
    return out[::-1]


@dataclass
class ShardResult:
    iters: int             # summed over all ranks (GLU's total)
    slice_theta: np.ndarray
    slice_iters: np.ndarray
    restarts: int


def _lib_solver(params):
    """The library's gfix_coulomb_slices / _finish on device tensors."""
    from . import _lib
    from ._lib import GfixResult, check
    lib = _lib.load()

    def solve(links, dims, g_first, g_last):
        cd = (C.c_size_t * 4)(*dims)
        r = GfixResult()
        th = np.zeros(dims[3])
        it = np.zeros(dims[3], dtype=np.uintp)
        check(lib.gfix_coulomb_slices(links.data_ptr(), cd, C.byref(params),
                                      C.byref(r),
                                      th.ctypes.data_as(C.POINTER(C.c_double)),
                                      it.ctypes.data_as(C.POINTER(C.c_size_t)),
                                      g_first.data_ptr(), g_last.data_ptr()))
        return int(r.iters), th, it.astype(np.int64), int(r.restarts)

    def finish(links, dims, g_last, g_next):
        cd = (C.c_size_t * 4)(*dims)
        check(lib.gfix_coulomb_slices_finish(links.data_ptr(), cd, g_last.data_ptr(),
                                             g_next.data_ptr()))

    return solve, finish


def coulomb_sharded(links, dims, group=None, params=None, solver=None):
    """Fix this rank's block of slices in place.

    links: this rank's block, a float64 tensor of double[V][4][9][2] (on the
    rank's GPU for the library solver); dims: the block's (Lx, Ly, Lz, T).
    params: a GfixParams (the library solver); solver: (solve, finish)
    callables with the library's contract, for other back ends.
    Collective over `group`: every rank calls it once."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    solve, finish = solver if solver is not None else _lib_solver(params)
    lcu = int(dims[0] * dims[1] * dims[2])
    g_first = torch.empty(9 * lcu * 2, dtype=torch.float64, device=links.device)
    g_last = torch.empty_like(g_first)
    iters, th, it, restarts = solve(links, dims, g_first, g_last)
    if world == 1:
        g_next = g_first
    else:
        g_next = torch.empty_like(g_first)
        prev, nxt = (rank - 1) % world, (rank + 1) % world
        # group-relative ranks -> global ranks for the point-to-point calls
        if group is not None:
            prev = dist.get_global_rank(group, prev)
            nxt = dist.get_global_rank(group, nxt)
        reqs = [dist.isend(g_first, prev, group=group),
                dist.irecv(g_next, nxt, group=group)]
        for q in reqs:
            q.wait()
    finish(links, dims, g_last, g_next)
    tot = torch.tensor([iters], dtype=torch.int64, device=links.device)
    if world > 1:
        dist.all_reduce(tot, group=group)
    return ShardResult(int(tot.item()), th, it, restarts)
