"""Host logic of the slice-sharded Coulomb fix (glu_b200/shard.py) on two
gloo ranks on the CPU: block partition, the ring exchange of the boundary
gauge field and the completion of the last temporal links.  The GPU solver
is replaced by one with the same contract that applies a known gauge field
per slice, so the assembled links can be checked against the same
transformation applied to the whole lattice in one process."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
dist = pytest.importorskip("torch.distributed")

from glu_b200.shard import coulomb_sharded, slice_blocks  # noqa: E402
from glu_b200.workload import random_su3  # noqa: E402

DIMS = (4, 4, 2, 8)


def _links(seed=3):
    rng = np.random.default_rng(seed)
    V = int(np.prod(DIMS))
    return random_su3(V * 4, rng).reshape(V, 4, 3, 3)


def _slice_g(t, lcu):
    return random_su3(lcu, np.random.default_rng(1000 + t))


def _fwd(i, mu):
    lx, ly, lz = DIMS[:3]
    x, y, z = i % lx, (i // lx) % ly, i // (lx * ly)
    if mu == 0:
        x = (x + 1) % lx
    elif mu == 1:
        y = (y + 1) % ly
    else:
        z = (z + 1) % lz
    return x + lx * (y + ly * z)


def _transform_whole(U):
    """Every slice t rotated by g_t (periodic in t), in one process."""
    lcu = DIMS[0] * DIMS[1] * DIMS[2]
    lt = DIMS[3]
    g = [_slice_g(t, lcu) for t in range(lt)]
    out = U.copy()
    for t in range(lt):
        for i in range(lcu):
            s = t * lcu + i
            for mu in range(3):
                out[s, mu] = g[t][i] @ U[s, mu] @ g[t][_fwd(i, mu)].conj().T
            out[s, 3] = g[t][i] @ U[s, 3] @ g[(t + 1) % lt][i].conj().T
    return out


def _mock_solver(t0):
    """solve/finish with the library's contract: slice t of the block is
    rotated by g_{t0 + t}; the last slice's temporal links wait for g_next."""
    lcu = DIMS[0] * DIMS[1] * DIMS[2]

    def solve(links, dims, g_first, g_last):
        U = links.numpy().view(np.complex128).reshape(-1, 4, 3, 3)
        tb = dims[3]
        g = [_slice_g(t0 + t, lcu) for t in range(tb)]
        new = U.copy()
        for t in range(tb):
            for i in range(lcu):
                s = t * lcu + i
                for mu in range(3):
                    new[s, mu] = g[t][i] @ U[s, mu] @ g[t][_fwd(i, mu)].conj().T
                if t < tb - 1:
                    new[s, 3] = g[t][i] @ U[s, 3] @ g[t + 1][i].conj().T
        U[...] = new
        # fields of the first and last slices as double[9][Lcu][2]
        for gt, buf in ((g[0], g_first), (g[-1], g_last)):
            gf = np.ascontiguousarray(gt.reshape(lcu, 9).T)
            buf.copy_(torch.from_numpy(gf.view(np.float64).reshape(-1)))
        return tb, np.zeros(tb), np.ones(tb, dtype=np.int64), 0

    def finish(links, dims, g_last, g_next):
        U = links.numpy().view(np.complex128).reshape(-1, 4, 3, 3)
        tb = dims[3]
        gl = g_last.numpy().view(np.complex128).reshape(9, lcu).T.reshape(lcu, 3, 3)
        gn = g_next.numpy().view(np.complex128).reshape(9, lcu).T.reshape(lcu, 3, 3)
        for i in range(lcu):
            s = (tb - 1) * lcu + i
            U[s, 3] = gl[i] @ U[s, 3] @ gn[i].conj().T

    return solve, finish


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        U = _links()
        lcu = DIMS[0] * DIMS[1] * DIMS[2]
        t0, t1 = slice_blocks(DIMS[3], world)[rank]
        block = torch.from_numpy(
            np.ascontiguousarray(U[t0 * lcu:t1 * lcu]).view(np.float64).reshape(-1).copy())
        dims = (DIMS[0], DIMS[1], DIMS[2], t1 - t0)
        r = coulomb_sharded(block, dims, solver=_mock_solver(t0))
        parts = [torch.zeros(0, dtype=torch.float64) for _ in range(world)]
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(sizes, torch.tensor([block.numel()]))
        parts = [torch.zeros(int(s.item()), dtype=torch.float64) for s in sizes]
        dist.all_gather(parts, block)
        if rank == 0:
            full = torch.cat(parts).numpy().view(np.complex128).reshape(-1, 4, 3, 3)
            np.save(out, full)
            np.save(out + ".iters.npy", np.array([r.iters]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_slice_blocks_partition():
    assert slice_blocks(8, 2) == [(0, 4), (4, 8)]
    assert slice_blocks(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert slice_blocks(128, 8)[-1] == (112, 128)
    with pytest.raises(ValueError):
        slice_blocks(5, 3)


@pytest.mark.parametrize("world", [1, 2])
def test_sharded_transform_equals_whole_lattice(tmp_path, world):
    out = str(tmp_path / "full.npy")
    if world == 1:
        U = _links()
        block = torch.from_numpy(U.view(np.float64).reshape(-1).copy())
        r = coulomb_sharded(block, DIMS, solver=_mock_solver(0))
        got = block.numpy().view(np.complex128).reshape(-1, 4, 3, 3)
        iters = r.iters
    else:
        import torch.multiprocessing as mp
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        got = np.load(out)
        iters = int(np.load(out + ".iters.npy")[0])
    ref = _transform_whole(_links())
    assert np.abs(got - ref).max() < 1e-13
    assert iters == DIMS[3]  # each mock slice reports one iteration


def test_slice_blocks_by_cost_minimise_the_largest_block():
    # exact optimum of the linear partition, checked by exhaustion
    import itertools
    rng = np.random.default_rng(5)
    for lt, world in ((8, 2), (9, 3), (12, 4), (10, 2)):
        c = rng.uniform(0.2, 5.0, size=lt)
        got = slice_blocks(lt, world, c)
        assert got[0][0] == 0 and got[-1][1] == lt
        assert all(b - a >= 2 for a, b in got)
        assert all(got[i][1] == got[i + 1][0] for i in range(world - 1))
        worst = max(c[a:b].sum() for a, b in got)
        best = min(
            max(c[a:b].sum() for a, b in zip((0,) + cuts, cuts + (lt,)))
            for cuts in itertools.combinations(range(2, lt - 1), world - 1)
            if all(b - a >= 2 for a, b in zip((0,) + cuts, cuts + (lt,))))
        assert abs(worst - best) < 1e-12
    with pytest.raises(ValueError):
        slice_blocks(8, 2, np.ones(7))


COSTS = np.array([6.0, 4.0, 1.0, 1.0, 1.0, 1.0, 1.0, 5.0])  # slices of DIMS
UNIT_S = 0.05  # seconds of mock solving per unit of cost


def _timed_rank(rank, world, port, out, weighted):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import time
        U = _links()
        lcu = DIMS[0] * DIMS[1] * DIMS[2]
        t0, t1 = slice_blocks(DIMS[3], world, COSTS if weighted else None)[rank]
        block = torch.from_numpy(
            np.ascontiguousarray(U[t0 * lcu:t1 * lcu]).view(np.float64).reshape(-1).copy())
        dims = (DIMS[0], DIMS[1], DIMS[2], t1 - t0)
        solve, finish = _mock_solver(t0)

        def slow_solve(links, d, g_first, g_last):
            # a slice costs UNIT_S x its cost: uneven per-slice iterations
            time.sleep(UNIT_S * COSTS[t0:t1].sum())
            return solve(links, d, g_first, g_last)

        dist.barrier()
        start = time.perf_counter()
        coulomb_sharded(block, dims, solver=(slow_solve, finish))
        mine = torch.tensor([time.perf_counter() - start], dtype=torch.float64)
        times = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(times, mine)
        if rank == 0:
            np.save(out, np.array([float(t.item()) for t in times]))
    finally:
        dist.destroy_process_group()


def test_cost_weighted_blocks_balance_uneven_slices(tmp_path):
    """Two gloo ranks, slices of uneven cost (a mock solver whose time is
    proportional to the block's cost): the count-balanced split leaves one
    rank 12 of 20 units; the cost-weighted split gives each 10, and the
    ranks' solve times agree within 10%."""
    import torch.multiprocessing as mp
    res = {}
    for weighted in (False, True):
        out = str(tmp_path / f"t{int(weighted)}.npy")
        mp.spawn(_timed_rank, args=(2, _free_port(), out, weighted), nprocs=2, join=True)
        res[weighted] = np.load(out)
    # each rank's own time includes its wait for the boundary exchange, so
    # compare through the busier rank's time
    even, weighted = res[False], res[True]
    assert max(even) > 1.1 * max(weighted)
    blocks = slice_blocks(DIMS[3], 2, COSTS)
    costs = [COSTS[a:b].sum() for a, b in blocks]
    assert max(costs) <= 1.1 * min(costs)
