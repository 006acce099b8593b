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
